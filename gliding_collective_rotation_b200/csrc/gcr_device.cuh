// gcr_device.cuh -- device-side types and helpers of the B200 SRK2 hot path.
//
// Data layout in HBM (one context, many systems):
//   * per system, caller-owned: pos/pos1 FP64 [n,d] (AoS), tangent/forces FT
//     [n,d], chain_id int32 [n], rest_lengths FP64 [n_chains];
//   * library scratch, per system at a bead / cell offset:
//       topo      uint8 [bead]        chain-neighbour bits of each bead
//       cnt       int32 [cell]        beads binned per GPU cell (zeroed by the sort)
//       ncell     int32 [cell]        beads of each cell at the last list build
//       items     int32 [cell*depth]  bead ids per cell, sorted by id
//       nbr       int32 [slot][bead]  neighbour list, slot-major (coalesced
//                                     across the beads of a warp)
//       ncount    int32 [bead]        neighbours of each bead
//       xref      FP64 [bead][d]      positions at the last list build
//       fp, xi    FT [bead][d]        pair force and step noise per bead
//   * SysP (read-only during a step) and SysS (device-updated) per slot.
// Binning writes a fixed-depth table (a count and `depth` slots per cell, the
// shape of the reference's grid_list, updates.py:502-522); a per-cell sort
// makes the slot order deterministic; the list build walks the 3^d cells
// around each bead (the reference's update_nbor_list, updates.py:586-669,
// with a skin added to the cutoff).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gcr {

constexpr int kMaxDim = 3;
// populations coupled in one box, at most
constexpr int kMaxPops = 4;

// topology bits of a bead (same chain as b-1, b-2, b+1, b+2)
constexpr uint8_t kHasPrev = 1, kHasPrev2 = 2, kHasNext = 4, kHasNext2 = 8;

// device status flags (mirror GCR_FLAG_* in gcr.h)
// The step graph launches its kernels with programmatic dependent launch: a
// kernel may be scheduled while the one before it on the stream drains.
// Every such kernel calls this first, before touching memory: it returns
// once the previous kernel has completed and its writes are visible (at
// once when the launch was an ordinary one).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

constexpr int kFlagCellOverflow = 1;
constexpr int kFlagNonFinite = 2;
constexpr int kFlagNextOverflow = 4;
constexpr int kFlagListCorrupt = 8;  // an inconsistent cell or neighbour list was detected and not used
constexpr int kFlagListOverflow = 16;  // more list partners of a bead than the list depth
constexpr int kFlagSeriesFull = 32;    // the series buffer was full (not fatal)
// a system with one of these stops: every kernel skips it until re-armed
constexpr int kFlagFatal = kFlagCellOverflow | kFlagNonFinite | kFlagListCorrupt | kFlagListOverflow;

struct SysP {
    // caller-owned state
    double *pos;
    double *pos1;
    void *tan;
    void *frc;
    const int32_t *chain;
    const double *rest;
    const int32_t *chain_start;  // first bead of each chain (+ end), library scratch
    double *pos2;                // SRK4: positions of the second virtual update, library scratch
    void *faux;                  // SRK4: force of the current stage (pop.forces_aux)
    // scratch placement
    int64_t bead_off;  // into topo
    int64_t cell_off;  // into cnt / items / rec
    int32_t n;
    int32_t n_chains;
    int32_t nc;        // GPU cells per side
    int32_t n_cells;   // nc^d
    int32_t n_bead_tiles;
    int32_t n_cell_tiles;
    double L, half_L, h, inv_h;
    // bonded
    double k, kappa, theta0;
    int32_t calc_springs, get_orient, calc_bend, calc_wca;
    // pair (WCA / LJ: coeff = ds^-4 (p0 - p1 ds^-3))
    double p0, p1, shift, rc2;
    double rl2;         // (r_cut + skin)^2: radius of the neighbour list
    double half_skin2;  // (skin / 2)^2: a bead that moved farther forces a rebuild
    int32_t n_nearby;
    int32_t self_propel;
    int32_t rotate_prop;  // 2D and v_tan_angle != 0
    int32_t row_cells;    // cells of a row tile of the cell-staged pair kernel
    double v0, cos_a, sin_a;
    // noise / SRK
    double D, Dr, radius, sqrt2D;
    double dtmax, mdps, rk;
    double rigid;  // rigid-rod projection factor (0: off, or no chain longer than 2 beads)
    uint64_t seed;
    // populations coupled in one box (updates.py:146-247, SRK.py:166-330):
    // the members step under one dt, rebuild their lists together, and each
    // moving member feels the others through WCA pair forces over its cross
    // lists.  A fixed member (pop.fixed) never moves; its pos1/pos2 alias pos.
    int32_t fixed;
    int32_t grp_n;                // members of its group (0: not coupled)
    int32_t grp[kMaxPops];        // member slots, in population order
    int32_t n_cross;              // partner populations whose force it feels
    int32_t cross_q[kMaxPops - 1];  // partner slots, in the order the reference adds them
    int32_t cross_w[kMaxPops - 1];  // cells scanned either side in the partner's grid
    int32_t n_row_tiles;          // row tiles of the cell-staged pair kernel (0: no pair forces)
    double cross_p0[kMaxPops - 1], cross_p1[kMaxPops - 1], cross_shift[kMaxPops - 1];
    double cross_rc2[kMaxPops - 1], cross_rl2[kMaxPops - 1];
    int64_t x_off;                // first row of its cross lists
    // motors (Motor_Population, populations.py:617-661; forces.calc_motor_push,
    // forces.py:248-283): a motor population pushes the beads of the chain
    // population on its cross list motor_k; the chains add the pushes
    int32_t motor;       // 1: this system is a motor population
    int32_t motor_k;     // its cross-list index of the chains it pushes
    int32_t motor_hold;  // b_motors_dont_diffuse_while_pushing: an attached motor keeps its position
    int32_t pushed;      // 1: chains pushed by a motor population
    double mparams[5];   // motors: [motor_max_dist_sq, b_one_motor_per_bead, imparts_force, k_on, k_off]
    double push_force;   // chains: the pushing motors' imparts_force
};

struct SysS {
    double dt;          // predictor dt of the coming step (status.dt)
    double dt_next;     // dt chosen by the max-force rule this step
    double dt_used;     // corrector dt of this step
    double elapsed;     // time elapsed in the call (shared_arr[:,1])
    double mfs;         // max_forces_strength of the last step
    double max_dt_usable;
    unsigned long long max_f2;  // bit pattern of max |F|^2 (non-negative double)
    int64_t step;       // global step index (Philox counter)
    int64_t steps_done; // steps completed in the call
    int64_t max_steps;
    const double *noise;  // injected noise_vec snapshots or nullptr
    int64_t noise_steps;
    int32_t active;
    int32_t flags;
    int32_t rebuild;      // the neighbour list must be rebuilt before the next pair kernel
    int32_t pad0;
    int64_t list_builds;  // neighbour-list builds since admission
    double *series;       // order-parameter rows of the call (step, elapsed, P, S, angle) or nullptr
    int64_t series_every;
    int64_t series_phase;
    int64_t series_cap;
    int64_t series_rows;
    int64_t series_mark;  // steps_done of the last row
};

struct Tile {
    int32_t sys;
    int32_t begin;
};

// ---------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11) and the Box-Muller pair drawn from one block.
// counter = (bead, step lo, step hi, stream), key = (seed lo, seed hi).
// ---------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t lo0 = c.x * 0xD2511F53u, hi0 = __umulhi(c.x, 0xD2511F53u);
        uint32_t lo1 = c.z * 0xCD9E8D57u, hi1 = __umulhi(c.z, 0xCD9E8D57u);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// two uniforms in [0, 1) for the motor decisions of (motor, bead) at a
// stage of a step: u0 against k_off, u1 against k_on (53 bits each); the
// keyed stand-in for the reference's sequential np.random.random() draws
// (forces.py:268, 275)
__device__ __forceinline__ void motor_uniforms(uint64_t seed, uint32_t motor, uint32_t bead, int64_t step,
                                               int stage, double &u0, double &u1)
{
    uint4 r = philox4x32_10(make_uint4(motor, bead, (uint32_t)((uint64_t)step & 0xffffffffu),
                                       ((uint32_t)((uint64_t)step >> 32) & 0xffffu) | ((uint32_t)stage << 16)),
                            (uint32_t)(seed & 0xffffffffu) ^ 0x6d6f746fu, (uint32_t)(seed >> 32));
    const double two_m53 = 1.1102230246251565e-16;
    uint64_t a = (((uint64_t)r.x << 21) ^ (uint64_t)(r.y >> 11)) & ((1ull << 53) - 1);
    uint64_t b = (((uint64_t)r.z << 21) ^ (uint64_t)(r.w >> 11)) & ((1ull << 53) - 1);
    u0 = (double)a * two_m53;
    u1 = (double)b * two_m53;
}

__device__ __forceinline__ void normal_pair(uint64_t seed, uint32_t bead, int64_t step,
                                            uint32_t stream, double &z0, double &z1)
{
    uint4 r = philox4x32_10(make_uint4(bead, (uint32_t)((uint64_t)step & 0xffffffffu),
                                       (uint32_t)((uint64_t)step >> 32), stream),
                            (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
    const double two_m53 = 1.1102230246251565e-16;
    uint64_t a = (((uint64_t)r.x << 21) ^ (uint64_t)(r.y >> 11)) & ((1ull << 53) - 1);
    uint64_t b = (((uint64_t)r.z << 21) ^ (uint64_t)(r.w >> 11)) & ((1ull << 53) - 1);
    double u1 = ((double)a + 1.0) * two_m53;
    double u2 = (double)b * two_m53;
    double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincos(6.283185307179586 * u2, &s, &c);
    z0 = rad * c;
    z1 = rad * s;
}

// The same Philox block turned into two FP32 deviates (mixed precision):
// 24-bit uniforms from the top bits of the words the FP64 pair uses, and the
// Box-Muller transform in FP32 from the same 53-bit u1 as the FP64 pair:
// r.x * 2^-32 + ((r.y >> 11) + 1) * 2^-53 summed in FP32 keeps 2^-24 of
// relative precision at every magnitude, so the normals agree with the FP64
// pair to about 1e-6 relative also in the far tail (the largest |z| is
// sqrt(2 ln 2^53) = 8.57 on both sides).  A u1 of 24 bits alone would cut the
// tail at 5.77 and give tail draws (one bead in ~1e6 per step) a visibly
// different displacement from the FP64 path's.
__device__ __forceinline__ void normal_pair_f(uint64_t seed, uint32_t bead, int64_t step, uint32_t stream,
                                              float &z0, float &z1)
{
    uint4 r = philox4x32_10(make_uint4(bead, (uint32_t)((uint64_t)step & 0xffffffffu),
                                       (uint32_t)((uint64_t)step >> 32), stream),
                            (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
    const float two_m24 = 5.9604644775390625e-08f;
    const float two_m32 = 2.3283064365386963e-10f, two_m53 = 1.1102230246251565e-16f;
    // (float)r.x may round up to 2^32: u1 <= 1 keeps the log finite
    float u1 = fminf((float)r.x * two_m32 + (float)((r.y >> 11) + 1u) * two_m53, 1.0f);
    float u2 = (float)(r.z >> 8) * two_m24;
    float rad = sqrtf(-2.0f * logf(u1));
    float s, c;
    sincospif(2.0f * u2, &s, &c);
    z0 = rad * c;
    z1 = rad * s;
}

template <int D>
__device__ __forceinline__ void philox_normals_f(uint64_t seed, uint32_t bead, int64_t step, bool rot,
                                                 float out[D])
{
    float z0, z1;
    uint32_t s0 = rot ? 2u : 0u;
    normal_pair_f(seed, bead, step, s0, z0, z1);
    out[0] = z0;
    out[1] = z1;
    if (D == 3) {
        float z2, z3;
        normal_pair_f(seed, bead, step, s0 + 1u, z2, z3);
        out[D - 1] = z2;
    }
}

// translational (stream 0,1) or rotational (stream 2,3) deviates of one bead
template <int D>
__device__ __forceinline__ void philox_normals(uint64_t seed, uint32_t bead, int64_t step, bool rot,
                                               double out[D])
{
    double z0, z1;
    uint32_t s0 = rot ? 2u : 0u;
    normal_pair(seed, bead, step, s0, z0, z1);
    out[0] = z0;
    out[1] = z1;
    if (D == 3) {
        double z2, z3;
        normal_pair(seed, bead, step, s0 + 1u, z2, z3);
        out[D - 1] = z2;
    }
}

// Python float modulo: result in [0, m) with the sign of m, the wrap the
// reference applies after every update (SRK.py:387).
__device__ __forceinline__ double py_mod(double x, double m)
{
    if (x >= 0.0 && x < m) return x == 0.0 ? 0.0 : x;
    if (x < 0.0 && x >= -m) return x + m;
    if (x >= m && x < 2.0 * m) return x - m;
    double r = fmod(x, m);
    if (r != 0.0) {
        if ((m < 0.0) != (r < 0.0)) r += m;
    } else {
        r = copysign(0.0, m);
    }
    return r;
}

// CPython float floor division (float_divmod), as Numba lowers `x // h`.
__device__ __forceinline__ double py_floordiv(double x, double m)
{
    double mod = fmod(x, m);
    double div = __ddiv_rn(__dsub_rn(x, mod), m);
    if (mod != 0.0) {
        if ((m < 0.0) != (mod < 0.0)) div = __dsub_rn(div, 1.0);
    }
    double fd;
    if (div != 0.0) {
        fd = floor(div);
        if (__dsub_rn(div, fd) > 0.5) fd = __dadd_rn(fd, 1.0);
    } else {
        fd = copysign(0.0, x / m);
    }
    return fd;
}

// minimum image of a - b along one axis, forces.inbounds_diff (forces.py:44-55)
__device__ __forceinline__ double inbounds(double a, double b, double half_L, double L)
{
    double o = a - b;
    if (o < -half_L)
        o += L;
    else if (o >= half_L)
        o -= L;
    return o;
}

// periodic images crossed by one coordinate in a real update: a bead moves
// far less than half a box per step, so a jump of more than L/2 is a wrap
__device__ __forceinline__ int image_step(double x_old, double x_new, double half_L)
{
    return (x_new - x_old > half_L) ? -1 : ((x_old - x_new > half_L) ? 1 : 0);
}

// read of a word that other CTAs may change during the kernel
__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

// GPU cell coordinate of a position (clamped; non-finite -> 0)
__device__ __forceinline__ int cell_coord(double x, double inv_h, int nc)
{
    double f = floor(x * inv_h);
    int c = (f >= 0.0 && f < (double)nc) ? (int)f : (f >= (double)nc ? nc - 1 : 0);
    return c;
}

}  // namespace gcr
