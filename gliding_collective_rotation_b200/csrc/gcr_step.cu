// gcr_step.cu -- the SRK2 step kernels (sm_100a).
//
// One step of every resident system is a fixed sequence of persistent,
// grid-stride launches over per-system tile tables (one captured graph
// serves any mix of systems):
//
//   bin<A>, sort, build<A>   neighbour lists from pos, for the systems whose
//                            rebuild flag is set (the others skip at once)
//   pair<A>                  per bead: pair forces over its neighbour list
//   stage<0>                 per bead: bond, bend and tangent + pair force +
//                            self-propulsion + predictor update
//                            pos1 = (pos + dt/r F0 + sqrt(2 D dt) xi) mod L;
//                            flags a rebuild if a bead left its skin
//   bin<B>, sort, build<B>   as above, from pos1
//   pair<B>, stage<1>        the same forces at pos1 accumulated onto F0;
//                            block max of |F0+F1|^2
//   sys_dt                   per system: dt rule (SRK.py:323-353)
//   update                   per bead: corrector pos = (pos + dt_used/(2r)
//                            (F0+F1) + sqrt(2 D dt_used) xi) mod L, rotational
//                            diffusion (SRK.py:398-423); flags a rebuild if a
//                            bead left its skin
//   sys_end                  per system: step bookkeeping
//
// The same xi is used by predictor and corrector (SRK.py:134-142, 385): it is
// drawn once from the counter-based Philox stream keyed by (seed, bead,
// global step, stream), or read from an injected noise_vec snapshot, and kept
// for the corrector.
//
// Reference functions restated per bead: forces.calc_chain_spring_forces
// (forces.py:285-403), forces.central_pair_force with forces.WCA
// (forces.py:57-145, 13-15), forces.self_propel (forces.py:206-224), the
// SRK2 stage updates (SRK.py:166-184, 355-396), the cell and neighbour lists
// (updates.update_grid_list_mini, updates.update_nbor_list,
// updates.py:502-522, 586-669).
#include <type_traits>

#include "gcr_device.cuh"
#include "gcr_kernels.h"

namespace gcr {

// ------------------------------------------------------------------------
// bonded forces (forces.py:285-403).  A tile of TB beads stages the
// positions of beads begin-2 .. begin+TB+1 in shared memory, computes every
// bond (j, j+1) once and every bend once, then each bead gathers
//   F -= s_{b-1} d_{b-1}; F -= bwd_{b-1}; F += s_b d_b; F += fwd_b + bwd_b;
//   F -= fwd_{b+1}
// which is the order in which the reference's sequential loop adds them.
// ------------------------------------------------------------------------
// Arithmetic type of the bonded terms on the mixed path: FP32 by default, as
// every force; FP64 with -DGCR_BONDED_FP64=1 (8-11% more time per step).  In
// FP32 the bend is taken from the chord of the two tangents (bend()), which
// keeps the relative L2 force error against FP64 at 3.9e-6 on the 500k-bead
// LJ system (3.2e-6 with FP64 bonded terms; 1.2e-4 with the FP32 dot
// product, which cancels near c = 1).
#ifndef GCR_BONDED_FP64
#define GCR_BONDED_FP64 0
#endif
template <typename FT>
struct Bonded {
    using type = typename std::conditional<GCR_BONDED_FP64 || sizeof(FT) == 8, double, FT>::type;
};

// list pairs a lane of the warp-wide list walk evaluates per round
#ifndef GCR_PAIR_CHUNK
#define GCR_PAIR_CHUNK 2
#endif
constexpr int kPairChunk = GCR_PAIR_CHUNK;

template <int D, typename FT>
struct StageSmem {
    using BT = typename Bonded<FT>::type;
    double *x;     // [TB+4][D] positions, index k <-> bead begin-2+k
    uint8_t *tp;   // [TB+4]    topology bits
    BT *bd;        // [TB+3][D] bond vector d_j = min_image(x_j - x_{j+1}), k <-> bond begin-2+k
    BT *bt;        // [TB+3][D] unit tangent of the bond (d itself when |d| = 0)
    BT *bf;        // [TB+3]    spring magnitude k (a/|d| - 1), 0 when |d| = 0
    BT *fw;        // [TB+2][D] bend "forward" term at bead begin-1+k
    BT *bw;        // [TB+2][D] bend "backward" term
    BT *ra;        // [TB+4]    rest length of the bead's chain
    FT *pb;        // [TB/32][D+1][32 kPairChunk] the warps' buffers of the list walk (fused pair forces)
    __device__ void carve(unsigned char *base, int TB)
    {
        x = reinterpret_cast<double *>(base);
        bd = reinterpret_cast<BT *>(x + (size_t)(TB + 4) * D);
        bt = bd + (size_t)(TB + 3) * D;
        bf = bt + (size_t)(TB + 3) * D;
        fw = bf + (TB + 3);
        bw = fw + (size_t)(TB + 2) * D;
        ra = bw + (size_t)(TB + 2) * D;
        tp = reinterpret_cast<uint8_t *>(ra + (TB + 4));
        pb = reinterpret_cast<FT *>(base + ((stage_base_bytes(TB) + 15) & ~(size_t)15));
    }
    static __host__ __device__ size_t stage_base_bytes(int TB)
    {
        return (size_t)(TB + 4) * D * sizeof(double) + (size_t)(TB + 3) * (2 * D + 1) * sizeof(BT) +
               (size_t)(TB + 2) * 2 * D * sizeof(BT) + (size_t)(TB + 4) * sizeof(BT) + (size_t)(TB + 4);
    }
};

template <int D, typename FT>
size_t stage_smem_bytes(int TB)
{
    return ((StageSmem<D, FT>::stage_base_bytes(TB) + 15) & ~(size_t)15) +
           (size_t)(TB / 32) * (D + 1) * 32 * kPairChunk * sizeof(FT);
}

// 1/sqrt(x): FP64 exactly as written in the reference; FP32 (mixed path) by
// the hardware reciprocal square root (at most 2 ulp), accurate enough for
// forces that are FP32 anyway
template <typename FT>
__device__ __forceinline__ FT inv_sqrt(FT x)
{
    if constexpr (sizeof(FT) == 4)
        return rsqrtf(x);
    else
        return 1.0 / sqrt(x);
}

// bend at a bead with forward tangent ti (its own bond) and backward tangent
// tj (the previous bond); false when the tangents are aligned.  In FP64 the
// reference's formula as written; in FP32 the same function from the chord
// dv = tj - ti: 1 - c = |dv|^2 / 2, acos(c) = 2 asin(|dv| / 2),
// sqrt(1 - c^2) = sqrt((1 - c)(1 + c)), c tj - ti = dv - (1 - c) tj and
// tj - c ti = dv + (1 - c) ti.  The dot product c of two nearly aligned
// FP32 unit vectors cancels: near c = 1 its ulp (6e-8) is a relative error
// of ~1e-3..1 in 1 - c and so in the bend force of a chain straight to a few
// 1e-4 rad (measured: 2-4% force errors at such beads); the chord keeps
// FP32's relative precision at every angle.
template <int D, typename FT>
__device__ __forceinline__ bool bend(const FT *ti, const FT *tj, FT theta0, FT kappa, FT *fwd, FT *bwd)
{
    if constexpr (sizeof(FT) == 4) {
        FT dv[D];
        FT ch2 = FT(0);
#pragma unroll
        for (int i = 0; i < D; i++) {
            dv[i] = tj[i] - ti[i];
            ch2 += dv[i] * dv[i];
        }
        const FT omc = FT(0.5) * ch2;  // 1 - c
        if (!(omc > FT(0) && omc < FT(2))) return false;
        FT phi = FT(2) * asinf(FT(0.5) * sqrtf(ch2));
        if (theta0 != FT(0)) {
            FT cr = -ti[0] * tj[1] + ti[1] * tj[0];
            FT sg = (FT)((cr > FT(0)) - (cr < FT(0)));
            phi += theta0 * sg;
        }
        phi *= kappa * inv_sqrt<FT>(omc * (FT(2) - omc));
#pragma unroll
        for (int i = 0; i < D; i++) {
            fwd[i] = phi * (dv[i] - omc * tj[i]);
            bwd[i] = phi * (dv[i] + omc * ti[i]);
        }
        return true;
    }
    FT c = FT(0);
#pragma unroll
    for (int i = 0; i < D; i++) c += ti[i] * tj[i];
    if (!(FT(-1) < c && c < FT(1))) return false;
    FT phi = acos(c);
    if (theta0 != FT(0)) {
        FT cr = -ti[0] * tj[1] + ti[1] * tj[0];
        FT sg = (FT)((cr > FT(0)) - (cr < FT(0)));
        phi += theta0 * sg;
    }
    phi *= kappa * inv_sqrt<FT>(FT(1) - c * c);
#pragma unroll
    for (int i = 0; i < D; i++) {
        fwd[i] = phi * (c * tj[i] - ti[i]);
        bwd[i] = phi * (tj[i] - c * ti[i]);
    }
    return true;
}

// CTAs of 512 threads per SM that the bead kernels are compiled for: the 2D
// mixed-precision kernels fit in 42 registers a thread with 3 (6 CTAs of 256
// per SM), 64 with 2; the FP64 and 3D kernels keep the registers they need
#ifndef GCR_MIXED2D_MIN_BLOCKS
#define GCR_MIXED2D_MIN_BLOCKS 3
#endif
template <int D, typename FT>
constexpr int min_blocks()
{
    return (D == 2 && sizeof(FT) == 4) ? GCR_MIXED2D_MIN_BLOCKS : 1;
}

// ------------------------------------------------------------------------
// the pair rule forces.WCA (forces.py:13-15): coeff = ds^-4 (p0 - p1 ds^-3)
// ------------------------------------------------------------------------
template <typename FT>
__device__ __forceinline__ FT wca_coeff(FT ds, FT p0, FT p1)
{
    if constexpr (sizeof(FT) == 4) {
        // r < 0.01: ds^-7 leaves the FP32 range (overlaps of a random
        // placement); evaluate in FP64 and clamp.  The adaptive dt rule turns
        // any huge force into a step of max_dist_per_step, as in FP64.
        if (ds < 1e-4f) {
            double d = ds, inv = 1.0 / d, i2 = inv * inv;
            double c = (i2 * i2) * ((double)p0 - (double)p1 * (i2 * inv));
            c = fmin(fmax(c, -1e30), 1e30);
            return (float)c;
        }
        // ds**-4 (p0 - p1 ds**-3) from one correctly rounded reciprocal
        float inv = __fdividef(1.0f, ds);  // at most 2 ulp
        float i2 = inv * inv;
        return (i2 * i2) * (p0 - p1 * (i2 * inv));
    } else {
        double inv = 1.0 / ds, i2 = inv * inv;
        return (i2 * i2) * (p0 - p1 * (i2 * inv));
    }
}

// ------------------------------------------------------------------------
// Verlet neighbour lists.  A system's list holds, per bead, every other bead
// within r_l = r_cut + skin that the pair rule does not exclude (same chain
// and |b1 - b2| <= n_nearby, forces.py:57-145), found through a cell grid of
// side >= r_l.  It is rebuilt only when some bead has moved more than skin/2
// since the last build, so no pair can come within r_cut without being on
// the list: the producers of positions (stage 0 for pos1, the update for
// pos) test every bead against the positions of the last build and raise the
// system's rebuild flag; the list plan lists the flagged systems and clears
// their flags, and the bin, sort and build kernels run for the listed
// systems only.  Each list
// is kept in ascending bead id, so a bead's pair force is summed over the
// partners within r_cut in id order: a function of the positions alone,
// whatever the batch, the skin, the cell grid or the rebuild history.
// ------------------------------------------------------------------------

// Stages (SRK.py:166-215).  SRK2: 0 predictor, 1 corrector.  SRK4: 10..13,
// the four force evaluations.  Positions are named 0 = pos, 1 = pos1,
// 2 = pos2: the SRK4 virtual updates alternate between pos1 and pos2 so
// that no kernel reads the positions it writes (the reference writes pos1
// over itself between barriers); the caller's pos1 ends as the last virtual
// update, as in the reference.
constexpr bool srk4_stage(int S) { return S >= 10; }
// positions the forces of a stage are taken at (check_force_at_pos)
constexpr int stage_reads(int S) { return (S == 0 || S == 10) ? 0 : (S == 12 ? 2 : 1); }
// positions a stage's update writes (write_to_pos): 0 for the real update
constexpr int stage_writes(int S) { return (S == 0 || S == 10 || S == 12) ? 1 : (S == 11 ? 2 : 0); }
// dt_rescale_factor * force_prefactor of a stage's update (SRK.py:188-192, 355-360)
constexpr double stage_dt_factor(int S) { return S == 1 ? 0.5 : ((S == 10 || S == 11) ? 0.5 : 1.0); }

template <int WHICH>
__device__ __forceinline__ double *stage_x(const SysP &p)
{
    return WHICH == 0 ? p.pos : (WHICH == 1 ? p.pos1 : p.pos2);
}

// a system that k_lists_plan listed still takes part in the build (its flags
// may have turned fatal since; a fixed member of coupled populations is
// binned whenever it was listed)
__device__ __forceinline__ bool builds(const SysP &p, const SysS &s)
{
    return p.calc_wca && (p.fixed || ld_volatile(&s.active)) && !(ld_volatile(&s.flags) & kFlagFatal);
}

template <int D>
__device__ __forceinline__ void cell_of(const SysP &p, const double *x, int *ci)
{
    ci[0] = ci[1] = ci[2] = 0;
#pragma unroll
    for (int i = 0; i < D; i++) ci[i] = cell_coord(x[i], p.inv_h, p.nc);
}

// a bead moved farther than skin/2 from where the list was built
template <int D>
__device__ __forceinline__ bool left_skin_of(const SysP &p, const double *r, const double *x)
{
    double dd = 0.0;
#pragma unroll
    for (int i = 0; i < D; i++) {
        double d = inbounds(x[i], r[i], p.half_L, p.L);
        dd += d * d;
    }
    return !(dd <= p.half_skin2);
}

template <int D>
__device__ __forceinline__ bool left_skin(const SysP &p, const BatchArgs &A, int b, const double *x)
{
    const double *r = A.xref + (size_t)(p.bead_off + b) * D;
    double dd = 0.0;
#pragma unroll
    for (int i = 0; i < D; i++) {
        double d = inbounds(x[i], r[i], p.half_L, p.L);
        dd += d * d;
    }
    return !(dd <= p.half_skin2);
}

// Work list of a list build: the flagged systems, compacted, with the
// running sum of their bead tiles and cell tiles.  Layout of A.work:
//   [0] flagged systems m, [1] their bead tiles, [2] their cell tiles,
//   then sys[S], bead_prefix[S+1], cell_prefix[S+1] (S = slot count).
// Built by one CTA before each stage's list kernels, which then visit the
// tiles of flagged systems only, and leave at once when there are none.
struct Work {
    int m, n_bead, n_cell;
    const int *sys, *bead0, *cell0;
};

__device__ __forceinline__ Work work_list(const BatchArgs &A)
{
    Work w;
    const int *q = A.work;
    w.m = q[0];
    w.n_bead = q[1];
    w.n_cell = q[2];
    w.sys = q + 3;
    w.bead0 = w.sys + A.n_slots;
    w.cell0 = w.bead0 + A.n_slots + 1;
    return w;
}

// the flagged system holding work item i of a prefix (largest k: pre[k] <= i)
__device__ __forceinline__ int work_owner(const int *pre, int m, int i)
{
    int lo = 0, hi = m - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// one CTA: compact the systems that take part in a list build now
__global__ void __launch_bounds__(1024) k_lists_plan(BatchArgs A)
{
    pdl_wait();
    __shared__ int sh[3][32];
    __shared__ int carry[3];
    int *q = A.work;
    int *wsys = q + 3, *wb = wsys + A.n_slots, *wc = wb + A.n_slots + 1;
    if (threadIdx.x < 3) carry[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < A.n_slots; base += blockDim.x) {
        const int i = base + threadIdx.x;
        int v[3] = {0, 0, 0};
        if (i < A.n_slots) {
            const SysP &p = A.P[i];
            const SysS &st = A.S[i];
            bool part = false;
            if (p.calc_wca && !(st.flags & kFlagFatal)) {
                if (p.grp_n == 0) {
                    part = st.active && st.rebuild;
                } else {
                    // coupled populations rebuild together: their cross lists
                    // read one another's cells.  Only moving, running members
                    // ask for a build (no flag changes during the scan, so
                    // every thread of the group reaches the same answer).
                    bool any = false;
                    for (int k = 0; k < p.grp_n && k < kMaxPops; k++) {
                        const int m = p.grp[k];
                        if (m < 0 || m >= A.n_slots) continue;
                        const SysS &sm = A.S[m];
                        any |= !A.P[m].fixed && sm.active && sm.rebuild && !(sm.flags & kFlagFatal);
                    }
                    part = any && (p.fixed || st.active);
                }
            }
            if (part) {
                v[0] = 1;
                v[1] = p.n_bead_tiles;
                v[2] = p.n_cell_tiles;
            }
        }
        int x[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[c] = v[c];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x[c], o);
                if (lane >= o) x[c] += y;
            }
            if (lane == 31) sh[c][wid] = x[c];
        }
        __syncthreads();
        if (wid == 0) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                int y = lane < nw ? sh[c][lane] : 0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int z = __shfl_up_sync(0xffffffffu, y, o);
                    if (lane >= o) y += z;
                }
                if (lane < nw) sh[c][lane] = y;  // inclusive prefix of warp totals
            }
        }
        __syncthreads();
        int ex[3];
#pragma unroll
        for (int c = 0; c < 3; c++) ex[c] = carry[c] + x[c] - v[c] + (wid > 0 ? sh[c][wid - 1] : 0);
        if (v[0]) {
            wsys[ex[0]] = i;
            wb[ex[0]] = ex[1];
            wc[ex[0]] = ex[2];
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
#pragma unroll
            for (int c = 0; c < 3; c++) carry[c] = ex[c] + v[c];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        q[0] = carry[0];
        q[1] = carry[1];
        q[2] = carry[2];
        wb[carry[0]] = carry[1];
        wc[carry[0]] = carry[2];
    }
    // the listed systems' flags are consumed: a stage kernel that finds a bead
    // outside its skin raises the flag again for the next build (kernels
    // later in this stage never clear it, so no raise can be lost)
    for (int k = threadIdx.x; k < carry[0]; k += blockDim.x) A.S[wsys[k]].rebuild = 0;
}

// bin every bead of a flagged system into its cell (fixed-depth slots)
template <int D, int WHICH>
__global__ void __launch_bounds__(512) k_bin(BatchArgs A)
{
    pdl_wait();
    const Work w = work_list(A);
    for (int t = blockIdx.x; t < w.n_bead; t += gridDim.x) {
        const int k = work_owner(w.bead0, w.m, t);
        const int sys = w.sys[k];
        const SysP &p = A.P[sys];
        SysS &s = A.S[sys];
        if (!builds(p, s)) continue;
        const int b = (t - w.bead0[k]) * A.tile_beads + threadIdx.x;
        if (b >= p.n || threadIdx.x >= A.tile_beads) continue;
        const double *X = stage_x<WHICH>(p);
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < D; i++) x[i] = X[(size_t)b * D + i];
        int ci[3];
        cell_of<D>(p, x, ci);
        const int64_t gc = p.cell_off + ((int64_t)ci[2] * p.nc + ci[1]) * p.nc + ci[0];
        const int slot = atomicAdd(A.cnt + gc, 1);
        if (slot < A.depth)
            A.items[(gc << A.log_depth) + slot] = b;
        else
            atomicOr(&s.flags, kFlagCellOverflow);
    }
}

// per cell of a flagged system: take the count (and zero it for the next
// binning), sort the slot contents by bead id
__global__ void __launch_bounds__(512) k_sort(BatchArgs A)
{
    pdl_wait();
    const Work w = work_list(A);
    for (int t = blockIdx.x; t < w.n_cell; t += gridDim.x) {
        const int k = work_owner(w.cell0, w.m, t);
        const int sys = w.sys[k];
        const SysP &p = A.P[sys];
        SysS &s = A.S[sys];
        if (!builds(p, s)) continue;
        const int c = (t - w.cell0[k]) * A.tile_cells + threadIdx.x;
        if (c >= p.n_cells || threadIdx.x >= A.tile_cells) continue;
        const int64_t gc = p.cell_off + c;
        int n = A.cnt[gc];
        A.cnt[gc] = 0;
        n = n < 0 ? 0 : (n < A.depth ? n : A.depth);
        A.ncell[gc] = n;
        if (n < 2) continue;
        int *it = A.items + (gc << A.log_depth);
        if (n <= 8) {
            int v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = j < n ? it[j] : 0x7fffffff;
            // Batcher odd-even merge sort network for 8 keys (19 comparators)
#define GCR_CX(a, b)                 \
    {                                \
        int lo = min(v[a], v[b]);    \
        int hi = max(v[a], v[b]);    \
        v[a] = lo;                   \
        v[b] = hi;                   \
    }
            GCR_CX(0, 1) GCR_CX(2, 3) GCR_CX(4, 5) GCR_CX(6, 7)
            GCR_CX(0, 2) GCR_CX(1, 3) GCR_CX(4, 6) GCR_CX(5, 7)
            GCR_CX(1, 2) GCR_CX(5, 6)
            GCR_CX(0, 4) GCR_CX(1, 5) GCR_CX(2, 6) GCR_CX(3, 7)
            GCR_CX(2, 4) GCR_CX(3, 5)
            GCR_CX(1, 2) GCR_CX(3, 4) GCR_CX(5, 6)
#undef GCR_CX
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (j < n) it[j] = v[j];
        } else {
            // insertion sort in place (cells this dense are rare)
            for (int j = 1; j < n; j++) {
                int key = it[j];
                int q = j - 1;
                while (q >= 0 && it[q] > key) {
                    it[q + 1] = it[q];
                    q--;
                }
                it[q + 1] = key;
            }
        }
    }
}

// cross list c of bead b of a coupled population: every bead of partner
// population q within its cross list radius, found through q's cell grid
// (binned in the same list build), in ascending id -- the partner's own
// nbor_list row of the reference (populations.py:156-180, updates.py:586-669
// with pop2 another population: no chain exclusion)
template <int D, int WHICH>
__device__ void build_cross(const BatchArgs &A, const SysP &p, SysS &s, int c, int b, const double *x)
{
    const int qs = p.cross_q[c];
    if (qs < 0 || qs >= A.n_slots) {
        atomicOr(&s.flags, kFlagListCorrupt);
        return;
    }
    const SysP &q = A.P[qs];
    const double *XQ = stage_x<WHICH>(q);
    const int nq = q.n, nc = q.nc, wnd = p.cross_w[c];
    const double rl2 = p.cross_rl2[c];
    int ci[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < D; i++) ci[i] = cell_coord(x[i], q.inv_h, nc);
    // cells either side; a window as wide as the grid visits every cell once
    const bool all = 2 * wnd + 1 >= nc;
    const int lo = all ? 0 : -wnd, hi = all ? nc - 1 : wnd;
    const int64_t row = p.x_off + (int64_t)c * p.n + b;
    int *out = A.xnbr + row;
    const int64_t stride = A.xstride;
    const int cap = A.list_depth;
    int cnt = 0;
    bool bad = false;
    const int zlo = (D == 3) ? lo : 0, zhi = (D == 3) ? hi : 0;
    for (int dz = zlo; dz <= zhi; dz++) {
        int cz = 0;
        if (D == 3) {
            cz = all ? dz : ci[2] + dz;
            cz = ((cz % nc) + nc) % nc;
        }
        for (int dy = lo; dy <= hi; dy++) {
            int cy = all ? dy : ci[1] + dy;
            cy = ((cy % nc) + nc) % nc;
            for (int dx = lo; dx <= hi; dx++) {
                int cx = all ? dx : ci[0] + dx;
                cx = ((cx % nc) + nc) % nc;
                const int64_t gc = q.cell_off + ((int64_t)cz * nc + cy) * nc + cx;
                int m = A.ncell[gc];
                m = m < 0 ? 0 : (m < A.depth ? m : A.depth);
                const int *it = A.items + (gc << A.log_depth);
                for (int k = 0; k < m; k++) {
                    const int j = it[k];
                    if ((unsigned)j >= (unsigned)nq) {
                        bad = true;
                        continue;
                    }
                    double ds = 0.0;
#pragma unroll
                    for (int i = 0; i < D; i++) {
                        double d = inbounds(XQ[(size_t)j * D + i], x[i], p.half_L, p.L);
                        ds += d * d;
                    }
                    if (ds <= rl2) {
                        if (cnt < cap) {
                            int q2 = cnt;
                            while (q2 > 0) {
                                const int prev = out[(size_t)(q2 - 1) * stride];
                                if (prev < j) break;
                                out[(size_t)q2 * stride] = prev;
                                q2--;
                            }
                            out[(size_t)q2 * stride] = j;
                        }
                        cnt++;
                    }
                }
            }
        }
    }
    A.xcount[row] = cnt < cap ? cnt : cap;
    if (cnt > cap) atomicOr(&s.flags, kFlagListOverflow);
    if (bad) atomicOr(&s.flags, kFlagListCorrupt);
}

// per bead of a flagged system: every non-excluded bead within r_l in the
// 3^d cells around it, in ascending id; records the positions of the build
template <int D, int WHICH>
__global__ void __launch_bounds__(512) k_build(BatchArgs A)
{
    pdl_wait();
    const Work w = work_list(A);
    for (int t = blockIdx.x; t < w.n_bead; t += gridDim.x) {
        const int k = work_owner(w.bead0, w.m, t);
        const int sys = w.sys[k];
        const SysP &p = A.P[sys];
        SysS &s = A.S[sys];
        // a fixed population is only binned: it feels no force and never moves
        if (!builds(p, s) || p.fixed) continue;
        const int begin = (t - w.bead0[k]) * A.tile_beads;
        if (begin == 0 && threadIdx.x == 0) s.list_builds += 1;  // one thread per system and build
        const int b = begin + threadIdx.x;
        if (b >= p.n || threadIdx.x >= A.tile_beads) continue;
        const int n = p.n, nc = p.nc;
        const double *X = stage_x<WHICH>(p);
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < D; i++) x[i] = X[(size_t)b * D + i];
        int ci[3];
        cell_of<D>(p, x, ci);
        // excluded partners: the beads of b's chain within n_nearby of b (all
        // of them when n_nearby < 0); chains are contiguous bead ranges
        int ch = p.chain[b];
        ch = ch < 0 ? 0 : (ch >= p.n_chains ? p.n_chains - 1 : ch);
        const int c_lo = p.chain_start[ch], c_hi = p.chain_start[ch + 1] - 1;
        const int nn = p.n_nearby;
        const int ex_lo = nn < 0 ? c_lo : max(c_lo, b - nn);
        const int ex_hi = nn < 0 ? c_hi : min(c_hi, b + nn);
        int *out = A.nbr + p.bead_off + b;
        const int64_t stride = A.list_stride;
        const int cap = A.list_depth;
        int cnt = 0;
        bool bad = false;
        // a motor needs only its cross list (the chain beads it may push)
        const int zlo = (D == 3) ? -1 : 0, zhi = p.motor ? zlo - 1 : ((D == 3) ? 1 : 0);
        for (int dz = zlo; dz <= zhi; dz++) {
            int cz = 0;
            if (D == 3) {
                cz = ci[2] + dz;
                cz = cz < 0 ? cz + nc : (cz >= nc ? cz - nc : cz);
            }
            for (int dy = -1; dy <= 1; dy++) {
                int cy = ci[1] + dy;
                cy = cy < 0 ? cy + nc : (cy >= nc ? cy - nc : cy);
                for (int dx = -1; dx <= 1; dx++) {
                    int cx = ci[0] + dx;
                    cx = cx < 0 ? cx + nc : (cx >= nc ? cx - nc : cx);
                    const int64_t gc = p.cell_off + ((int64_t)cz * nc + cy) * nc + cx;
                    int m = A.ncell[gc];
                    m = m < 0 ? 0 : (m < A.depth ? m : A.depth);
                    const int *it = A.items + (gc << A.log_depth);
                    for (int q = 0; q < m; q++) {
                        const int j = it[q];
                        if ((unsigned)j >= (unsigned)n) {
                            bad = true;  // never index outside the system
                            continue;
                        }
                        if (j >= ex_lo && j <= ex_hi) continue;  // b itself is in this range
                        double ds = 0.0;
#pragma unroll
                        for (int i = 0; i < D; i++) {
                            double d = inbounds(X[(size_t)j * D + i], x[i], p.half_L, p.L);
                            ds += d * d;
                        }
                        if (ds <= p.rl2) {
                            if (cnt < cap) {
                                // insert in ascending bead id: the pair sum then
                                // depends on the positions only, not on when
                                // or on which cell grid the list was built
                                int q2 = cnt;
                                while (q2 > 0) {
                                    const int prev = out[(size_t)(q2 - 1) * stride];
                                    if (prev < j) break;
                                    out[(size_t)q2 * stride] = prev;
                                    q2--;
                                }
                                out[(size_t)q2 * stride] = j;
                            }
                            cnt++;
                        }
                    }
                }
            }
        }
        A.ncount[p.bead_off + b] = cnt < cap ? cnt : cap;
        double *r = A.xref + (size_t)(p.bead_off + b) * D;
#pragma unroll
        for (int i = 0; i < D; i++) r[i] = x[i];
        if (cnt > cap) atomicOr(&s.flags, kFlagListOverflow);
        if (bad) atomicOr(&s.flags, kFlagListCorrupt);
        for (int c = 0; c < p.n_cross && c < kMaxPops - 1; c++) build_cross<D, WHICH>(A, p, s, c, b, x);
    }
}

// pair forces between coupled populations: the force on bead b of one
// population from the beads of each other population (central_pair_force
// over the cross nbor_list with other_pop another population,
// SRK.py:229-245; the pair parameters of interpop_forces,
// updates.py:274-312; rule forces.WCA), added after the bead's own pair
// force, partner by partner in the order the reference adds the other
// populations' forces (SRK.py:287-294).  Only the pair kernels of a graph
// holding coupled populations carry it.
template <int D, typename FT, int WHICH>
__device__ __forceinline__ void add_cross(const BatchArgs &A, const SysP &p, int b, const double *xb, FT *F,
                                          bool &bad)
{
    for (int c = 0; c < p.n_cross && c < kMaxPops - 1; c++) {
        const int qs = p.cross_q[c];
        if ((unsigned)qs >= (unsigned)A.n_slots) {
            bad = true;
            continue;
        }
        const SysP &q = A.P[qs];
        const double *XQ = stage_x<WHICH>(q);
        const int nq = q.n;
        const int64_t row = p.x_off + (int64_t)c * p.n + b;
        int cnt = A.xcount[row];
        cnt = cnt < 0 ? 0 : (cnt < A.list_depth ? cnt : A.list_depth);
        const FT rc2 = (FT)p.cross_rc2[c], p0 = (FT)p.cross_p0[c], p1 = (FT)p.cross_p1[c];
        const FT shift = (FT)p.cross_shift[c];
        for (int k = 0; k < cnt; k++) {
            const int j = A.xnbr[row + (int64_t)k * A.xstride];
            if ((unsigned)j >= (unsigned)nq) {
                bad = true;
                continue;
            }
            FT sep[3];
            FT ds = FT(0);
#pragma unroll
            for (int i = 0; i < D; i++) {
                sep[i] = (FT)inbounds(XQ[(size_t)j * D + i], xb[i], p.half_L, p.L);
                ds += sep[i] * sep[i];
            }
            if (!(FT(0) < ds && ds <= rc2)) continue;
            if (shift != FT(0)) {
                FT mag = sqrt(ds);
                FT nm = mag + shift;
                nm = nm < FT(0) ? FT(0) : nm;
                FT rs = nm / mag;
#pragma unroll
                for (int i = 0; i < D; i++) sep[i] *= rs;
                ds = nm * nm;
            }
            FT coeff = wca_coeff<FT>(ds, p0, p1);
#pragma unroll
            for (int i = 0; i < D; i++) F[i] += sep[i] * coeff;
        }
    }
}

// one pair of the rule forces.WCA (forces.py:57-145): min-image separation
// of the FP64 positions xj - xb, rounded to FT, then the rule in FT, added to
// F when 0 < r^2 <= r_cut^2 (with the optional shift rescale, 123-131)
template <int D, typename FT>
__device__ __forceinline__ bool pair_coeff(const SysP &p, const double *xj, const double *xb, FT rc2, FT p0, FT p1,
                                           FT shift, FT *sep, FT &coeff)
{
    FT ds = FT(0);
#pragma unroll
    for (int i = 0; i < D; i++) {
        sep[i] = (FT)inbounds(xj[i], xb[i], p.half_L, p.L);
        ds += sep[i] * sep[i];
    }
    const bool in = FT(0) < ds && ds <= rc2;
    if (shift != FT(0)) {
        if (!in) return false;
        FT mag = sqrt(ds);
        FT nm = mag + shift;
        nm = nm < FT(0) ? FT(0) : nm;
        FT rs = nm / mag;
#pragma unroll
        for (int i = 0; i < D; i++) sep[i] *= rs;
        ds = nm * nm;
    }
    // without a shift, branch-free: a pair outside the cutoff takes the
    // (finite) coefficient at r_c, which the caller does not use
    coeff = wca_coeff<FT>(in ? ds : rc2, p0, p1);
    return in;
}

template <int D, typename FT>
__device__ __forceinline__ void pair_term(const SysP &p, const double *xj, const double *xb, FT rc2, FT p0, FT p1,
                                          FT shift, FT *F)
{
    FT sep[3], coeff;
    const bool in = pair_coeff<D, FT>(p, xj, xb, rc2, p0, p1, shift, sep, coeff);
    // a pair outside the cutoff adds sep * 0: F unchanged, bit for bit (F
    // starts at +0 and a sum never turns it into -0)
    coeff = in ? coeff : FT(0);
#pragma unroll
    for (int i = 0; i < D; i++) F[i] += sep[i] * coeff;
}

// The pair forces of the 32 beads of a warp over their neighbour lists, each
// bead's partners in ascending id (an entry outside the system sets `bad`
// and is not used).  When the warp's pairs fill
// more than one round of the flattened walk below, the list rows that keep at
// least kRowBusy lanes busy (row k: the lanes whose count exceeds k) are
// walked bead by bead, one lane per bead (a walked row costs half the instructions of
// a flattened one, but its gathers wait on one another: for short lists one
// flattened round is faster).  The rest -- the tails of the longer lists --
// is flattened: those (bead, list entry) pairs are numbered bead by bead (a
// warp scan of the remaining counts) and each lane evaluates pairs q = lane,
// lane + 32, ..., kPairChunk of them in flight at a time, every lane busy
// whatever the spread of the list lengths.  A lane finds the owner of its pair
// by a binary search over the warp's exclusive prefix (owner = last lane whose
// prefix <= q).  The pair terms (separation and coefficient, zero outside the
// cutoff) go to the warp's shared buffer and each owner then adds its own in
// ascending list order after its walked rows, F += sep * coeff as the serial
// walk does: the same sums, bit for bit.  A flattened pair costs about two
// walked rows' instructions (search, shuffles, hand-back), hence kRowBusy 16.
#ifndef GCR_PAIR_ROW_BUSY
#define GCR_PAIR_ROW_BUSY 16
#endif
#ifndef GCR_PAIR3D_MIN_BLOCKS
#define GCR_PAIR3D_MIN_BLOCKS 2
#endif
constexpr int kRowBusy = GCR_PAIR_ROW_BUSY;

template <int D, typename FT>
size_t pair_smem_bytes(int TB)
{
    return (size_t)(TB / 32) * (D + 1) * 32 * kPairChunk * sizeof(FT);
}

template <int D, typename FT>
__device__ __forceinline__ void warp_list_pair_force(const BatchArgs &A, const SysP &p, const double *X,
                                                     const double *xb, int b, int cnt, FT *F, bool &bad, FT *buf)
{
    constexpr unsigned kAll = 0xffffffffu;
    constexpr int C = kPairChunk, Q = 32 * C;
    const int lane = threadIdx.x & 31;
    cnt = cnt < 0 ? 0 : (cnt < A.list_depth ? cnt : A.list_depth);
    const int n = p.n;
    const int64_t stride = A.list_stride;
    const FT rc2 = (FT)p.rc2, p0 = (FT)p.p0, p1 = (FT)p.p1, shift = (FT)p.shift;
    // the busy rows, walked bead by bead
    int rows = 0;
    if (__reduce_add_sync(kAll, (unsigned)cnt) > (unsigned)Q)
        while (rows < A.list_depth && __popc(__ballot_sync(kAll, cnt > rows)) >= kRowBusy) rows++;
    {
        const int m = cnt < rows ? cnt : rows;
        const int *nb = A.nbr + p.bead_off + b;
        int j_next = m > 0 ? nb[0] : 0;
        for (int k = 0; k < m; k++) {
            const int j = j_next;
            if (k + 1 < m) j_next = nb[(size_t)(k + 1) * stride];
            if ((unsigned)j >= (unsigned)n) {
                bad = true;
                continue;
            }
            pair_term<D, FT>(p, X + (size_t)j * D, xb, rc2, p0, p1, shift, F);
        }
    }
    // the tails, flattened
    cnt = cnt > rows ? cnt - rows : 0;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += v;
    }
    const int excl = incl - cnt;
    const int total = __shfl_sync(kAll, incl, 31);
    const int *nb0 = A.nbr + p.bead_off + (b - lane) + (size_t)rows * stride;
    for (int base = 0; base < total; base += Q) {
        int own[C], j[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int q = base + 32 * c + lane;
            int lo = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (__shfl_sync(kAll, excl, lo + step) <= q) lo += step;
            own[c] = lo;
            const int k = q - __shfl_sync(kAll, excl, lo);
            j[c] = q < total ? nb0[lo + (size_t)k * stride] : 0;
        }
        double xj[C][3];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool ok = base + 32 * c + lane < total && (unsigned)j[c] < (unsigned)n;
#pragma unroll
            for (int i = 0; i < D; i++) xj[c][i] = ok ? X[(size_t)j[c] * D + i] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int q = base + 32 * c + lane;
            double xo[3];
#pragma unroll
            for (int i = 0; i < D; i++) xo[i] = __shfl_sync(kAll, xb[i], own[c]);
            FT sep[3] = {FT(0), FT(0), FT(0)}, coeff = FT(0);
            if (q < total) {
                if ((unsigned)j[c] >= (unsigned)n) {
                    bad = true;
                } else if (!pair_coeff<D, FT>(p, xj[c], xo, rc2, p0, p1, shift, sep, coeff)) {
#pragma unroll
                    for (int i = 0; i < D; i++) sep[i] = FT(0);
                    coeff = FT(0);
                }
            }
#pragma unroll
            for (int i = 0; i < D; i++) buf[i * Q + 32 * c + lane] = sep[i];
            buf[D * Q + 32 * c + lane] = coeff;
        }
        __syncwarp();
        const int q0 = excl > base ? excl : base, q1 = incl < base + Q ? incl : base + Q;
        for (int q = q0; q < q1; q++) {
            const FT cf = buf[D * Q + q - base];
#pragma unroll
            for (int i = 0; i < D; i++) F[i] += buf[i * Q + q - base] * cf;
        }
        __syncwarp();
    }
}

// resident CTAs of 512 threads the pair kernel is compiled for: the 3D mixed
// kernel is held to 64 registers (1024 threads per SM; unbounded it takes 96
// and four fewer 128-bead CTAs fit)
template <int D, typename FT>
constexpr int pair_min_blocks()
{
    return (D == 3 && sizeof(FT) == 4) ? GCR_PAIR3D_MIN_BLOCKS : min_blocks<D, FT>();
}

// pair forces of every bead (the list walk above, then the coupled
// populations' cross lists); writes them to fp[bead]
template <int D, typename FT, int WHICH, bool CROSS>
__global__ void __launch_bounds__(512, pair_min_blocks<D, FT>()) k_pair(BatchArgs A)
{
    pdl_wait();
    extern __shared__ __align__(16) unsigned char pair_smem[];
    FT *wbuf = reinterpret_cast<FT *>(pair_smem) + (size_t)(threadIdx.x >> 5) * (D + 1) * 32 * kPairChunk;
    const int nt = *A.n_bead_tiles;
    // the next tile's table entry is loaded while the current tile runs
    Tile nx = (int)blockIdx.x < nt ? A.bead_tiles[blockIdx.x] : Tile{0, 0};
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = nx;
        if (t + (int)gridDim.x < nt) nx = A.bead_tiles[t + gridDim.x];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        const int b = tl.begin + threadIdx.x;
        const bool valid = b < p.n && threadIdx.x < A.tile_beads;
        // the bead's own position and list count are loaded (from a valid
        // bead of the tile, whatever the lane) together with the system's
        // state; plain loads: only the per-system kernel between steps
        // changes `active`, and a fatal flag raised meanwhile costs one
        // wasted tile at most
        const int bc = valid ? b : tl.begin;
        const double *X = stage_x<WHICH>(p);
        double xb[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < D; i++) xb[i] = X[(size_t)bc * D + i];
        const int cnt = A.ncount[p.bead_off + bc];
        // block-uniform: every lane of a warp reaches the warp-wide walk
        if (!s.active || (s.flags & kFlagFatal) || !p.calc_wca) continue;
        FT F[3] = {FT(0), FT(0), FT(0)};
        bool bad = false;
        // motors have no pair force of their own (their zero-strength WCA
        // only bins them) and no list of one another
        warp_list_pair_force<D, FT>(A, p, X, xb, b, valid && !p.motor ? cnt : 0, F, bad, wbuf);
        // a motor's cross list is its candidate beads, not a force
        if constexpr (CROSS)
            if (valid && !p.motor) add_cross<D, FT, WHICH>(A, p, b, xb, F, bad);
        if (bad) atomicOr(&s.flags, kFlagListCorrupt);
        if (!valid) continue;
        FT *fp = reinterpret_cast<FT *>(A.fp) + (size_t)(p.bead_off + b) * D;
#pragma unroll
        for (int i = 0; i < D; i++) fp[i] = F[i];
    }
}

// ------------------------------------------------------------------------
// cell-staged pair forces (gcr_config.pair_mode = 2: SRK2 without coupled
// populations).  Instead of each bead gathering its list partners, a CTA
// takes a row tile -- the cells x0 .. x0+w-1 of one row (y, z) of a
// system's GPU grid -- and copies the beads of those cells and of their
// neighbour cells (3 rows in 2D, 9 in 3D; columns x0-1 .. x0+w) into shared
// memory, bead ids and FP64 positions, compacted by a block-wide scan of the
// cell counts.  Each bead of the tile then walks the beads of its 3^d
// neighbour cells there.  The cells are those of the last list build: a
// cell is at least r_cut + skin wide and no bead has moved skin/2 since, so
// every pair within r_cut is among them (the argument that makes the lists
// complete).  The pair sum runs cell by cell -- rows (dz, dy) ascending, then
// the three columns, each cell in ascending id -- so it has the list walk's
// pairs in another order: the forces differ from the list path's in FP
// rounding only.  A tile with more beads than the staging capacity reads
// the same beads from global memory in the same order.
// ------------------------------------------------------------------------
constexpr int kMaxRowCells = 128;

// exclusive prefix sum of a[0..n) in shared memory, in place; returns the
// total.  Every thread of the CTA calls it (blockDim.x a multiple of 32).
__device__ int block_exclusive_scan(int *a, int n, int *warp_sums)
{
    const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int lo = threadIdx.x * per, hi = min(n, lo + per);
    int sum = 0;
    for (int k = lo; k < hi; k++) sum += a[k];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int y = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int z = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += z;
        }
        if (lane < nw) warp_sums[lane] = y;  // inclusive prefix of the warp totals
    }
    __syncthreads();
    int run = x - sum + (wid > 0 ? warp_sums[wid - 1] : 0);
    const int total = warp_sums[nw - 1];
    for (int k = lo; k < hi; k++) {
        const int v = a[k];
        a[k] = run;
        run += v;
    }
    __syncthreads();
    return total;
}

// largest q in [0, n) with off[q] <= k (off non-decreasing, off[0] <= k)
__device__ __forceinline__ int cell_of_slot(const int *off, int n, int k)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int D, typename FT, int WHICH>
__global__ void __launch_bounds__(512) k_pair_cells(BatchArgs A)
{
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int R = D == 3 ? 9 : 3;  // rows of a tile with its neighbour rows
    __shared__ int off[R * (kMaxRowCells + 2) + 1];
    __shared__ int warp_sums[32];
    __shared__ int sh_run;
    const int cap = A.cell_stage_cap;
    double *xs = reinterpret_cast<double *>(smem_raw);            // [cap][D]
    int *ids = reinterpret_cast<int *>(xs + (size_t)cap * D);      // [cap]
    const int nt = A.row_prefix[A.n_slots];
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int sys = work_owner(A.row_prefix, A.n_slots, t);
        const Tile tl{sys, t - A.row_prefix[sys]};
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        __syncthreads();  // the previous tile is done with shared memory
        // one decision per CTA (every thread must reach the same barriers)
        if (threadIdx.x == 0)
            sh_run = ld_volatile(&s.active) && !(ld_volatile(&s.flags) & kFlagFatal) && p.calc_wca;
        __syncthreads();
        if (!sh_run) continue;
        const int nc = p.nc;
        const int T = max(1, min(p.row_cells, kMaxRowCells));
        const int segs = (nc + T - 1) / T;
        const int row = tl.begin / segs;
        const int x0 = (tl.begin - row * segs) * T;
        const int w = min(T, nc - x0), W = w + 2;
        const int ry = row % nc, rz = (D == 3) ? row / nc : 0;
        // staged cell q = r W + c: row r = 3 (dz + 1) + (dy + 1), column x0 - 1 + c
        auto cell_at = [&](int q) -> int64_t {
            const int r = q / W, c = q - r * W;
            int cx = x0 - 1 + c;
            cx = cx < 0 ? cx + nc : (cx >= nc ? cx - nc : cx);
            int cy = ry + (r % 3) - 1;
            cy = cy < 0 ? cy + nc : (cy >= nc ? cy - nc : cy);
            int cz = 0;
            if (D == 3) {
                cz = rz + r / 3 - 1;
                cz = cz < 0 ? cz + nc : (cz >= nc ? cz - nc : cz);
            }
            return p.cell_off + ((int64_t)cz * nc + cy) * nc + cx;
        };
        const int nq = R * W;
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            const int m = A.ncell[cell_at(q)];
            off[q] = m < 0 ? 0 : (m < A.depth ? m : A.depth);
        }
        __syncthreads();
        const int total = block_exclusive_scan(off, nq, warp_sums);
        if (threadIdx.x == 0) off[nq] = total;
        __syncthreads();
        const bool staged = total <= cap;
        const double *__restrict__ X = stage_x<WHICH>(p);
        const int n = p.n;
        bool bad = false;
        if (staged) {
            for (int k = threadIdx.x; k < total; k += blockDim.x) {
                const int q = cell_of_slot(off, nq, k);
                const int j = A.items[(cell_at(q) << A.log_depth) + (k - off[q])];
                const bool ok = (unsigned)j < (unsigned)n;
                bad |= !ok;
                ids[k] = ok ? j : -1;
#pragma unroll
                for (int i = 0; i < D; i++) xs[(size_t)k * D + i] = ok ? X[(size_t)j * D + i] : 0.0;
            }
            __syncthreads();
        }
        // the tile's own beads: centre row (dz = dy = 0), columns 1 .. w
        const int rmid = (R - 1) / 2;
        const int i_lo = off[rmid * W + 1], i_hi = off[rmid * W + 1 + w];
        const FT rc2 = (FT)p.rc2, p0 = (FT)p.p0, p1 = (FT)p.p1, shift = (FT)p.shift;
        for (int k = i_lo + threadIdx.x; k < i_hi; k += blockDim.x) {
            const int q = cell_of_slot(off, nq, k);
            const int c = q - rmid * W;  // column of the bead's cell in the tile, 1 .. w
            int b;
            double xb[3] = {0.0, 0.0, 0.0};
            if (staged) {
                b = ids[k];
            } else {
                b = A.items[(cell_at(q) << A.log_depth) + (k - off[q])];
            }
            if ((unsigned)b >= (unsigned)n) {
                bad = true;
                continue;
            }
#pragma unroll
            for (int i = 0; i < D; i++) xb[i] = staged ? xs[(size_t)k * D + i] : X[(size_t)b * D + i];
            // excluded partners, as the list build excludes them
            int ch = p.chain[b];
            ch = ch < 0 ? 0 : (ch >= p.n_chains ? p.n_chains - 1 : ch);
            const int c_lo = p.chain_start[ch], c_hi = p.chain_start[ch + 1] - 1;
            const int nn = p.n_nearby;
            const int ex_lo = nn < 0 ? c_lo : max(c_lo, b - nn);
            const int ex_hi = nn < 0 ? c_hi : min(c_hi, b + nn);
            FT F[3] = {FT(0), FT(0), FT(0)};
            for (int r = 0; r < R; r++) {
                const int q0 = r * W + c - 1;
                if (staged) {
                    const int k_hi = off[q0 + 3];
                    for (int kk = off[q0]; kk < k_hi; kk++) {
                        const int j = ids[kk];
                        if (j < 0 || (j >= ex_lo && j <= ex_hi)) continue;
                        pair_term<D, FT>(p, xs + (size_t)kk * D, xb, rc2, p0, p1, shift, F);
                    }
                } else {
                    for (int cc = 0; cc < 3; cc++) {
                        const int *it = A.items + (cell_at(q0 + cc) << A.log_depth);
                        const int m = off[q0 + cc + 1] - off[q0 + cc];
                        for (int kk = 0; kk < m; kk++) {
                            const int j = it[kk];
                            if ((unsigned)j >= (unsigned)n) {
                                bad = true;
                                continue;
                            }
                            if (j >= ex_lo && j <= ex_hi) continue;
                            pair_term<D, FT>(p, X + (size_t)j * D, xb, rc2, p0, p1, shift, F);
                        }
                    }
                }
            }
            FT *fp = reinterpret_cast<FT *>(A.fp) + (size_t)(p.bead_off + b) * D;
#pragma unroll
            for (int i = 0; i < D; i++) fp[i] = F[i];
        }
        if (bad) atomicOr(&s.flags, kFlagListCorrupt);
    }
}

// dynamic shared memory of k_pair_cells for `cap` staged beads
template <int D>
size_t pair_cells_smem_bytes(int cap)
{
    return (size_t)cap * (D * sizeof(double) + sizeof(int));
}

template <int D, typename FT>
__device__ __forceinline__ void noise_trans(const SysP &p, const SysS &s, int b, FT *xi)
{
    if (s.noise) {
        const double *q = s.noise + ((size_t)s.steps_done * p.n + b) * 2 * D;
#pragma unroll
        for (int i = 0; i < D; i++) xi[i] = (FT)q[i];
    } else if constexpr (sizeof(FT) == 4) {
        philox_normals_f<D>(p.seed, (uint32_t)b, s.step, false, xi);
    } else {
        double z[D];
        philox_normals<D>(p.seed, (uint32_t)b, s.step, false, z);
#pragma unroll
        for (int i = 0; i < D; i++) xi[i] = (FT)z[i];
    }
}

template <int D, typename FT>
__device__ __forceinline__ void noise_rot(const SysP &p, const SysS &s, int b, FT *xi)
{
    if (s.noise) {
        const double *q = s.noise + ((size_t)s.steps_done * p.n + b) * 2 * D + D;
#pragma unroll
        for (int i = 0; i < D; i++) xi[i] = (FT)q[i];
    } else if constexpr (sizeof(FT) == 4) {
        philox_normals_f<D>(p.seed, (uint32_t)b, s.step, true, xi);
    } else {
        double z[D];
        philox_normals<D>(p.seed, (uint32_t)b, s.step, true, z);
#pragma unroll
        for (int i = 0; i < D; i++) xi[i] = (FT)z[i];
    }
}

// pos + dt_eff F + s2 xi, wrapped; FP64 in the reference's operation order,
// mixed: the increment in FP32 and the accumulation in FP64
template <typename FT>
__device__ __forceinline__ double srk_update(double x, double dt_eff, double s2, FT f, FT xi, double L)
{
    double tmp;
    if constexpr (sizeof(FT) == 8) {
        tmp = x + dt_eff * f;
        if (s2 != 0.0) tmp += s2 * xi;
    } else {
        float inc = (float)dt_eff * f + (float)s2 * xi;
        tmp = x + (double)inc;
    }
    return py_mod(tmp, L);
}


// ------------------------------------------------------------------------
// stage and update kernels.  FUSED: the stage walks its beads' neighbour
// lists itself (warp_list_pair_force, the same sums as k_pair) instead of
// reading fp, which saves the pair kernel's launch, its second read of the
// positions and the fp round trip (SRK2 without coupled populations only;
// gcr_config.pair_mode 1).
// ------------------------------------------------------------------------
template <int D, typename FT, int STAGE, bool FUSED = false>
__global__ void __launch_bounds__(512, min_blocks<D, FT>()) k_stage(BatchArgs A)
{
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long sh_bits[16];
    __shared__ int sh_run;
    const int TB = blockDim.x;
    StageSmem<D, FT> sm;
    using BT = typename StageSmem<D, FT>::BT;
    sm.carve(smem_raw, TB);
    const int nt = *A.n_bead_tiles;
    // the next tile's table entry is loaded while the current tile runs
    Tile nx = (int)blockIdx.x < nt ? A.bead_tiles[blockIdx.x] : Tile{0, 0};
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        __syncthreads();  // the previous tile is done with shared memory
        const Tile tl = nx;
        if (t + (int)gridDim.x < nt) nx = A.bead_tiles[t + gridDim.x];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        // the system's constants are read before the barrier, with its flags
        const int n = p.n;
        const int base = tl.begin - 2;
        const double *__restrict__ X = stage_x<stage_reads(STAGE)>(p);
        // one decision per CTA: other CTAs may raise the system's flags while
        // this one runs, and every thread must reach the same barriers
        if (threadIdx.x == 0) sh_run = ld_volatile(&s.active) && !(ld_volatile(&s.flags) & kFlagFatal);
        __syncthreads();
        if (!sh_run) continue;
        // 1. positions and topology of beads begin-2 .. begin+TB+1
        for (int k = threadIdx.x; k < TB + 4; k += TB) {
            int m = base + k;
            if (m >= 0 && m < n) {
#pragma unroll
                for (int i = 0; i < D; i++) sm.x[k * D + i] = __ldg(X + (size_t)m * D + i);
                sm.tp[k] = A.topo[p.bead_off + m];
                sm.ra[k] = p.calc_springs ? (BT)A.restb[p.bead_off + m] : BT(0);
            } else {
                sm.tp[k] = 0;
                sm.ra[k] = BT(0);
            }
        }
        __syncthreads();
        // the bead's own inputs of phase 4, loaded before the barriers (the
        // build positions of a virtual update's skin test too: loaded after
        // the pos1 stores, they would wait behind them)
        FT pre_t[D], pre_f[D], pre_p[D];
        double pre_r[D];
        int pre_cnt = 0;  // list count of the fused pair walk
        {
            const int bq = tl.begin + (int)threadIdx.x;
            const bool ok = bq < n;
            const FT *tq = reinterpret_cast<const FT *>(p.tan);
            const FT *fq = reinterpret_cast<const FT *>(p.frc);
            const FT *pq = reinterpret_cast<const FT *>(A.fp) + (size_t)(p.bead_off + (ok ? bq : 0)) * D;
#pragma unroll
            for (int i = 0; i < D; i++) {
                pre_t[i] = ok ? tq[(size_t)bq * D + i] : FT(0);
                pre_f[i] = (ok && STAGE == 1) ? fq[(size_t)bq * D + i] : FT(0);
                pre_p[i] = (!FUSED && ok && p.calc_wca) ? pq[i] : FT(0);
            }
            if constexpr (stage_writes(STAGE) != 0) {
                const double *rq = A.xref + (size_t)(p.bead_off + (ok ? bq : 0)) * D;
#pragma unroll
                for (int i = 0; i < D; i++) pre_r[i] = (ok && p.calc_wca) ? rq[i] : 0.0;
            }
            if constexpr (FUSED) pre_cnt = (ok && p.calc_wca && !p.motor) ? A.ncount[p.bead_off + bq] : 0;
        }
        const bool springs = p.calc_springs, cb = p.calc_bend;
        if (springs) {
            // 2. every bond (j, j+1) of the tile once
            const BT kspring = (BT)p.k;
            for (int k = threadIdx.x; k < TB + 3; k += TB) {
                BT d[D], tt[D], f = BT(0);
#pragma unroll
                for (int i = 0; i < D; i++) d[i] = tt[i] = BT(0);
                if (sm.tp[k] & kHasNext) {
                    BT r2 = BT(0);
#pragma unroll
                    for (int i = 0; i < D; i++) {
                        d[i] = (BT)inbounds(sm.x[k * D + i], sm.x[(k + 1) * D + i], p.half_L, p.L);
                        r2 += d[i] * d[i];
                    }
                    if (r2 != BT(0)) {
                        const BT a = sm.ra[k];
                        BT inv = inv_sqrt<BT>(r2);
                        f = kspring * (a * inv - BT(1));
#pragma unroll
                        for (int i = 0; i < D; i++) tt[i] = d[i] * inv;
                    } else {
#pragma unroll
                        for (int i = 0; i < D; i++) tt[i] = d[i];
                    }
                }
#pragma unroll
                for (int i = 0; i < D; i++) {
                    sm.bd[k * D + i] = d[i];
                    sm.bt[k * D + i] = tt[i];
                }
                sm.bf[k] = f;
            }
            __syncthreads();
            // 3. every bend once: bead begin-1+k uses bonds k+1 (own) and k
            if (cb) {
                const BT kappa = (BT)p.kappa, theta0 = (BT)p.theta0;
                for (int k = threadIdx.x; k < TB + 2; k += TB) {
                    BT fw[D], bw[D];
#pragma unroll
                    for (int i = 0; i < D; i++) fw[i] = bw[i] = BT(0);
                    const uint8_t tp = sm.tp[k + 1];
                    if ((tp & kHasPrev) && (tp & kHasNext)) {
                        if (!bend<D, BT>(sm.bt + (k + 1) * D, sm.bt + k * D, theta0, kappa, fw, bw)) {
#pragma unroll
                            for (int i = 0; i < D; i++) fw[i] = bw[i] = BT(0);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < D; i++) {
                        sm.fw[k * D + i] = fw[i];
                        sm.bw[k * D + i] = bw[i];
                    }
                }
            }
            __syncthreads();
        }
        // 4. per bead: gather bonded terms, pair forces, propulsion, update
        const int tid = threadIdx.x;
        const int b = tl.begin + tid;
        // fused pair forces: the warp-wide list walk of k_pair, which every
        // lane of the warp joins (a lane past the system with no list)
        FT Fp[3] = {FT(0), FT(0), FT(0)};
        if constexpr (FUSED) {
            if (p.calc_wca) {
                bool bad = false;
                double xq[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int i = 0; i < D; i++) xq[i] = sm.x[(tid + 2) * D + i];
                warp_list_pair_force<D, FT>(A, p, X, xq, b, pre_cnt, Fp, bad,
                                            sm.pb + (size_t)(tid >> 5) * (D + 1) * 32 * kPairChunk);
                if (bad) atomicOr(&s.flags, kFlagListCorrupt);
            }
        }
        double mf2 = 0.0;
        if (b < n) {
            FT *frc = reinterpret_cast<FT *>(p.frc);
            FT *tan = reinterpret_cast<FT *>(p.tan);
            double xb[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < D; i++) xb[i] = sm.x[(tid + 2) * D + i];
            // F0 (stage 1) and the bonded terms summed in BT, then FT
            BT Fb[3];
            FT F[3], tg[3];
#pragma unroll
            for (int i = 0; i < D; i++) {
                // the SRK2 corrector adds to F0; every other stage starts from 0
                Fb[i] = STAGE == 1 ? (BT)pre_f[i] : BT(0);
                tg[i] = pre_t[i];
            }
            bool tang_set = false;
            if (springs) {
                const uint8_t tp = sm.tp[tid + 2];
                const bool prev = tp & kHasPrev, next = tp & kHasNext;
                if (prev) {
                    const BT f = sm.bf[tid + 1];
#pragma unroll
                    for (int i = 0; i < D; i++) Fb[i] -= sm.bd[(tid + 1) * D + i] * f;
                    if ((tp & kHasPrev2) && cb) {
#pragma unroll
                        for (int i = 0; i < D; i++) Fb[i] -= sm.bw[tid * D + i];
                    }
                }
                if (next) {
                    const BT f = sm.bf[tid + 2];
#pragma unroll
                    for (int i = 0; i < D; i++) Fb[i] += sm.bd[(tid + 2) * D + i] * f;
                }
                if (prev && next && cb) {
#pragma unroll
                    for (int i = 0; i < D; i++) Fb[i] += sm.fw[(tid + 1) * D + i] + sm.bw[(tid + 1) * D + i];
                }
                if ((tp & kHasNext2) && cb) {
#pragma unroll
                    for (int i = 0; i < D; i++) Fb[i] -= sm.fw[(tid + 2) * D + i];
                }
                if (p.get_orient && (prev || next)) {
                    const BT *ti = sm.bt + (tid + 2) * D, *tj = sm.bt + (tid + 1) * D;
                    if (prev && next) {
                        // (ti + tj) / sqrt(2 (1 + c)); aligned tangents give ti.  In
                        // FP32 1 + c = 2 - |tj - ti|^2 / 2 and the aligned test
                        // from the chord, as in bend()
                        bool interior;
                        BT coeff;
                        if constexpr (sizeof(BT) == 4) {
                            BT ch2 = BT(0);
#pragma unroll
                            for (int i = 0; i < D; i++) ch2 += (tj[i] - ti[i]) * (tj[i] - ti[i]);
                            const BT omc = BT(0.5) * ch2;
                            interior = omc > BT(0) && omc < BT(2);
                            coeff = inv_sqrt<BT>(BT(2) * (BT(2) - omc));
                        } else {
                            BT c = BT(0);
#pragma unroll
                            for (int i = 0; i < D; i++) c += ti[i] * tj[i];
                            interior = BT(-1) < c && c < BT(1);
                            coeff = inv_sqrt<BT>(BT(2) * (BT(1) + c));
                        }
                        if (interior) {
#pragma unroll
                            for (int i = 0; i < D; i++) tg[i] = (FT)(coeff * (ti[i] + tj[i]));
                        } else {
#pragma unroll
                            for (int i = 0; i < D; i++) tg[i] = (FT)ti[i];
                        }
                    } else if (next) {  // head bead
#pragma unroll
                        for (int i = 0; i < D; i++) tg[i] = (FT)ti[i];
                    } else {  // tail bead
#pragma unroll
                        for (int i = 0; i < D; i++) tg[i] = (FT)tj[i];
                    }
                    tang_set = true;
                }
            }
#pragma unroll
            for (int i = 0; i < D; i++) F[i] = (FT)Fb[i];
            if (p.calc_wca) {
                if constexpr (FUSED) {
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] += Fp[i];
                } else {
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] += pre_p[i];
                }
            }
            if (p.self_propel) {
                const FT v0 = (FT)p.v0;
                if (p.rotate_prop) {
                    const FT cs = (FT)p.cos_a, sn = (FT)p.sin_a;
                    FT fx = v0 * (cs * tg[0] - sn * tg[1]);
                    FT fy = v0 * (sn * tg[0] + cs * tg[1]);
                    F[0] += fx;
                    F[1] += fy;
                } else {
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] += v0 * tg[i];
                }
            }
            if constexpr (!srk4_stage(STAGE)) {
                if (p.pushed) {
                    // the motor pushes of this stage (k_motor), added after
                    // the chains' own forces as the other population's
                    // force (SRK.py:261-267, 287-294); where_active counts
                    // the attached motors from -1 at each step (SRK.py:132)
                    int *mp = A.mpush + p.bead_off + b, *md = A.mdelta + p.bead_off + b;
                    const int npush = *mp, dl = *md;
                    *mp = 0;
                    *md = 0;
                    int *ab = A.act + p.bead_off + b;
                    *ab = (STAGE == 0 ? -1 : *ab) + dl;
                    if (npush > 0) {
                        const FT f = (FT)p.push_force;
                        FT M[3] = {FT(0), FT(0), FT(0)};
                        for (int k = 0; k < npush; k++) {
#pragma unroll
                            for (int i = 0; i < D; i++) M[i] += f * tg[i];
                        }
#pragma unroll
                        for (int i = 0; i < D; i++) F[i] += M[i];
                    }
                }
            }
            // G: the force the caller and the dt rule see -- F0 + F1 (SRK2),
            // the weighted sum of the stage forces (SRK4, SRK.py:296-321,
            // with the stage's own force kept in faux)
            FT G[3];
            if constexpr (srk4_stage(STAGE)) {
                FT *faux = reinterpret_cast<FT *>(p.faux);
                const FT w = (STAGE == 10 || STAGE == 13) ? FT(1. / 6.) : FT(1. / 3.);
#pragma unroll
                for (int i = 0; i < D; i++) {
                    faux[(size_t)b * D + i] = F[i];
                    G[i] = STAGE == 10 ? F[i] * w : frc[(size_t)b * D + i] + F[i] * w;
                }
            } else {
#pragma unroll
                for (int i = 0; i < D; i++) G[i] = F[i];
            }
#pragma unroll
            for (int i = 0; i < D; i++) frc[(size_t)b * D + i] = G[i];
            if (tang_set) {
#pragma unroll
                for (int i = 0; i < D; i++) tan[(size_t)b * D + i] = tg[i];
            }
            if constexpr (stage_writes(STAGE) != 0) {
                // the step's translational noise, drawn once in the first stage
                FT xi[3] = {FT(0), FT(0), FT(0)};
                if (p.D > 0.0) {
                    FT *xs = reinterpret_cast<FT *>(A.xi) + (size_t)(p.bead_off + b) * D;
                    if constexpr (STAGE == 0 || STAGE == 10) {
                        noise_trans<D, FT>(p, s, b, xi);
#pragma unroll
                        for (int i = 0; i < D; i++) xs[i] = xi[i];
                    } else {
#pragma unroll
                        for (int i = 0; i < D; i++) xi[i] = xs[i];
                    }
                }
                // virtual update: (pos + dt_eff/r F + sqrt(2 D dt) xi) mod L
                // from the step's old positions (with the rigid-rod
                // projection on, k_rigid writes it)
                if (p.rigid == 0.0) {
                    const double dt = s.dt;
                    const double dt_eff = dt * stage_dt_factor(STAGE) / p.radius;
                    const double s2 = sqrt(2.0 * dt * p.D);
                    double *W = stage_x<stage_writes(STAGE)>(p);
                    double x1[3] = {0.0, 0.0, 0.0};
                    bool finite = true;
                    // an attached motor writes no virtual position: its pos1
                    // keeps the previous value (SRK.py:389-395)
                    const bool hold = p.motor && p.motor_hold && A.act[p.bead_off + b] >= 0;
#pragma unroll
                    for (int i = 0; i < D; i++) {
                        if (hold) {
                            x1[i] = W[(size_t)b * D + i];
                            continue;
                        }
                        const double x0 = stage_reads(STAGE) == 0 ? xb[i] : p.pos[(size_t)b * D + i];
                        x1[i] = srk_update<FT>(x0, dt_eff, s2, F[i], xi[i], p.L);
                        finite &= isfinite(x1[i]);
                        W[(size_t)b * D + i] = x1[i];
                    }
                    if (!finite)
                        atomicOr(&s.flags, kFlagNonFinite);
                    else if (p.calc_wca && left_skin_of<D>(p, pre_r, x1))
                        s.rebuild = 1;  // the list no longer covers the new positions
                }
            }
            if constexpr (STAGE == 1 || STAGE == 13) {
                // |G|^2 in FP64 for the dt rule (SRK.py:323-330)
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < D; i++) acc += (double)G[i] * (double)G[i];
                mf2 = acc;
            }
        }
        if (STAGE == 1 || STAGE == 13) {
            // warp / block max over non-negative doubles via their bit patterns
            unsigned long long bits = (unsigned long long)__double_as_longlong(mf2);
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
                bits = other > bits ? other : bits;
            }
            if ((threadIdx.x & 31) == 0) sh_bits[threadIdx.x >> 5] = bits;
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned long long mx = 0;
                for (int w = 0; w < (TB + 31) / 32; w++) mx = sh_bits[w] > mx ? sh_bits[w] : mx;
                if (mx) atomicMax(&s.max_f2, mx);
            }
        }
    }
}

// the update kernel holds all its inputs in registers at once
#ifndef GCR_UPDATE_MIN_BLOCKS
#define GCR_UPDATE_MIN_BLOCKS 3
#endif
template <int D, typename FT>
constexpr int update_min_blocks()
{
    return (D == 2 && sizeof(FT) == 4) ? GCR_UPDATE_MIN_BLOCKS : 1;
}

template <int D, typename FT>
__global__ void __launch_bounds__(512, update_min_blocks<D, FT>()) k_update(BatchArgs A)
{
    pdl_wait();
    const int nt = *A.n_bead_tiles;
    // the next tile's table entry is loaded while the current tile runs
    Tile nx = (int)blockIdx.x < nt ? A.bead_tiles[blockIdx.x] : Tile{0, 0};
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = nx;
        if (t + (int)gridDim.x < nt) nx = A.bead_tiles[t + gridDim.x];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        const int b = tl.begin + threadIdx.x;
        const bool valid = b < p.n && threadIdx.x < A.tile_beads;
        const FT *frc = reinterpret_cast<const FT *>(p.frc);
        const bool plain = p.rigid == 0.0;  // else k_rigid writes pos
        // every input is loaded before the first store: a store to pos may
        // alias them for the compiler, which would order each later load
        // behind it.  They go out (from a valid bead of the tile, whatever
        // the thread) together with the system's state: plain loads, as a
        // fatal flag raised meanwhile by another thread costs at most the
        // update of a system that is stopping anyway
        const int bc = valid ? b : tl.begin;
        FT xi[3] = {FT(0), FT(0), FT(0)}, fo[3] = {FT(0), FT(0), FT(0)};
        double xold[3] = {0.0, 0.0, 0.0}, xr[3] = {0.0, 0.0, 0.0};
        if (p.D > 0.0) {
            const FT *xs = reinterpret_cast<const FT *>(A.xi) + (size_t)(p.bead_off + bc) * D;
#pragma unroll
            for (int i = 0; i < D; i++) xi[i] = xs[i];
        }
        if (plain) {
#pragma unroll
            for (int i = 0; i < D; i++) {
                xold[i] = p.pos[(size_t)bc * D + i];
                fo[i] = frc[(size_t)bc * D + i];
            }
            if (p.calc_wca) {
                const double *r = A.xref + (size_t)(p.bead_off + bc) * D;
#pragma unroll
                for (int i = 0; i < D; i++) xr[i] = r[i];
            }
        }
        // no barriers in this kernel: a per-thread decision is safe
        if (!s.active || (s.flags & kFlagFatal) || !valid) continue;
        const double dtu = s.dt_used;
        // force_prefactor 0.5 of the SRK2 corrector; 1 for SRK4's weighted sum
        const double dt_eff = dtu * (A.order == 4 ? 1.0 : 0.5) / p.radius;
        const double s2 = sqrt(2.0 * dtu * p.D);
        double x[3] = {0.0, 0.0, 0.0};
        bool finite = true;
        // an attached motor keeps its position (SRK.py:389-395)
        const bool hold = p.motor && p.motor_hold && A.act[p.bead_off + b] >= 0;
        if (plain) {
#pragma unroll
            for (int i = 0; i < D; i++) {
                const double xo = xold[i];
                if (hold) {
                    x[i] = xo;
                    continue;
                }
                x[i] = srk_update<FT>(xo, dt_eff, s2, fo[i], xi[i], p.L);
                finite &= isfinite(x[i]);
                p.pos[(size_t)b * D + i] = x[i];
                const int di = image_step(xo, x[i], p.half_L);
                if (di) A.img[(size_t)(p.bead_off + b) * D + i] += di;
            }
            if (!finite) atomicOr(&s.flags, kFlagNonFinite);
        }
        if (p.Dr > 0.0 && !p.get_orient) {
            // rotational diffusion, SRK.py:399-423 (note the factor pi)
            FT xr[3] = {FT(0), FT(0), FT(0)};
            noise_rot<D, FT>(p, s, b, xr);
            FT *tan = reinterpret_cast<FT *>(p.tan);
            FT tb[3];
#pragma unroll
            for (int i = 0; i < D; i++) tb[i] = tan[(size_t)b * D + i];
            const FT sq = (FT)(sqrt(2.0 * dtu * p.Dr) * 3.141592653589793);
            FT proj = FT(0);
#pragma unroll
            for (int i = 0; i < D; i++) proj += xr[i] * tb[i];
#pragma unroll
            for (int i = 0; i < D; i++) xr[i] -= proj * tb[i];
            FT mag = FT(0);
#pragma unroll
            for (int i = 0; i < D; i++) {
                FT v = tb[i] + sq * xr[i];
                mag += v * v;
                tb[i] = v;
            }
            mag = sqrt(mag);
#pragma unroll
            for (int i = 0; i < D; i++) tan[(size_t)b * D + i] = tb[i] / mag;
        }
        if (plain && finite && p.calc_wca && left_skin_of<D>(p, xr, x)) s.rebuild = 1;  // rebuild before the next step
    }
}

// ------------------------------------------------------------------------
// rigid-rod projection, updates.project_updates_for_rigid_rod
// (updates.py:347-499), in place of the plain update when the factor is on
// (SRK.py:364-371).  One thread per chain (the thread of its head bead),
// three passes over the chain's beads; all arithmetic in FP64.
//   STAGE 0 (predictor): pos  -> pos1, dt_eff = dt
//   STAGE 1 (corrector): pos1 -> pos,  dt_eff = dt_used / 2, forces F0 + F1
//   SRK4 stages 10..13: the stage's positions -> its virtual update (pos1,
//   pos2, pos1) with dt/2, dt/2, dt and the stage force, then pos with
//   dt_used and the weighted sum
// The projection reads the positions the forces were taken at (pos, then
// pos1: check_force_at_pos), as the reference does.  Per chain:
//   u_b      = dt_eff / r F_b + sqrt(2 D dt_eff) xi_b
//   d_b      = a (b - (n-1)/2), I = dim sum_b d_b^2
//   c        = head + mean_b wrap(x_b - head), mod L; r_hat = wrap(x_last - head) / |.|
//   o_b      = wrap(x_b - (c + r_hat d_b))                  (deviation from the rod)
//   2D: tau_i = sum_b (2i-1) r_hat_{1-i} u_{b,i} d_b / I,
//       u_b,i <- (1-f) u_b,i + f (-o_b,i + mean u_i + tau_i d_b (2i-1) r_hat_{1-i})
//   3D: tau = |r| sum_b r_hat x u_b,
//       u_b <- (1-f) u_b + f (-o_b + mean u + (|r| / I) tau x r_hat)
//   x_b <- (x_b + u_b) mod L
// (the 2D torque per component and the 3D rotation term without a distance
// factor are the reference's expressions as written).  A one-bead chain in
// 3D (I = 0) gets no rotation term; the reference divides by zero there.
// ------------------------------------------------------------------------
__device__ __forceinline__ double wrap_open(double sep, double half, double L)
{
    if (sep < -half)
        sep += L;
    else if (sep > half)
        sep -= L;
    return sep;
}

template <int D, typename FT, int STAGE>
__global__ void __launch_bounds__(512) k_rigid(BatchArgs A)
{
    pdl_wait();
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        // no barriers in this kernel: a per-thread decision is safe
        if (p.rigid == 0.0) continue;
        if (!ld_volatile(&s.active) || (ld_volatile(&s.flags) & kFlagFatal)) continue;
        const int b0 = tl.begin + threadIdx.x;
        if (b0 >= p.n || threadIdx.x >= A.tile_beads) continue;
        if (A.topo[p.bead_off + b0] & kHasPrev) continue;  // not a chain's head bead
        const int c = p.chain[b0];
        const int len = p.chain_start[c + 1] - b0;
        const double *prev = stage_x<stage_reads(STAGE)>(p);
        double *rtn = stage_x<stage_writes(STAGE)>(p);
        // dt_eff of SRK.py:355-360: the step's dt in a virtual update, dt_used
        // in the real one
        const double dt = (stage_writes(STAGE) != 0 ? s.dt : s.dt_used) * stage_dt_factor(STAGE);
        // write_to_forces: the stage's own force in SRK4's virtual updates
        const FT *frc = reinterpret_cast<const FT *>(srk4_stage(STAGE) && STAGE != 13 ? p.faux : p.frc);
        const FT *xs = reinterpret_cast<const FT *>(A.xi) + (size_t)p.bead_off * D;
        const double L = p.L, half = 0.5 * L, f = p.rigid;
        const double dt_over_r = dt / p.radius;
        const double s2 = sqrt(2.0 * p.D * dt);
        const double rest = p.rest[c];
        const double half_clm1 = (double)(len - 1) / 2.0;
        auto upd = [&](int b, int i) {
            double u = dt_over_r * (double)frc[(size_t)b * D + i];
            if (s2 != 0.0) u += s2 * (double)xs[(size_t)b * D + i];
            return u;
        };
        const double *x0 = prev + (size_t)b0 * D;
        // pass 1: moment of inertia, mean update, centre, end-to-end vector
        double inertia = 0.0, r_mag = 0.0, mean[D], com[D], rh[D];
#pragma unroll
        for (int i = 0; i < D; i++) mean[i] = com[i] = rh[i] = 0.0;
        for (int k = 0; k < len; k++) {
            const int b = b0 + k;
            const double dk = rest * ((double)k - half_clm1);
#pragma unroll
            for (int i = 0; i < D; i++) {
                inertia += dk * dk;
                mean[i] += upd(b, i);
                const double sep = wrap_open(prev[(size_t)b * D + i] - x0[i], half, L);
                com[i] += sep;
                if (k == len - 1) {
                    rh[i] = sep;
                    r_mag += sep * sep;
                }
            }
        }
#pragma unroll
        for (int i = 0; i < D; i++) {
            mean[i] /= (double)len;
            com[i] = py_mod(x0[i] + com[i] / (double)len, L);
        }
        if (r_mag > 0.0) {
            r_mag = sqrt(r_mag);
#pragma unroll
            for (int i = 0; i < D; i++) rh[i] /= r_mag;
        }
        // pass 2: torque
        double tq[3] = {0.0, 0.0, 0.0}, rot[3] = {0.0, 0.0, 0.0};
        if constexpr (D == 2) {
            for (int k = 0; k < len; k++) {
                const double dk = rest * ((double)k - half_clm1);
#pragma unroll
                for (int i = 0; i < 2; i++) tq[i] += (double)(2 * i - 1) * rh[1 - i] * upd(b0 + k, i) * dk;
            }
            if (inertia != 0.0) {
                tq[0] /= inertia;
                tq[1] /= inertia;
            }
        } else {
            for (int k = 0; k < len; k++) {
                const double u0 = upd(b0 + k, 0), u1 = upd(b0 + k, 1), u2 = upd(b0 + k, 2);
                tq[0] += rh[1] * u2 - rh[2] * u1;
                tq[1] += rh[2] * u0 - rh[0] * u2;
                tq[2] += rh[0] * u1 - rh[1] * u0;
            }
#pragma unroll
            for (int i = 0; i < 3; i++) tq[i] = r_mag * tq[i];
            const double q = inertia != 0.0 ? r_mag / inertia : 0.0;
            rot[0] = q * (tq[1] * rh[2] - tq[2] * rh[1]);
            rot[1] = q * (tq[2] * rh[0] - tq[0] * rh[2]);
            rot[2] = q * (tq[0] * rh[1] - tq[1] * rh[0]);
        }
        // pass 3: projected updates and the new positions
        const double keep = 1. - f;
        bool finite = true, moved = false;
        for (int k = 0; k < len; k++) {
            const int b = b0 + k;
            const double dk = rest * ((double)k - half_clm1);
            double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < D; i++) {
                double o = prev[(size_t)b * D + i] - (com[i] + rh[i] * dk);
                if (o < -half)
                    o += L;
                else if (o >= half)
                    o -= L;
                double u = upd(b, i) * keep;
                if constexpr (D == 2)
                    u += f * (-o + mean[i] + (tq[i] * dk * (double)(2 * i - 1) * rh[1 - i]));
                else
                    u += f * (-o + mean[i] + rot[i]);
                x[i] = py_mod(prev[(size_t)b * D + i] + u, L);
                finite &= isfinite(x[i]);
                if constexpr (stage_writes(STAGE) == 0) {
                    // the real update: count the images crossed since the old pos
                    const int di = image_step(rtn[(size_t)b * D + i], x[i], half);
                    if (di) A.img[(size_t)(p.bead_off + b) * D + i] += di;
                }
                rtn[(size_t)b * D + i] = x[i];
            }
            if (finite && p.calc_wca && left_skin<D>(p, A, b, x)) moved = true;
        }
        if (!finite) atomicOr(&s.flags, kFlagNonFinite);
        if (moved) s.rebuild = 1;  // the list no longer covers the new positions
    }
}

// per-system dt rule after stage 1 (SRK.py:323-353): one thread per slot
__global__ void k_sys_dt(BatchArgs A, int n_slots)
{
    pdl_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slots) return;
    const SysP &p = A.P[i];
    SysS &s = A.S[i];
    if (!s.active || (s.flags & kFlagFatal)) return;
    const double pref = A.order == 4 ? 1.0 : 0.5;
    double mf2s = __longlong_as_double((long long)s.max_f2);
    double S = p.sqrt2D + pref * sqrt(mf2s) / p.radius;
    // coupled populations: one dt from the largest S over the moving members
    // (the max over every thread's shared_arr[:,3], SRK.py:333-340)
    double Sg = (p.grp_n && p.fixed) ? 0.0 : S;
    // the rule's constants of a group come from its first moving member, so
    // every member takes the same dt
    double dtmax = p.dtmax, mdps = p.mdps, rk = p.rk;
    bool lead = false;
    int group_fatal = 0;
    for (int k = 0; k < p.grp_n && k < kMaxPops; k++) {
        const int m = p.grp[k];
        if (m < 0 || m >= n_slots) continue;
        const SysP &pm = A.P[m];
        if (!pm.fixed && !lead) {
            dtmax = pm.dtmax;
            mdps = pm.mdps;
            rk = pm.rk;
            lead = true;
        }
        const SysS &sm = A.S[m];
        if (m != i) group_fatal |= sm.flags & kFlagFatal;
        if (m == i || pm.fixed || !sm.active || (sm.flags & kFlagFatal)) continue;
        const double Sm = pm.sqrt2D + pref * sqrt(__longlong_as_double((long long)sm.max_f2)) / pm.radius;
        Sg = Sm > Sg ? Sm : Sg;
    }
    if (group_fatal) {
        // a population of the box stopped this step (its forces on the others
        // are stale): the whole box stops before the real update, the step is
        // not counted, and the host sees the same flag on every member
        s.flags |= group_fatal;
        return;
    }
    double dt;
    if (Sg == 0.0)
        dt = dtmax;
    else {
        double q = mdps / Sg;
        dt = (q < dtmax) ? q : dtmax;
    }
    double dt_used = rk * dt;
    if (s.max_dt_usable > 0.0) {
        double lim = s.max_dt_usable - s.elapsed;
        dt_used = (lim < dt_used) ? lim : dt_used;
    }
    s.dt_next = dt;
    s.dt_used = dt_used;
    s.mfs = S;
}

// per-system step bookkeeping after the corrector (SRK.py:330, 348-349,
// 128-130): one thread per slot; a step aborted by a fatal flag is not counted
__global__ void k_sys_end(BatchArgs A, int n_slots)
{
    pdl_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slots) return;
    SysS &s = A.S[i];
    if (!s.active || (s.flags & kFlagFatal)) return;
    s.dt = s.dt_next;
    s.elapsed += s.dt_used;
    s.step += 1;
    s.steps_done += 1;
    s.max_f2 = 0ull;
    bool more = (s.steps_done < s.max_steps || s.max_steps < 0) &&
                (s.elapsed < s.max_dt_usable || s.max_dt_usable < 0.0);
    s.active = more ? 1 : 0;
}

// chain-neighbour bits of every bead of one system
__global__ void k_topo(const int32_t *__restrict__ chain, int n, uint8_t *topo)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    int c = chain[b];
    uint8_t t = 0;
    if (b >= 1 && chain[b - 1] == c) t |= kHasPrev;
    if (b >= 2 && chain[b - 2] == c) t |= kHasPrev2;
    if (b + 1 < n && chain[b + 1] == c) t |= kHasNext;
    if (b + 2 < n && chain[b + 2] == c) t |= kHasNext2;
    topo[b] = t;
}


// flag system `slot` for a list build (every resident system when slot < 0):
// admission, a new descriptor, a coupling change
__global__ void k_sys_mark(BatchArgs A, int n_slots, int slot)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slots || (slot >= 0 && i != slot)) return;
    A.S[i].rebuild = 1;
}

// start of a run: the rest length of every armed bead's chain into restb;
// the host may have written positions since the last list
// build, so every armed system is tested against its list as the step
// kernels test it -- a bead farther than skin/2 from where the list was built
// flags a rebuild, and otherwise the list still holds every pair within
// r_cut.  Coupled populations are flagged outright: their fixed members have
// no bead tiles to test.
template <int D>
__global__ void __launch_bounds__(512) k_run_check(BatchArgs A)
{
    pdl_wait();
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        // no barriers in this kernel: a per-thread decision is safe
        if (!ld_volatile(&s.active) || (ld_volatile(&s.flags) & kFlagFatal)) continue;
        const int b = tl.begin + threadIdx.x;
        if (b >= p.n || threadIdx.x >= A.tile_beads) continue;
        if (p.calc_springs) {
            int ch = p.chain[b];
            ch = ch < 0 ? 0 : (ch >= p.n_chains ? p.n_chains - 1 : ch);
            A.restb[p.bead_off + b] = p.rest[ch];
        }
        if (!p.calc_wca || ld_volatile(&s.rebuild)) continue;
        if (p.grp_n > 0) {
            s.rebuild = 1;
            continue;
        }
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < D; i++) x[i] = p.pos[(size_t)b * D + i];
        if (left_skin<D>(p, A, b, x)) s.rebuild = 1;
    }
}

// ------------------------------------------------------------------------
// motor decisions of one SRK2 stage (forces.calc_motor_push,
// forces.py:248-283), one thread per motor.  The reference loops over the
// chain beads in order and, for each, over the motors on its list; a motor's
// fate depends only on the beads that reach it, in bead order, so each
// thread replays its motor's sequence: over its candidate beads (the chain
// beads within the list radius, cross_rc2, at the stage's positions, in
// ascending id) an attached motor stays with probability 1 - k_off, else
// detaches (the drawing bead's where_active drops by one), and a free motor
// attaches with probability k_on when within motor_max_dist (that bead's
// where_active rises by one and it gets one push).  The chain beads' pushes
// and where_active changes are summed with integer atomics, so the result
// does not depend on the order of the motors' threads; the stage kernel
// turns them into forces.  Draws: motor_uniforms(seed, motor, bead, step,
// stage).  Distances in FP64 without contraction, as the reference computes
// them (forces.inbounds_diff, forces.py:44-55).
// ------------------------------------------------------------------------
template <int D, int WHICH>
__global__ void __launch_bounds__(512) k_motor(BatchArgs A)
{
    pdl_wait();
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        if (!p.motor) continue;
        SysS &s = A.S[tl.sys];
        if (!ld_volatile(&s.active) || (ld_volatile(&s.flags) & kFlagFatal)) continue;
        const int m = tl.begin + threadIdx.x;
        if (m >= p.n || threadIdx.x >= A.tile_beads) continue;
        int *act_m = A.act + p.bead_off + m;
        // where_active is wiped at the start of each step (SRK.py:132)
        int am = WHICH == 0 ? -1 : *act_m;
        const int k = p.motor_k;
        const int qs = (k >= 0 && k < p.n_cross && k < kMaxPops - 1) ? p.cross_q[k] : -1;
        if ((unsigned)qs >= (unsigned)A.n_slots) {
            *act_m = am;
            atomicOr(&s.flags, kFlagListCorrupt);
            continue;
        }
        const SysP &q = A.P[qs];
        const double *XM = stage_x<WHICH>(p);
        const double *XQ = stage_x<WHICH>(q);
        double xm[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < D; i++) xm[i] = XM[(size_t)m * D + i];
        const int64_t row = p.x_off + (int64_t)k * p.n + m;
        int cnt = A.xcount[row];
        cnt = cnt < 0 ? 0 : (cnt < A.list_depth ? cnt : A.list_depth);
        const double r2 = p.cross_rc2[k], dmax2 = p.mparams[0], k_on = p.mparams[3], k_off = p.mparams[4];
        const int64_t step = s.step;
        bool bad = false;
        for (int e = 0; e < cnt; e++) {
            const int j = A.xnbr[row + (int64_t)e * A.xstride];
            if ((unsigned)j >= (unsigned)q.n) {
                bad = true;
                continue;
            }
            double ds = 0.0;
#pragma unroll
            for (int i = 0; i < D; i++) {
                const double d = inbounds(xm[i], XQ[(size_t)j * D + i], p.half_L, p.L);
                ds = __dadd_rn(ds, __dmul_rn(d, d));
            }
            if (!(ds <= r2)) continue;
            double u_off, u_on;
            motor_uniforms(p.seed, (uint32_t)m, (uint32_t)j, step, WHICH, u_off, u_on);
            if (am >= 0) {
                if (u_off > k_off) continue;
                am = -1;
                atomicAdd(A.mdelta + q.bead_off + j, -1);
            }
            if (am < 0 && u_on < k_on && ds <= dmax2) {
                atomicAdd(A.mdelta + q.bead_off + j, 1);
                atomicAdd(A.mpush + q.bead_off + j, 1);
                am = j;
            }
        }
        *act_m = am;
        if (bad) atomicOr(&s.flags, kFlagListCorrupt);
    }
}

// ------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------
template <int D, typename FT>
struct StepKernels {
    static void *pair0() { return (void *)k_pair<D, FT, 0, false>; }
    static void *pair1() { return (void *)k_pair<D, FT, 1, false>; }
    static void *stage0() { return (void *)k_stage<D, FT, 0>; }
    static void *stage1() { return (void *)k_stage<D, FT, 1>; }
    static void *stage0f() { return (void *)k_stage<D, FT, 0, true>; }
    static void *stage1f() { return (void *)k_stage<D, FT, 1, true>; }
    static void *pair_cells0() { return (void *)k_pair_cells<D, FT, 0>; }
    static void *pair_cells1() { return (void *)k_pair_cells<D, FT, 1>; }
    static void *update() { return (void *)k_update<D, FT>; }
    static void *rigid0() { return (void *)k_rigid<D, FT, 0>; }
    static void *rigid1() { return (void *)k_rigid<D, FT, 1>; }
    static void fill4(KernelSet &k)
    {
        k.pair2 = (void *)k_pair<D, FT, 2, false>;
        k.stage4[0] = (void *)k_stage<D, FT, 10>;
        k.stage4[1] = (void *)k_stage<D, FT, 11>;
        k.stage4[2] = (void *)k_stage<D, FT, 12>;
        k.stage4[3] = (void *)k_stage<D, FT, 13>;
        k.rigid4[0] = (void *)k_rigid<D, FT, 10>;
        k.rigid4[1] = (void *)k_rigid<D, FT, 11>;
        k.rigid4[2] = (void *)k_rigid<D, FT, 12>;
        k.rigid4[3] = (void *)k_rigid<D, FT, 13>;
        k.pair_cross[0] = (void *)k_pair<D, FT, 0, true>;
        k.pair_cross[1] = (void *)k_pair<D, FT, 1, true>;
        k.pair_cross[2] = (void *)k_pair<D, FT, 2, true>;
    }
};

KernelSet kernel_set(int dim, int precision)
{
    KernelSet k{};
    if (dim == 2)
        k.stage_smem = precision == 0 ? stage_smem_bytes<2, double> : stage_smem_bytes<2, float>;
    else
        k.stage_smem = precision == 0 ? stage_smem_bytes<3, double> : stage_smem_bytes<3, float>;
    if (dim == 2)
        k.pair_smem = precision == 0 ? pair_smem_bytes<2, double> : pair_smem_bytes<2, float>;
    else
        k.pair_smem = precision == 0 ? pair_smem_bytes<3, double> : pair_smem_bytes<3, float>;
    k.pair_cells_smem = dim == 2 ? pair_cells_smem_bytes<2> : pair_cells_smem_bytes<3>;
    k.pair_cells_rows = dim == 2 ? 3 : 9;
    k.max_row_cells = kMaxRowCells;
#define GCR_FILL(D_, FT_)                       \
    k.pair0 = StepKernels<D_, FT_>::pair0();    \
    k.pair1 = StepKernels<D_, FT_>::pair1();    \
    k.stage0 = StepKernels<D_, FT_>::stage0();  \
    k.stage1 = StepKernels<D_, FT_>::stage1();  \
    k.stage0f = StepKernels<D_, FT_>::stage0f(); \
    k.stage1f = StepKernels<D_, FT_>::stage1f(); \
    k.pair_cells[0] = StepKernels<D_, FT_>::pair_cells0(); \
    k.pair_cells[1] = StepKernels<D_, FT_>::pair_cells1(); \
    k.update = StepKernels<D_, FT_>::update();  \
    k.rigid0 = StepKernels<D_, FT_>::rigid0();  \
    k.rigid1 = StepKernels<D_, FT_>::rigid1();  \
    StepKernels<D_, FT_>::fill4(k);
    if (dim == 2 && precision == 0) {
        GCR_FILL(2, double)
    } else if (dim == 2) {
        GCR_FILL(2, float)
    } else if (precision == 0) {
        GCR_FILL(3, double)
    } else {
        GCR_FILL(3, float)
    }
#undef GCR_FILL
    if (dim == 2) {
        k.bin0 = (void *)k_bin<2, 0>;
        k.bin1 = (void *)k_bin<2, 1>;
        k.build0 = (void *)k_build<2, 0>;
        k.build1 = (void *)k_build<2, 1>;
        k.bin2 = (void *)k_bin<2, 2>;
        k.build2 = (void *)k_build<2, 2>;
        k.run_check = (void *)k_run_check<2>;
        k.motor[0] = (void *)k_motor<2, 0>;
        k.motor[1] = (void *)k_motor<2, 1>;
    } else {
        k.bin0 = (void *)k_bin<3, 0>;
        k.bin1 = (void *)k_bin<3, 1>;
        k.build0 = (void *)k_build<3, 0>;
        k.build1 = (void *)k_build<3, 1>;
        k.bin2 = (void *)k_bin<3, 2>;
        k.build2 = (void *)k_build<3, 2>;
        k.run_check = (void *)k_run_check<3>;
        k.motor[0] = (void *)k_motor<3, 0>;
        k.motor[1] = (void *)k_motor<3, 1>;
    }
    k.sort = (void *)k_sort;
    k.topo = (void *)k_topo;
    k.sys_dt = (void *)k_sys_dt;
    k.sys_end = (void *)k_sys_end;
    k.sys_mark = (void *)k_sys_mark;
    k.lists_plan = (void *)k_lists_plan;
    return k;
}

}  // namespace gcr
