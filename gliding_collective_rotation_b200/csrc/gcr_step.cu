// gcr_step.cu -- the SRK2 step kernels (sm_100a).
//
// One step of every resident system is five persistent, grid-stride launches
// over per-system tile tables:
//
//   pack<A>    per GPU cell: sort the slot contents by bead id, write packed
//              records of pos, clear the B counters
//   stage<0>   per bead: pair forces over the 3^d neighbour cells + bond,
//              bend and tangent + self-propulsion + predictor update
//              pos1 = (pos + dt/r F0 + sqrt(2 D dt) xi) mod L; bins pos1 into B
//   pack<B>    as pack<A> for pos1, clears the A counters
//   stage<1>   per bead: the same forces at pos1 accumulated onto F0; block
//              max of |F0+F1|^2; the last tile of each system picks dt
//              (SRK.py:323-353)
//   update     per bead: corrector pos = (pos + dt_used/(2r) (F0+F1)
//              + sqrt(2 D dt_used) xi) mod L, rotational diffusion
//              (SRK.py:398-423), bins pos into A; the last tile advances the
//              system's step bookkeeping
//
// The same xi is used by predictor and corrector (SRK.py:134-142, 385): it is
// drawn twice from the counter-based Philox stream keyed by (seed, bead,
// global step, stream), or read from an injected noise_vec snapshot.
//
// Reference functions restated per bead: forces.calc_chain_spring_forces
// (forces.py:285-403), forces.central_pair_force with forces.WCA
// (forces.py:57-145, 13-15), forces.self_propel (forces.py:206-224), the
// SRK2 stage updates (SRK.py:166-184, 355-396).
#include "gcr_device.cuh"
#include "gcr_kernels.h"

namespace gcr {

template <typename FT>
struct Rec;
template <>
struct Rec<float> {
    using type = float4;
};
struct alignas(32) Dbl4 {
    double x, y, z, w;
};
template <>
struct Rec<double> {
    using type = Dbl4;
};

// ------------------------------------------------------------------------
// bonded forces (forces.py:285-403).  A tile of TB beads stages the
// positions of beads begin-2 .. begin+TB+1 in shared memory, computes every
// bond (j, j+1) once and every bend once, then each bead gathers
//   F -= s_{b-1} d_{b-1}; F -= bwd_{b-1}; F += s_b d_b; F += fwd_b + bwd_b;
//   F -= fwd_{b+1}
// which is the order in which the reference's sequential loop adds them.
// ------------------------------------------------------------------------
template <int D, typename FT>
struct StageSmem {
    double *x;     // [TB+4][D] positions, index k <-> bead begin-2+k
    uint8_t *tp;   // [TB+4]    topology bits
    FT *bd;        // [TB+3][D] bond vector d_j = min_image(x_j - x_{j+1}), k <-> bond begin-2+k
    FT *bt;        // [TB+3][D] unit tangent of the bond (d itself when |d| = 0)
    FT *bf;        // [TB+3]    spring magnitude k (a/|d| - 1), 0 when |d| = 0
    FT *fw;        // [TB+2][D] bend "forward" term at bead begin-1+k
    FT *bw;        // [TB+2][D] bend "backward" term
    __device__ void carve(unsigned char *base, int TB)
    {
        x = reinterpret_cast<double *>(base);
        bd = reinterpret_cast<FT *>(x + (size_t)(TB + 4) * D);
        bt = bd + (size_t)(TB + 3) * D;
        bf = bt + (size_t)(TB + 3) * D;
        fw = bf + (TB + 3);
        bw = fw + (size_t)(TB + 2) * D;
        tp = reinterpret_cast<uint8_t *>(bw + (size_t)(TB + 2) * D);
    }
};

template <int D, typename FT>
size_t stage_smem_bytes(int TB)
{
    return (size_t)(TB + 4) * D * sizeof(double) + (size_t)(TB + 3) * (2 * D + 1) * sizeof(FT) +
           (size_t)(TB + 2) * 2 * D * sizeof(FT) + (size_t)(TB + 4) + 16;
}

// bend at a bead with forward tangent ti (its own bond) and backward tangent
// tj (the previous bond); false when the tangents are aligned
template <int D, typename FT>
__device__ __forceinline__ bool bend(const FT *ti, const FT *tj, FT theta0, FT kappa, FT *fwd, FT *bwd)
{
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
    phi *= kappa / sqrt(FT(1) - c * c);
#pragma unroll
    for (int i = 0; i < D; i++) {
        fwd[i] = phi * (c * tj[i] - ti[i]);
        bwd[i] = phi * (tj[i] - c * ti[i]);
    }
    return true;
}

// ------------------------------------------------------------------------
// pair forces (forces.py:57-145, rule forces.WCA) over the 3^d GPU cells
// around the bead; records are packed per cell, sorted by bead id
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
        float inv = __frcp_rn(ds);
        float i2 = inv * inv;
        return (i2 * i2) * (p0 - p1 * (i2 * inv));
    } else {
        double inv = 1.0 / ds, i2 = inv * inv;
        return (i2 * i2) * (p0 - p1 * (i2 * inv));
    }
}

// One bead's pair force, the bead taken in cell order: record k of the
// system's compact cell list.  All lanes of a warp sit in the same or
// neighbouring cells, so they walk the same candidate records (uniform trip
// counts, broadcast loads).  Candidates of cell c are records
// [cstart[c], cstart[c+1]), sorted by bead id.
// Pair force of the bead at record k of its system's compact cell list
// (forces.py:57-145).  Threads of a warp hold beads of the same or of
// neighbouring cells, so they walk the same candidate records (broadcast
// loads, similar trip counts).  The three cells cx-1, cx, cx+1 of one row are
// one contiguous range of records; a row that wraps around the box is two
// ranges.  Candidates of cell c are records [cstart[c], cstart[c+1]), sorted
// by bead id, so the sum is taken in a fixed order.
template <int D, typename FT>
__device__ __forceinline__ void pair_force_sorted(const SysP &p, const BatchArgs &A, int k, int &b_out, FT *F)
{
    using R = typename Rec<FT>::type;
    const int nc = p.nc;
    const int n = p.n;
    const R *__restrict__ rec = reinterpret_cast<const R *>(A.rec) + p.bead_off;
    const int *__restrict__ cs = A.cstart + p.cell_off;
    int c = __ldg(A.rcell + p.bead_off + k);
    c = (c < 0 || c >= p.n_cells) ? 0 : c;
    const int cx = c % nc;
    const int cy0 = (c / nc) % nc;
    const int cz0 = (D == 3) ? c / (nc * nc) : 0;
    FT own[3] = {FT(0), FT(0), FT(0)};
    double xb[3] = {0.0, 0.0, 0.0};
    int b, my_chain = 0;
    if constexpr (sizeof(FT) == 4) {
        float4 r = __ldg(rec + k);
        own[0] = r.x;
        own[1] = r.y;
        own[2] = r.z;
        b = __float_as_int(r.w);
        if (D == 2) my_chain = __float_as_int(r.z);
    } else {
        const double2 *q = reinterpret_cast<const double2 *>(rec + k);
        double2 r0 = __ldg(q), r1 = __ldg(q + 1);
        xb[0] = r0.x;
        xb[1] = r0.y;
        xb[2] = r1.x;
        b = (int)r1.y;
        if (D == 2) my_chain = (int)r1.x;
    }
    b_out = b;
    if ((unsigned)b >= (unsigned)n) return;  // inconsistent list: the caller flags it
    if (D == 3) my_chain = __ldg(p.chain + b);
    const FT rc2 = (FT)p.rc2, p0 = (FT)p.p0, p1 = (FT)p.p1, shift = (FT)p.shift;
    const FT hf = (FT)p.hf;
    const double L = p.L, half_L = p.half_L;
    const int nn = p.n_nearby;
    const int span = 3 * A.depth;
    // the row's ranges: [lo, hi) with the x offset -1/0/+1 cells changing at m1, m2
    const bool wrap_lo = cx == 0, wrap_hi = cx == nc - 1;
    const int x_first = wrap_lo ? 0 : cx - 1;          // first cell of the contiguous part
    const int x_last = wrap_hi ? nc - 1 : cx + 1;      // last cell of the contiguous part
    const int d_first = wrap_lo ? 0 : -1;              // its x offset in cells
    const int x_extra = wrap_lo ? nc - 1 : 0;          // the wrapped cell, if any
    const int d_extra = wrap_lo ? -1 : 1;
    const int n_seg = (wrap_lo || wrap_hi) ? 2 : 1;
    const int zlo = (D == 3) ? -1 : 0, zhi = (D == 3) ? 1 : 0;
    for (int dz = zlo; dz <= zhi; dz++) {
        int cz = 0;
        if (D == 3) {
            cz = cz0 + dz;
            cz = cz < 0 ? cz + nc : (cz >= nc ? cz - nc : cz);
        }
#pragma unroll
        for (int dy = -1; dy <= 1; dy++) {
            int cy = cy0 + dy;
            cy = cy < 0 ? cy + nc : (cy >= nc ? cy - nc : cy);
            const int row = (cz * nc + cy) * nc;
            for (int seg = 0; seg < n_seg; seg++) {
                int lo, hi, m1, m2, d0;
                if (seg == 0) {
                    lo = __ldg(cs + row + x_first);
                    m1 = __ldg(cs + row + x_first + 1);
                    m2 = __ldg(cs + row + x_first + 2);
                    hi = __ldg(cs + row + x_last + 1);
                    d0 = d_first;
                } else {
                    lo = __ldg(cs + row + x_extra);
                    hi = __ldg(cs + row + x_extra + 1);
                    m1 = m2 = 0x7fffffff;
                    d0 = d_extra;
                }
                // clamps keep every record index inside [0, n), whatever the list holds
                lo = lo < 0 ? 0 : (lo > n ? n : lo);
                hi = hi < lo ? lo : (hi > n ? n : hi);
                hi = hi - lo > span ? lo + span : hi;
                const FT o0 = (FT)d0 * hf, o1 = (FT)(d0 + 1) * hf, o2 = (FT)(d0 + 2) * hf;
                const FT oy = (FT)dy * hf, oz = (FT)dz * hf;
                for (int j = lo; j < hi; j++) {
                    int bj, cj = 0;
                    FT sep[3];
                    if constexpr (sizeof(FT) == 4) {
                        float4 r = __ldg(rec + j);
                        const FT ox = j < m1 ? o0 : (j < m2 ? o1 : o2);
                        sep[0] = (r.x - own[0]) + ox;
                        sep[1] = (r.y - own[1]) + oy;
                        if (D == 3) sep[2] = (r.z - own[2]) + oz;
                        else cj = __float_as_int(r.z);
                        bj = __float_as_int(r.w);
                    } else {
                        const double2 *q = reinterpret_cast<const double2 *>(rec + j);
                        double2 r0 = __ldg(q), r1 = __ldg(q + 1);
                        sep[0] = inbounds(r0.x, xb[0], half_L, L);
                        sep[1] = inbounds(r0.y, xb[1], half_L, L);
                        if (D == 3) sep[2] = inbounds(r1.x, xb[2], half_L, L);
                        else cj = (int)r1.x;
                        bj = (int)r1.y;
                    }
                    FT ds = sep[0] * sep[0] + sep[1] * sep[1];
                    if (D == 3) ds += sep[2] * sep[2];
                    if (!(FT(0) < ds && ds <= rc2)) continue;
                    if ((unsigned)bj >= (unsigned)n) continue;  // never index outside the system
                    int db = b - bj;
                    db = db < 0 ? -db : db;
                    if (nn < 0 || db <= nn) {
                        if (D == 3) cj = __ldg(p.chain + bj);
                        if (cj == my_chain) continue;
                    }
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
    }
}

template <int D>
__device__ __forceinline__ bool bin_bead(const SysP &p, const BatchArgs &A, int *cnt, const double *x, int b)
{
    int c[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < D; i++) c[i] = cell_coord(x[i], p.inv_h, p.nc);
    int64_t gc = p.cell_off + ((int64_t)c[2] * p.nc + c[1]) * p.nc + c[0];
    int slot = atomicAdd(cnt + gc, 1);
    if (slot < A.depth) {
        A.items[(gc << A.log_depth) + slot] = b;
        return true;
    }
    return false;
}

template <int D, typename FT>
__device__ __forceinline__ void noise_trans(const SysP &p, const SysS &s, int b, FT *xi)
{
    if (s.noise) {
        const double *q = s.noise + ((size_t)s.steps_done * p.n + b) * 2 * D;
#pragma unroll
        for (int i = 0; i < D; i++) xi[i] = (FT)q[i];
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
// kernels
// ------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(512) k_insert(BatchArgs A)
{
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        if (!ld_volatile(&s.active) || (ld_volatile(&s.flags) & kFlagFatal) || !p.calc_wca) continue;
        int b = tl.begin + threadIdx.x;
        if (b >= p.n || threadIdx.x >= A.tile_beads) continue;
        double x[3];
#pragma unroll
        for (int i = 0; i < D; i++) x[i] = p.pos[(size_t)b * D + i];
        if (!bin_bead<D>(p, A, A.cnt0, x, b)) atomicOr(&s.flags, kFlagCellOverflow);
    }
}

// exclusive scan of the binned counts of one tile of cells (block scan),
// clearing the other count buffer for the next binning
template <int WHICH>
__global__ void __launch_bounds__(512) k_scan_local(BatchArgs A)
{
    __shared__ int sh_w[16];
    __shared__ int sh_run;
    const int nt = *A.n_cell_tiles;
    const int *cnt = WHICH == 0 ? A.cnt0 : A.cnt1;
    int *other = WHICH == 0 ? A.cnt1 : A.cnt0;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        __syncthreads();
        const Tile tl = A.cell_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        if (threadIdx.x == 0)
            sh_run = ld_volatile(&s.active) && p.calc_wca && !(ld_volatile(&s.flags) & kFlagFatal);
        __syncthreads();
        if (!sh_run) continue;
        const int c = tl.begin + threadIdx.x;
        const bool in = c < p.n_cells && threadIdx.x < A.tile_cells;
        const int64_t gc = p.cell_off + c;
        int v = 0;
        if (in) {
            v = cnt[gc];
            v = v < A.depth ? v : A.depth;
            other[gc] = 0;
        }
        // block exclusive scan
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh_w[w] = x;
        __syncthreads();
        if (w == 0) {
            int nw = (blockDim.x + 31) >> 5;
            int y = lane < nw ? sh_w[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += z;
            }
            if (lane < nw) sh_w[lane] = y;  // inclusive prefix of warp totals
        }
        __syncthreads();
        int ex = x - v + (w > 0 ? sh_w[w - 1] : 0);
        if (in) A.cstart[gc] = ex;
        if (threadIdx.x == blockDim.x - 1) A.tsum[t] = ex + v;
    }
}

// exclusive scan of the tile totals of each system (one CTA per system);
// writes the end sentinel cstart[n_cells]
__global__ void __launch_bounds__(256) k_scan_tiles(BatchArgs A, int n_slots)
{
    __shared__ int sh_w[8];
    __shared__ int sh_carry;
    const int sys = blockIdx.x;
    if (sys >= n_slots) return;
    const SysP &p = A.P[sys];
    SysS &s = A.S[sys];
    if (!(s.active && p.calc_wca && !(s.flags & kFlagFatal)) || p.n_cell_tiles == 0) return;
    if (p.cell_tile0 < 0 || p.cell_tile0 + p.n_cell_tiles > *A.n_cell_tiles) {
        if (threadIdx.x == 0) atomicOr(&s.flags, kFlagListCorrupt);
        return;
    }
    if (threadIdx.x == 0) sh_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < p.n_cell_tiles; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const int v = t < p.n_cell_tiles ? A.tsum[p.cell_tile0 + t] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh_w[w] = x;
        __syncthreads();
        if (w == 0) {
            int nw = blockDim.x >> 5;
            int y = lane < nw ? sh_w[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += z;
            }
            if (lane < nw) sh_w[lane] = y;
        }
        __syncthreads();
        const int carry = sh_carry;
        const int ex = x - v + (w > 0 ? sh_w[w - 1] : 0) + carry;
        if (t < p.n_cell_tiles) A.toff[p.cell_tile0 + t] = ex;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) sh_carry = ex + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) A.cstart[p.cell_off + p.n_cells] = sh_carry;
}

// per GPU cell: final start, the slot contents sorted by bead id, packed
// records of the build's positions written to the compact list
template <int D, typename FT, int WHICH>
__global__ void __launch_bounds__(512) k_pack(BatchArgs A)
{
    using R = typename Rec<FT>::type;
    const int nt = *A.n_cell_tiles;
    const int *cnt = WHICH == 0 ? A.cnt0 : A.cnt1;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.cell_tiles[t];
        const SysP &p = A.P[tl.sys];
        const SysS &s = A.S[tl.sys];
        bool run = ld_volatile(&s.active) && p.calc_wca && !(ld_volatile(&s.flags) & kFlagFatal);
        if (!run) continue;
        int c = tl.begin + threadIdx.x;
        if (c >= p.n_cells || threadIdx.x >= A.tile_cells) continue;
        const int64_t gc = p.cell_off + c;
        int n = cnt[gc];
        n = n < A.depth ? n : A.depth;
        const int start = A.toff[t] + A.cstart[gc];
        A.cstart[gc] = start;
        if (n == 0) continue;
        if (start < 0 || start + n > p.n) {
            // never write outside the system's part of the list
            atomicOr((int *)&s.flags, kFlagListCorrupt);
            continue;
        }
        int *it = A.items + (gc << A.log_depth);
        const double *X = WHICH == 0 ? p.pos : p.pos1;
        int cc[3];
        cc[0] = c % p.nc;
        cc[1] = (c / p.nc) % p.nc;
        cc[2] = (D == 3) ? c / (p.nc * p.nc) : 0;
        double ctr[3];
#pragma unroll
        for (int i = 0; i < 3; i++) ctr[i] = ((double)cc[i] + 0.5) * p.h;
        R *out = reinterpret_cast<R *>(A.rec) + p.bead_off + start;
        int *ocell = A.rcell + p.bead_off + start;
        auto emit = [&](int j, int b) {
            double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < D; i++) x[i] = X[(size_t)b * D + i];
            R r;
            // 2D records carry the bead's chain id in the spare z slot, so the
            // pair loop's exclusion test needs no second load
            if constexpr (sizeof(FT) == 4) {
                r.x = (float)(x[0] - ctr[0]);
                r.y = (float)(x[1] - ctr[1]);
                r.z = (D == 3) ? (float)(x[2] - ctr[2]) : __int_as_float(__ldg(p.chain + b));
                r.w = __int_as_float(b);
            } else {
                r.x = x[0];
                r.y = x[1];
                r.z = (D == 3) ? x[2] : (double)__ldg(p.chain + b);
                r.w = (double)b;
            }
            out[j] = r;
            ocell[j] = c;
        };
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
                if (j < n) emit(j, v[j]);
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
            for (int j = 0; j < n; j++) emit(j, it[j]);
        }
    }
}

// pair forces in cell order (forces.py:57-145, rule forces.WCA); writes the
// pair force of every bead to fp[bead]
template <int D, typename FT>
__global__ void __launch_bounds__(512) k_pair(BatchArgs A)
{
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        if (!ld_volatile(&s.active) || (ld_volatile(&s.flags) & kFlagFatal) || !p.calc_wca) continue;
        const int k = tl.begin + threadIdx.x;
        if (k >= p.n || threadIdx.x >= A.tile_beads) continue;
        FT F[3] = {FT(0), FT(0), FT(0)};
        int b;
        pair_force_sorted<D, FT>(p, A, k, b, F);
        if (b < 0 || b >= p.n) {
            atomicOr(&s.flags, kFlagListCorrupt);
            continue;
        }
        FT *fp = reinterpret_cast<FT *>(A.fp) + (size_t)(p.bead_off + b) * D;
#pragma unroll
        for (int i = 0; i < D; i++) fp[i] = F[i];
    }
}

template <int D, typename FT, int STAGE>
__global__ void __launch_bounds__(512) k_stage(BatchArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long sh_bits[16];
    __shared__ int sh_run;
    const int TB = blockDim.x;
    StageSmem<D, FT> sm;
    sm.carve(smem_raw, TB);
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        __syncthreads();  // the previous tile is done with shared memory
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        // one decision per CTA: other CTAs may raise the system's flags while
        // this one runs, and every thread must reach the same barriers
        if (threadIdx.x == 0) sh_run = ld_volatile(&s.active) && !(ld_volatile(&s.flags) & kFlagFatal);
        __syncthreads();
        if (!sh_run) continue;
        const int n = p.n;
        const int base = tl.begin - 2;
        const double *__restrict__ X = STAGE == 0 ? p.pos : p.pos1;
        // 1. positions and topology of beads begin-2 .. begin+TB+1
        for (int k = threadIdx.x; k < TB + 4; k += TB) {
            int m = base + k;
            if (m >= 0 && m < n) {
#pragma unroll
                for (int i = 0; i < D; i++) sm.x[k * D + i] = __ldg(X + (size_t)m * D + i);
                sm.tp[k] = A.topo[p.bead_off + m];
            } else {
                sm.tp[k] = 0;
            }
        }
        __syncthreads();
        const bool springs = p.calc_springs, cb = p.calc_bend;
        if (springs) {
            // 2. every bond (j, j+1) of the tile once
            const FT kspring = (FT)p.k;
            for (int k = threadIdx.x; k < TB + 3; k += TB) {
                FT d[D], tt[D], f = FT(0);
#pragma unroll
                for (int i = 0; i < D; i++) d[i] = tt[i] = FT(0);
                if (sm.tp[k] & kHasNext) {
                    FT r2 = FT(0);
#pragma unroll
                    for (int i = 0; i < D; i++) {
                        d[i] = (FT)inbounds(sm.x[k * D + i], sm.x[(k + 1) * D + i], p.half_L, p.L);
                        r2 += d[i] * d[i];
                    }
                    if (r2 != FT(0)) {
                        const FT a = (FT)__ldg(p.rest + __ldg(p.chain + base + k));
                        FT inv = FT(1) / sqrt(r2);
                        f = kspring * (a * inv - FT(1));
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
                const FT kappa = (FT)p.kappa, theta0 = (FT)p.theta0;
                for (int k = threadIdx.x; k < TB + 2; k += TB) {
                    FT fw[D], bw[D];
#pragma unroll
                    for (int i = 0; i < D; i++) fw[i] = bw[i] = FT(0);
                    const uint8_t tp = sm.tp[k + 1];
                    if ((tp & kHasPrev) && (tp & kHasNext)) {
                        if (!bend<D, FT>(sm.bt + (k + 1) * D, sm.bt + k * D, theta0, kappa, fw, bw)) {
#pragma unroll
                            for (int i = 0; i < D; i++) fw[i] = bw[i] = FT(0);
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
        double mf2 = 0.0;
        if (b < n) {
            FT *frc = reinterpret_cast<FT *>(p.frc);
            FT *tan = reinterpret_cast<FT *>(p.tan);
            double xb[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < D; i++) xb[i] = sm.x[(tid + 2) * D + i];
            FT F[3], tg[3];
#pragma unroll
            for (int i = 0; i < D; i++) {
                F[i] = STAGE == 0 ? FT(0) : frc[(size_t)b * D + i];
                tg[i] = tan[(size_t)b * D + i];
            }
            bool tang_set = false;
            if (springs) {
                const uint8_t tp = sm.tp[tid + 2];
                const bool prev = tp & kHasPrev, next = tp & kHasNext;
                if (prev) {
                    const FT f = sm.bf[tid + 1];
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] -= sm.bd[(tid + 1) * D + i] * f;
                    if ((tp & kHasPrev2) && cb) {
#pragma unroll
                        for (int i = 0; i < D; i++) F[i] -= sm.bw[tid * D + i];
                    }
                }
                if (next) {
                    const FT f = sm.bf[tid + 2];
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] += sm.bd[(tid + 2) * D + i] * f;
                }
                if (prev && next && cb) {
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] += sm.fw[(tid + 1) * D + i] + sm.bw[(tid + 1) * D + i];
                }
                if ((tp & kHasNext2) && cb) {
#pragma unroll
                    for (int i = 0; i < D; i++) F[i] -= sm.fw[(tid + 2) * D + i];
                }
                if (p.get_orient && (prev || next)) {
                    const FT *ti = sm.bt + (tid + 2) * D, *tj = sm.bt + (tid + 1) * D;
                    if (prev && next) {
                        FT c = FT(0);
#pragma unroll
                        for (int i = 0; i < D; i++) c += ti[i] * tj[i];
                        if (FT(-1) < c && c < FT(1)) {
                            FT coeff = FT(1) / sqrt(FT(2) * (FT(1) + c));
#pragma unroll
                            for (int i = 0; i < D; i++) tg[i] = coeff * (ti[i] + tj[i]);
                        } else {
#pragma unroll
                            for (int i = 0; i < D; i++) tg[i] = ti[i];
                        }
                    } else if (next) {  // head bead
#pragma unroll
                        for (int i = 0; i < D; i++) tg[i] = ti[i];
                    } else {  // tail bead
#pragma unroll
                        for (int i = 0; i < D; i++) tg[i] = tj[i];
                    }
                    tang_set = true;
                }
            }
            if (p.calc_wca) {
                const FT *fp = reinterpret_cast<const FT *>(A.fp) + (size_t)(p.bead_off + b) * D;
#pragma unroll
                for (int i = 0; i < D; i++) F[i] += fp[i];
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
#pragma unroll
            for (int i = 0; i < D; i++) frc[(size_t)b * D + i] = F[i];
            if (tang_set) {
#pragma unroll
                for (int i = 0; i < D; i++) tan[(size_t)b * D + i] = tg[i];
            }
            if (STAGE == 0) {
                // the step's translational noise, drawn once and kept for the corrector
                FT xi[3] = {FT(0), FT(0), FT(0)};
                if (p.D > 0.0) {
                    noise_trans<D, FT>(p, s, b, xi);
                    FT *xs = reinterpret_cast<FT *>(A.xi) + (size_t)(p.bead_off + b) * D;
#pragma unroll
                    for (int i = 0; i < D; i++) xs[i] = xi[i];
                }
                // predictor: pos1 = (pos + dt/r F0 + sqrt(2 D dt) xi) mod L
                const double dt = s.dt;
                const double dt_eff = dt * 1.0 / p.radius;
                const double s2 = sqrt(2.0 * dt * p.D);
                double x1[3] = {0.0, 0.0, 0.0};
                bool finite = true;
#pragma unroll
                for (int i = 0; i < D; i++) {
                    x1[i] = srk_update<FT>(xb[i], dt_eff, s2, F[i], xi[i], p.L);
                    finite &= isfinite(x1[i]);
                    p.pos1[(size_t)b * D + i] = x1[i];
                }
                if (!finite)
                    atomicOr(&s.flags, kFlagNonFinite);
                else if (p.calc_wca && !bin_bead<D>(p, A, A.cnt1, x1, b))
                    atomicOr(&s.flags, kFlagCellOverflow);
            } else {
                // |F0+F1|^2 in FP64 for the dt rule (SRK.py:328)
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < D; i++) acc += (double)F[i] * (double)F[i];
                mf2 = acc;
            }
        }
        if (STAGE == 1) {
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

template <int D, typename FT>
__global__ void __launch_bounds__(512) k_update(BatchArgs A)
{
    const int nt = *A.n_bead_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const Tile tl = A.bead_tiles[t];
        const SysP &p = A.P[tl.sys];
        SysS &s = A.S[tl.sys];
        // no barriers in this kernel: a per-thread decision is safe
        if (!ld_volatile(&s.active) || (ld_volatile(&s.flags) & kFlagFatal)) continue;
        const int b = tl.begin + threadIdx.x;
        if (b >= p.n || threadIdx.x >= A.tile_beads) continue;
        const FT *frc = reinterpret_cast<const FT *>(p.frc);
        const double dtu = s.dt_used;
        const double dt_eff = dtu * 0.5 / p.radius;
        const double s2 = sqrt(2.0 * dtu * p.D);
        FT xi[3] = {FT(0), FT(0), FT(0)};
        if (p.D > 0.0) {
            const FT *xs = reinterpret_cast<const FT *>(A.xi) + (size_t)(p.bead_off + b) * D;
#pragma unroll
            for (int i = 0; i < D; i++) xi[i] = xs[i];
        }
        double x[3] = {0.0, 0.0, 0.0};
        bool finite = true;
#pragma unroll
        for (int i = 0; i < D; i++) {
            x[i] = srk_update<FT>(p.pos[(size_t)b * D + i], dt_eff, s2, frc[(size_t)b * D + i], xi[i], p.L);
            finite &= isfinite(x[i]);
            p.pos[(size_t)b * D + i] = x[i];
        }
        if (!finite) atomicOr(&s.flags, kFlagNonFinite);
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
        if (finite && p.calc_wca && !bin_bead<D>(p, A, A.cnt0, x, b)) atomicOr(&s.flags, kFlagNextOverflow);
    }
}

// per-system dt rule after stage 1 (SRK.py:323-353): one thread per slot
__global__ void k_sys_dt(BatchArgs A, int n_slots)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slots) return;
    const SysP &p = A.P[i];
    SysS &s = A.S[i];
    if (!s.active || (s.flags & kFlagFatal)) return;
    double mf2s = __longlong_as_double((long long)s.max_f2);
    double S = p.sqrt2D + 0.5 * sqrt(mf2s) / p.radius;
    double dt;
    if (S == 0.0)
        dt = p.dtmax;
    else {
        double q = p.mdps / S;
        dt = (q < p.dtmax) ? q : p.dtmax;
    }
    double dt_used = p.rk * dt;
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
                (s.elapsed < s.max_dt_usable || s.max_dt_usable < 0.0) && !(s.flags & kFlagNextOverflow);
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

// ------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------
template <int D, typename FT>
struct StepKernels {
    static void *pair() { return (void *)k_pair<D, FT>; }
    static void *insert() { return (void *)k_insert<D>; }
    static void *pack0() { return (void *)k_pack<D, FT, 0>; }
    static void *pack1() { return (void *)k_pack<D, FT, 1>; }
    static void *stage0() { return (void *)k_stage<D, FT, 0>; }
    static void *stage1() { return (void *)k_stage<D, FT, 1>; }
    static void *update() { return (void *)k_update<D, FT>; }
};

KernelSet kernel_set(int dim, int precision)
{
    KernelSet k{};
    if (dim == 2)
        k.stage_smem = precision == 0 ? stage_smem_bytes<2, double> : stage_smem_bytes<2, float>;
    else
        k.stage_smem = precision == 0 ? stage_smem_bytes<3, double> : stage_smem_bytes<3, float>;
#define GCR_FILL(D_, FT_)                           \
    k.pair = StepKernels<D_, FT_>::pair();          \
    k.insert = StepKernels<D_, FT_>::insert();      \
    k.pack0 = StepKernels<D_, FT_>::pack0();        \
    k.pack1 = StepKernels<D_, FT_>::pack1();        \
    k.stage0 = StepKernels<D_, FT_>::stage0();      \
    k.stage1 = StepKernels<D_, FT_>::stage1();      \
    k.update = StepKernels<D_, FT_>::update();
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
    k.topo = (void *)k_topo;
    k.sys_dt = (void *)k_sys_dt;
    k.scan_local0 = (void *)k_scan_local<0>;
    k.scan_local1 = (void *)k_scan_local<1>;
    k.scan_tiles = (void *)k_scan_tiles;
    k.sys_end = (void *)k_sys_end;
    return k;
}

}  // namespace gcr
