// gcr_lists.cu -- device builders of the reference's own list formats, the
// order-parameter reduction and small exports.
//
//   where_is_bead = int(pos // h)          SRK.py:432-434 (CPython floor division)
//   grid_list fill, bead-index order      updates.update_grid_list_mini, updates.py:502-522
//   nbor_list, cell-window loop order     updates.update_nbor_list,      updates.py:586-669
//   nbor_list, all-pairs loop order       updates.update_nbor_list_few,  updates.py:672-734
//   chain angle and P, S, director        output_methods.py:492-510, analysis.py:294-328
//
// The list builders reproduce the reference's arrays exactly (same counts,
// same entries, same order); distances are evaluated with explicitly rounded
// FP64 operations so that no contraction changes a borderline comparison.
#include "gcr_device.cuh"
#include "gcr_kernels.h"

namespace gcr {

__global__ void k_ref_where(int dim, const double *__restrict__ pos, int n, double spacing, int64_t *w)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    for (int i = 0; i < dim; i++) w[(size_t)b * 3 + i] = (int64_t)py_floordiv(pos[(size_t)b * dim + i], spacing);
    if (dim == 2) w[(size_t)b * 3 + 2] = 0;
}

__global__ void k_ref_grid_zero(int64_t *grid, int64_t n_cells, int64_t depth1)
{
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n_cells) grid[c * depth1] = 0;
}

__global__ void k_ref_grid_fill(int dim, const int64_t *__restrict__ w, int n, int64_t ng, int64_t ngz,
                                int64_t *grid, int64_t depth1, int *err)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    int64_t x = w[(size_t)b * 3], y = w[(size_t)b * 3 + 1], z = w[(size_t)b * 3 + 2];
    // a bead at exactly x == L has index n_grid; the reference then writes
    // outside its array, here it is left out of every cell
    if (x < 0 || x >= ng || y < 0 || y >= ng || z < 0 || z >= ngz) return;
    int64_t *cell = grid + ((x * ng + y) * ngz + z) * depth1;
    unsigned long long old = atomicAdd((unsigned long long *)cell, 1ull);
    int64_t cnt = (int64_t)old + 1;
    if (cnt < depth1 - 2)
        cell[cnt] = b;
    else
        atomicOr(err, 1);
}

__global__ void k_ref_grid_sort(int64_t *grid, int64_t n_cells, int64_t depth1)
{
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    int64_t *cell = grid + c * depth1;
    int64_t m = cell[0];
    if (m > depth1 - 3) m = depth1 - 3;
    for (int64_t j = 2; j <= m; j++) {
        int64_t key = cell[j];
        int64_t q = j - 1;
        while (q >= 1 && cell[q] > key) {
            cell[q + 1] = cell[q];
            q--;
        }
        cell[q + 1] = key;
    }
}

__device__ __forceinline__ int64_t pmod(int64_t a, int64_t m)
{
    int64_t r = a % m;
    return r < 0 ? r + m : r;
}

// updates.update_nbor_list for one population against itself (same_pop)
__global__ void k_ref_nbor_cells(int dim, const double *__restrict__ pos, const int32_t *__restrict__ chain,
                                 int n, double L, const int64_t *__restrict__ w,
                                 const int64_t *__restrict__ grid, int64_t ng, int64_t ngz, int64_t depth1,
                                 int64_t gw, double max_dist_sq, int n_nearby, int64_t *nb, int64_t nbd1,
                                 int *err)
{
    int b1 = blockIdx.x * blockDim.x + threadIdx.x;
    if (b1 >= n) return;
    const bool b3d = dim == 3;
    const double half_L = L / 2.0;
    int64_t *row = nb + (size_t)b1 * nbd1;
    int64_t count = 0;
    int64_t dg_start = -(gw < ng / 2 ? gw : ng / 2);
    int64_t dg_end = (1 + gw < ng + dg_start) ? 1 + gw : ng + dg_start;
    bool flags[3] = {false, false, false};
    int64_t wb[3] = {w[(size_t)b1 * 3], w[(size_t)b1 * 3 + 1], w[(size_t)b1 * 3 + 2]};
    for (int i = 0; i < dim; i++) flags[i] = (wb[i] < gw + 1) || (wb[i] >= ng - (gw + 1));
    double x1[3];
    for (int i = 0; i < dim; i++) x1[i] = pos[(size_t)b1 * dim + i];
    int64_t gz0 = b3d ? dg_start + wb[2] : 0, gz1 = b3d ? wb[2] + dg_end : 1;
    bool overflow = false;
    for (int64_t gx2r = dg_start + wb[0]; gx2r < wb[0] + dg_end && !overflow; gx2r++) {
        int64_t gx2 = flags[0] ? pmod(gx2r, ng) : gx2r;
        for (int64_t gy2r = dg_start + wb[1]; gy2r < wb[1] + dg_end && !overflow; gy2r++) {
            int64_t gy2 = flags[1] ? pmod(gy2r, ng) : gy2r;
            for (int64_t gz2r = gz0; gz2r < gz1 && !overflow; gz2r++) {
                int64_t gz2 = (b3d && flags[2]) ? pmod(gz2r, ng) : gz2r;
                if (gx2 < 0 || gx2 >= ng || gy2 < 0 || gy2 >= ng || gz2 < 0 || gz2 >= ngz) continue;
                const int64_t *cell = grid + ((gx2 * ng + gy2) * ngz + gz2) * depth1;
                int64_t m = cell[0];
                if (m > depth1 - 3) m = depth1 - 3;
                for (int64_t k = 0; k < m; k++) {
                    int64_t b2 = cell[1 + k];
                    if (chain[b1] == chain[b2]) {
                        if (n_nearby < 0) continue;
                        int64_t d = b1 - b2;
                        d = d < 0 ? -d : d;
                        if (d <= n_nearby) continue;
                    }
                    double ds = 0.0;
                    for (int i = 0; i < dim; i++) {
                        double sep = __dsub_rn(pos[(size_t)b2 * dim + i], x1[i]);
                        if (flags[i]) {
                            if (sep < -half_L)
                                sep = __dadd_rn(sep, L);
                            else if (sep >= half_L)
                                sep = __dsub_rn(sep, L);
                        }
                        ds = __dadd_rn(ds, __dmul_rn(sep, sep));
                    }
                    if (ds <= max_dist_sq) {
                        if (count + 1 >= nbd1) {
                            overflow = true;
                            break;
                        }
                        count++;
                        row[count] = b2;
                    }
                }
            }
        }
    }
    if (overflow) {
        row[0] = -1;
        atomicOr(err, 2);
    } else {
        row[0] = count;
    }
}

// updates.update_nbor_list_few (all pairs, cell window checked per pair)
__global__ void k_ref_nbor_few(int dim, const double *__restrict__ pos, const int32_t *__restrict__ chain,
                               int n, double L, const int64_t *__restrict__ w, int64_t ng, int64_t gw,
                               double max_dist_sq, int n_nearby, int64_t *nb, int64_t nbd1, int *err)
{
    int b1 = blockIdx.x * blockDim.x + threadIdx.x;
    if (b1 >= n) return;
    const double half_L = L / 2.0;
    const double half_ng = (double)ng / 2.0;
    int64_t *row = nb + (size_t)b1 * nbd1;
    int64_t count = 0;
    for (int b2 = 0; b2 < n; b2++) {
        bool use = true;
        for (int i = 0; i < dim; i++) {
            double dg = (double)(w[(size_t)b2 * 3 + i] - w[(size_t)b1 * 3 + i]);
            if (dg < -half_ng)
                dg += (double)ng;
            else if (dg >= half_ng)
                dg -= (double)ng;
            if (fabs(dg) > (double)gw) {
                use = false;
                break;
            }
        }
        if (!use) continue;
        if (chain[b1] == chain[b2]) {
            if (n_nearby < 0) continue;
            int d = b1 - b2;
            d = d < 0 ? -d : d;
            if (d <= n_nearby) continue;
        }
        double ds = 0.0;
        for (int i = 0; i < dim; i++) {
            double sep = __dsub_rn(pos[(size_t)b2 * dim + i], pos[(size_t)b1 * dim + i]);
            if (sep < -half_L)
                sep = __dadd_rn(sep, L);
            else if (sep >= half_L)
                sep = __dsub_rn(sep, L);
            ds = __dadd_rn(ds, __dmul_rn(sep, sep));
        }
        if (ds <= max_dist_sq) {
            if (count + 1 >= nbd1) {
                row[0] = -1;
                atomicOr(err, 2);
                return;
            }
            count++;
            row[count] = b2;
        }
    }
    row[0] = count;
}

cudaError_t launch_reference_lists(int dim, const SysP &p, int64_t n_grid, int64_t grid_window,
                                   int64_t *where_is_bead, int64_t *grid_list, int64_t grid_depth1,
                                   int64_t *nbor_list, int64_t nbor_depth1, int *d_err, cudaStream_t st)
{
    const int n = p.n;
    const int bs = 256;
    const int gb = (n + bs - 1) / bs;
    const double spacing = p.L / (double)n_grid;
    const int64_t ngz = dim == 3 ? n_grid : 1;
    const int64_t n_cells = n_grid * n_grid * ngz;
    k_ref_where<<<gb, bs, 0, st>>>(dim, p.pos, n, spacing, where_is_bead);
    if (grid_list) {
        k_ref_grid_zero<<<(unsigned)((n_cells + bs - 1) / bs), bs, 0, st>>>(grid_list, n_cells, grid_depth1);
        k_ref_grid_fill<<<gb, bs, 0, st>>>(dim, where_is_bead, n, n_grid, ngz, grid_list, grid_depth1, d_err);
        k_ref_grid_sort<<<(unsigned)((n_cells + bs - 1) / bs), bs, 0, st>>>(grid_list, n_cells, grid_depth1);
    }
    if (nbor_list) {
        const double hg = (double)grid_window * p.L / (double)n_grid;
        const double max_dist_sq = hg * hg;
        int64_t n_pow = 1;
        for (int i = 0; i < dim; i++) n_pow *= n_grid;
        if (grid_list && !(n < n_pow))
            k_ref_nbor_cells<<<gb, bs, 0, st>>>(dim, p.pos, p.chain, n, p.L, where_is_bead, grid_list, n_grid, ngz,
                                                grid_depth1, grid_window, max_dist_sq, p.n_nearby, nbor_list,
                                                nbor_depth1, d_err);
        else
            k_ref_nbor_few<<<gb, bs, 0, st>>>(dim, p.pos, p.chain, n, p.L, where_is_bead, n_grid, grid_window,
                                              max_dist_sq, p.n_nearby, nbor_list, nbor_depth1, d_err);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// order parameters: one block per system, fixed reduction order
// ---------------------------------------------------------------------------
template <typename FT>
__device__ void order_params_block(int dim, const FT *__restrict__ tan, const int32_t *__restrict__ cs,
                                   int n_chains, double *out)
{
    // one CTA of 1024 threads, a fixed reduction tree: the same bits from
    // gcr_order_params and from the in-graph series
    __shared__ double sh[4][1024];
    double ex = 0.0, ey = 0.0, q11 = 0.0, q12 = 0.0;
    for (int c = threadIdx.x; c < n_chains; c += blockDim.x) {
        double sx = 0.0, sy = 0.0;
        for (int b = cs[c]; b < cs[c + 1]; b++) {
            sx += (double)tan[(size_t)b * dim];
            sy += (double)tan[(size_t)b * dim + 1];
        }
        double phi = atan2(sy, sx);
        double cx = cos(phi), sy2 = sin(phi);
        ex += cx;
        ey += sy2;
        q11 += 2.0 * cx * cx - 1.0;
        q12 += 2.0 * cx * sy2;
    }
    sh[0][threadIdx.x] = ex;
    sh[1][threadIdx.x] = ey;
    sh[2][threadIdx.x] = q11;
    sh[3][threadIdx.x] = q12;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double P = sqrt(sh[0][0] * sh[0][0] + sh[1][0] * sh[1][0]) / (double)n_chains;
        double Sf = sqrt(sh[2][0] * sh[2][0] + sh[3][0] * sh[3][0]);
        out[0] = P;
        out[1] = Sf / (double)n_chains;
        out[2] = atan((Sf - sh[2][0]) / sh[3][0]);
    }
}

template <typename FT>
__global__ void __launch_bounds__(1024) k_order(int dim, const FT *__restrict__ tan, const int32_t *__restrict__ cs,
                                                int n_chains, double *out)
{
    order_params_block<FT>(dim, tan, cs, n_chains, out);
}

// The in-graph series: one CTA per slot after each step; a system whose call
// asked for a series and whose step count in the call, plus the call's phase,
// has just reached a multiple of series_every appends (step, elapsed, P, S,
// angle).  Every thread of a CTA reads the same state words (the step kernels
// are done), so all take one branch.
template <typename FT>
__global__ void __launch_bounds__(1024) k_observe(BatchArgs A, int dim)
{
    pdl_wait();
    const int i = blockIdx.x;
    if (i >= A.n_slots) return;
    const SysP &p = A.P[i];
    SysS &s = A.S[i];
    if (!s.series || s.series_every <= 0 || s.steps_done == 0 || s.steps_done == s.series_mark) return;
    if ((s.steps_done + s.series_phase) % s.series_every != 0 || (s.flags & kFlagFatal)) return;
    __shared__ double row[3];
    order_params_block<FT>(dim, reinterpret_cast<const FT *>(p.tan), p.chain_start, p.n_chains, row);
    __syncthreads();
    if (threadIdx.x == 0) {
        s.series_mark = s.steps_done;
        if (s.series_rows < s.series_cap) {
            double *r = s.series + (size_t)s.series_rows * 5;
            r[0] = (double)s.step;
            r[1] = s.elapsed;
            r[2] = row[0];
            r[3] = row[1];
            r[4] = row[2];
            s.series_rows += 1;
        } else {
            s.flags |= kFlagSeriesFull;
        }
    }
}

void *observe_kernel(int precision)
{
    return precision == 0 ? (void *)k_observe<double> : (void *)k_observe<float>;
}

cudaError_t launch_order_params(int dim, int precision, const SysP &p, const int32_t *chain_start,
                                double *d_out, cudaStream_t st)
{
    if (precision == 0)
        k_order<double><<<1, 1024, 0, st>>>(dim, (const double *)p.tan, chain_start, p.n_chains, d_out);
    else
        k_order<float><<<1, 1024, 0, st>>>(dim, (const float *)p.tan, chain_start, p.n_chains, d_out);
    return cudaGetLastError();
}

// chain start offsets; flags chain ids that do not run 0, 1, ..., n_chains-1
// in order (chains must be contiguous, non-empty bead ranges): the first
// bead is in chain 0, each next bead in the same chain or the next one, the
// last bead in chain n_chains-1 -- so every chain id owns a bead range and
// every start offset is written
__global__ void k_chain_starts(const int32_t *__restrict__ chain, int n, int n_chains, int32_t *cs, int *err)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b == 0) cs[n_chains] = n;
    if (b >= n) return;
    int c = chain[b];
    const int step = b > 0 ? c - chain[b - 1] : (c == 0 ? 0 : -1);
    if (c < 0 || c >= n_chains || step < 0 || step > 1 || (b == n - 1 && c != n_chains - 1)) {
        atomicOr(err, 4);
        return;
    }
    if (b == 0 || step == 1) cs[c] = b;
}

// beads of the longest chain (err[1])
__global__ void k_chain_longest(const int32_t *__restrict__ cs, int n_chains, const int *err, int *longest)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chains || *err) return;
    atomicMax(longest, cs[c + 1] - cs[c]);
}

cudaError_t launch_chain_starts(const int32_t *chain, int n, int n_chains, int32_t *chain_start, int *d_err,
                                cudaStream_t st)
{
    k_chain_starts<<<(n + 255) / 256, 256, 0, st>>>(chain, n, n_chains, chain_start, d_err);
    k_chain_longest<<<(n_chains + 255) / 256, 256, 0, st>>>(chain_start, n_chains, d_err, d_err + 1);
    return cudaGetLastError();
}

__global__ void k_cell_assign(int dim, const double *__restrict__ pos, int n, double inv_h, int nc, int32_t *out)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    int c[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) c[i] = cell_coord(pos[(size_t)b * dim + i], inv_h, nc);
    out[b] = (c[2] * nc + c[1]) * nc + c[0];
}

cudaError_t launch_cell_assignment(int dim, const SysP &p, int32_t *cell_of_bead, cudaStream_t st)
{
    k_cell_assign<<<(p.n + 255) / 256, 256, 0, st>>>(dim, p.pos, p.n, p.inv_h, p.nc, cell_of_bead);
    return cudaGetLastError();
}

__global__ void k_unwrap(int dim, const double *__restrict__ pos, const int *__restrict__ img, int n, double L,
                         double *out)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * dim) return;
    out[i] = pos[i] + L * (double)img[i];
}

cudaError_t launch_unwrap(int dim, const double *pos, const int *img, int n, double L, double *out, cudaStream_t st)
{
    int64_t m = (int64_t)n * dim;
    if (m <= 0) return cudaSuccess;
    k_unwrap<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(dim, pos, img, n, L, out);
    return cudaGetLastError();
}

template <int D>
__global__ void k_philox_noise(uint64_t seed, int64_t step, int64_t n, int do_trans, int do_rot, double *out)
{
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    double z[D];
    double *row = out + b * 2 * D;
    if (do_trans) {
        philox_normals<D>(seed, (uint32_t)b, step, false, z);
        for (int i = 0; i < D; i++) row[i] = z[i];
    }
    if (do_rot) {
        philox_normals<D>(seed, (uint32_t)b, step, true, z);
        for (int i = 0; i < D; i++) row[D + i] = z[i];
    }
}

cudaError_t launch_philox_noise(int dim, uint64_t seed, int64_t step, int64_t n, int do_trans, int do_rot,
                                double *out, cudaStream_t st)
{
    unsigned g = (unsigned)((n + 255) / 256);
    if (dim == 2)
        k_philox_noise<2><<<g, 256, 0, st>>>(seed, step, n, do_trans, do_rot, out);
    else
        k_philox_noise<3><<<g, 256, 0, st>>>(seed, step, n, do_trans, do_rot, out);
    return cudaGetLastError();
}

// the neighbour list of one system, slot-major -> bead-major, and its total
__global__ void k_export_list(const int *__restrict__ nbr, const int *__restrict__ ncount, int64_t stride,
                              int list_depth, int n, int32_t *counts, int32_t *partners, int partners_depth,
                              unsigned long long *total)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    int c = ncount[b];
    c = c < 0 ? 0 : (c > list_depth ? list_depth : c);
    if (counts) counts[b] = c;
    if (partners)
        for (int k = 0; k < c; k++) partners[(size_t)b * partners_depth + k] = nbr[(size_t)k * stride + b];
    atomicAdd(total, (unsigned long long)c);
}

cudaError_t launch_export_list(const int *nbr, const int *ncount, int64_t stride, int list_depth, int n,
                               int32_t *counts, int32_t *partners, int partners_depth, unsigned long long *total,
                               cudaStream_t st)
{
    k_export_list<<<(n + 255) / 256, 256, 0, st>>>(nbr, ncount, stride, list_depth, n, counts, partners,
                                                   partners_depth, total);
    return cudaGetLastError();
}

}  // namespace gcr
