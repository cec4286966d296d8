// gcr_observables.cu -- the reference's analysis observables on the device.
//
// Chain frames (analysis.chain_COM, analysis.py:288-292; the mean chain angle
// output_methods.calc_avg_phi_chain, output_methods.py:492-510) and the pair
// correlations over chain centres (analysis.correlation_func with g_of_r,
// Cvv, Cnn, analysis.py:203-275), for the resident systems of a context.
// The reference computes them in Python loops, O(n_chains^2) for the
// correlations; here one thread per chain and one per chain pair.
//
// Determinism: g(r) counts are integers; the Cvv / Cnn sums are accumulated
// in 64-bit fixed point (2^-32 resolution per pair), so the histograms do not
// depend on the order of the atomic additions.  Separations use explicitly
// rounded products and sums, as numpy evaluates them.
#include "gcr_device.cuh"
#include "gcr_kernels.h"

namespace gcr {

// analysis.true_sep (analysis.py:185-187): np.mod(pt2 - pt1 + L/2, L) - L/2
__device__ __forceinline__ double true_sep(double pt1, double pt2, double L)
{
    return __dsub_rn(py_mod(__dadd_rn(__dsub_rn(pt2, pt1), 0.5 * L), L), 0.5 * L);
}

// one thread per chain: the reference's chain "centre" (head + sum of the
// separations head - x_i, wrapped: analysis.chain_COM as written) and the
// mean angle of the tangents with 1- and 2-fold symmetry
template <int D, typename FT>
__global__ void k_chain_frame(const double *__restrict__ pos, const FT *__restrict__ tan,
                              const int32_t *__restrict__ cs, int n_chains, double L, double *com, double *phi)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chains) return;
    const int b0 = cs[c], b1 = cs[c + 1];
    if (com) {
        double head[D], acc[D];
#pragma unroll
        for (int i = 0; i < D; i++) {
            head[i] = pos[(size_t)b0 * D + i];
            acc[i] = 0.0;
        }
        for (int b = b0; b < b1; b++)
#pragma unroll
            for (int i = 0; i < D; i++) acc[i] = __dadd_rn(acc[i], true_sep(pos[(size_t)b * D + i], head[i], L));
#pragma unroll
        for (int i = 0; i < D; i++) com[(size_t)c * D + i] = py_mod(__dadd_rn(head[i], acc[i]), L);
    }
    if (phi) {
        double sx = 0.0, sy = 0.0, s2 = 0.0, c2 = 0.0;
        for (int b = b0; b < b1; b++) {
            const double tx = (double)tan[(size_t)b * D], ty = (double)tan[(size_t)b * D + 1];
            sx = __dadd_rn(sx, tx);
            sy = __dadd_rn(sy, ty);
            const double a = atan2(ty, tx);
            double sn, cn;
            sincos(2.0 * a, &sn, &cn);
            s2 = __dadd_rn(s2, sn);
            c2 = __dadd_rn(c2, cn);
        }
        phi[(size_t)c * 2] = atan2(sy, sx);
        phi[(size_t)c * 2 + 1] = atan2(s2, c2) / 2.0;
    }
}

constexpr double kFix = 4294967296.0;  // 2^32: fixed-point scale of the pair sums

// one thread per chain pair (ci > cj), histograms in shared memory
__global__ void k_pair_corr(const double *__restrict__ com, const double *__restrict__ phi, int n_chains, double L,
                            double binsize, int n_bins, int kind, unsigned long long *counts,
                            unsigned long long *sums)
{
    extern __shared__ unsigned long long sh_hist[];  // [n_bins] counts, [n_bins] fixed-point sums
    unsigned long long *hc = sh_hist, *hs = sh_hist + n_bins;
    for (int i = threadIdx.x; i < 2 * n_bins; i += blockDim.x) sh_hist[i] = 0ull;
    __syncthreads();
    const long long n_pairs = (long long)n_chains * (n_chains - 1) / 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n_pairs; p += stride) {
        // pair p -> (i, j), j < i, rows of the lower triangle in order
        long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
        while (i * (i - 1) / 2 > p) i--;
        while ((i + 1) * i / 2 <= p) i++;
        const long long j = p - i * (i - 1) / 2;
        const double s0 = true_sep(com[i * 2], com[j * 2], L);
        const double s1 = true_sep(com[i * 2 + 1], com[j * 2 + 1], L);
        const double dist = sqrt(__dadd_rn(__dmul_rn(s0, s0), __dmul_rn(s1, s1)));
        const long long bin = (long long)__ddiv_rn(dist, binsize);
        if (bin < 0 || bin >= n_bins) continue;  // past the last bin of the reference's range
        atomicAdd(hc + bin, 2ull);
        if (kind != 0) {
            const int k = kind == 1 ? 0 : 1;
            const double a = phi[i * 2 + k], b = phi[j * 2 + k];
            double f = __dadd_rn(__dmul_rn(cos(a), cos(b)), __dmul_rn(sin(a), sin(b)));
            if (kind == 2) f = fabs(f);
            const long long fx = __double2ll_rn(2.0 * f * kFix);
            atomicAdd(hs + bin, (unsigned long long)fx);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_bins; i += blockDim.x) {
        if (hc[i]) atomicAdd(counts + i, hc[i]);
        if (hs[i]) atomicAdd(sums + i, hs[i]);
    }
}

cudaError_t launch_chain_frames(int dim, int precision, const SysP &p, const int32_t *chain_start, double *com,
                                double *phi, cudaStream_t st)
{
    const unsigned g = (unsigned)((p.n_chains + 127) / 128);
    if (dim == 2) {
        if (precision == 0)
            k_chain_frame<2, double><<<g, 128, 0, st>>>(p.pos, (const double *)p.tan, chain_start, p.n_chains, p.L,
                                                        com, phi);
        else
            k_chain_frame<2, float><<<g, 128, 0, st>>>(p.pos, (const float *)p.tan, chain_start, p.n_chains, p.L,
                                                       com, phi);
    } else {
        if (precision == 0)
            k_chain_frame<3, double><<<g, 128, 0, st>>>(p.pos, (const double *)p.tan, chain_start, p.n_chains, p.L,
                                                        com, phi);
        else
            k_chain_frame<3, float><<<g, 128, 0, st>>>(p.pos, (const float *)p.tan, chain_start, p.n_chains, p.L,
                                                       com, phi);
    }
    return cudaGetLastError();
}

cudaError_t launch_pair_corr(const double *com, const double *phi, int n_chains, double L, double binsize, int n_bins,
                             int kind, unsigned long long *counts, unsigned long long *sums, int sm_count,
                             cudaStream_t st)
{
    const size_t smem = (size_t)n_bins * 2 * sizeof(unsigned long long);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_pair_corr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const long long n_pairs = (long long)n_chains * (n_chains - 1) / 2;
    long long blocks = (n_pairs + 255) / 256;
    blocks = blocks < 1 ? 1 : (blocks > 4LL * sm_count ? 4LL * sm_count : blocks);
    k_pair_corr<<<(unsigned)blocks, 256, smem, st>>>(com, phi, n_chains, L, binsize, n_bins, kind, counts, sums);
    return cudaGetLastError();
}

}  // namespace gcr
