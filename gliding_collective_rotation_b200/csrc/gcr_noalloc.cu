// gcr_noalloc.cu -- the order parameters of one system without any device
// allocation.
//
// gcr_order_params_noalloc computes what gcr_order_params computes (the
// per-chain angle and the polar / nematic order parameters), but for caller
// owned device arrays and without a context, so it never calls cudaMalloc or
// cudaFree.  It is meant for callers that cannot allocate device memory: an
// analysis hook that samples a system while other work is queued on the
// device (cudaFree waits for the whole device, stalling that work), or a host
// application that hands out all device memory from its own pool under a
// fixed budget and leaves none to a library.  The call waits for its own
// stream before it returns, with the results on the host.
//
// Its scratch (chain start offsets, the three results and two error words)
// lives in the file-scope array below, sized for at most
// GCR_NOALLOC_MAX_CHAINS chains: about 1 MiB that every GPU which loads
// the library holds until the process exits.  In host code the array's name
// only stands for the device object; its device address is looked up with
// cudaGetSymbolAddress once per device, with that device current, by the
// first call made on that device, and kept for the life of the process (a
// cudaDeviceReset after that first call leaves the kept address stale and is
// not supported).  All calls share the one array and it keeps the last
// call's contents: each call clears the words that must start at zero, and
// calls that overlap on the GPU (different streams, or different host
// threads on one device) race on it.
#include <cstring>
#include <mutex>

#include "../../include/gcr.h"
#include "gcr_device.cuh"
#include "gcr_kernels.h"

namespace {

constexpr int64_t kMaxChains = GCR_NOALLOC_MAX_CHAINS;
constexpr size_t kStartsBytes = sizeof(int32_t) * (size_t)(kMaxChains + 1);
constexpr size_t kOutOff = (kStartsBytes + 255) / 256 * 256;
constexpr size_t kErrOff = kOutOff + 4 * sizeof(double);
constexpr size_t kScratchBytes = kErrOff + 256;

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[kMaxDevices] = {nullptr};

// failures report through gcr_last_error(), like every other entry point
int noalloc_fail(int code, const char *msg)
{
    gcr::set_last_error(msg);
    return code;
}

}  // namespace

// the scratch of gcr_order_params_noalloc (see the file comment)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

// device address of the scratch on the current device (set-up once per device)
int scratch_on_current_device(unsigned char **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(GCR_ERR_CUDA, "no current CUDA device");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return noalloc_fail(GCR_ERR_CUDA, "cudaGetSymbolAddress of the no-allocation scratch failed");
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[dev];
    return GCR_OK;
}

}  // namespace

extern "C" {

int gcr_order_params_noalloc(int32_t dim, int32_t precision, const void *tangent, const int32_t *chain_id,
                             int64_t n_beads, int64_t n_chains, double out[3], void *cuda_stream)
{
    if (dim != 2) return noalloc_fail(GCR_ERR_BAD_ARG, "order parameters are defined for 2D systems");
    if (precision != GCR_FP64 && precision != GCR_MIXED) return noalloc_fail(GCR_ERR_BAD_ARG, "bad precision");
    if (!tangent || !chain_id || !out) return noalloc_fail(GCR_ERR_BAD_ARG, "null pointer");
    if (n_beads <= 0 || n_beads > (int64_t)1 << 30) return noalloc_fail(GCR_ERR_BAD_ARG, "n_beads out of range");
    if (n_chains <= 0 || n_chains > n_beads) return noalloc_fail(GCR_ERR_BAD_ARG, "n_chains out of range");
    if (n_chains > kMaxChains)
        return noalloc_fail(GCR_ERR_CAPACITY, "more chains than GCR_NOALLOC_MAX_CHAINS (262144)");
    unsigned char *base = nullptr;
    int rc = scratch_on_current_device(&base);
    if (rc) return rc;
    int32_t *starts = reinterpret_cast<int32_t *>(base);
    double *d_out = reinterpret_cast<double *>(base + kOutOff);
    int *d_err = reinterpret_cast<int *>(base + kErrOff);
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    const int n = (int)n_beads, nch = (int)n_chains;
    // the error words (bad chain ids, longest chain) and the results start at
    // zero; launch_chain_starts checks the chain ids (first bead in chain 0,
    // steps of 0 or 1, last bead in chain n_chains-1) and, when they pass,
    // has written every start offset of this call
    if (cudaMemsetAsync(d_err, 0, 2 * sizeof(int), st) != cudaSuccess ||
        cudaMemsetAsync(d_out, 0, 4 * sizeof(double), st) != cudaSuccess)
        return noalloc_fail(GCR_ERR_CUDA, "clearing the scratch failed");
    if (gcr::launch_chain_starts(chain_id, n, nch, starts, d_err, st) != cudaSuccess)
        return noalloc_fail(GCR_ERR_CUDA, "chain start kernel failed to launch");
    int err = 0;
    if (cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return noalloc_fail(GCR_ERR_CUDA, "chain id check failed");
    if (err)
        return noalloc_fail(GCR_ERR_BAD_ARG, "chain ids must run 0..n_chains-1 in contiguous, increasing ranges");
    gcr::SysP p;
    std::memset(&p, 0, sizeof(p));
    p.tan = const_cast<void *>(tangent);
    p.n = n;
    p.n_chains = nch;
    if (gcr::launch_order_params(dim, precision, p, starts, d_out, st) != cudaSuccess)
        return noalloc_fail(GCR_ERR_CUDA, "order parameter kernel failed to launch");
    if (cudaMemcpyAsync(out, d_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return noalloc_fail(GCR_ERR_CUDA, "order parameter kernel failed");
    return GCR_OK;
}

}  // extern "C"
