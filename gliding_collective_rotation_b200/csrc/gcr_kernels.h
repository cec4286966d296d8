// gcr_kernels.h -- kernel arguments and entry points shared by the host
// library (gcr_abi.cu) and the kernel translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gcr_device.cuh"

namespace gcr {

// Everything a step kernel reads: device pointers of one context.
struct BatchArgs {
    const SysP *P;
    SysS *S;
    const Tile *bead_tiles;
    const int *n_bead_tiles;
    const Tile *cell_tiles;
    const int *n_cell_tiles;
    const uint8_t *topo;
    int *cnt0;
    int *cnt1;
    int *items;
    void *rec;
    void *xi;      // translational noise of the current step per bead, FT [bead][dim]
    void *fp;      // pair force per bead (bead order), FT [bead][dim]
    int *cstart;   // start of each cell in the compact list (+ end sentinel per system)
    int *rcell;    // cell of each compact-list record
    int *tsum;     // cell count of each cell tile
    int *toff;     // start of each cell tile within its system
    int depth;
    int log_depth;
    int tile_beads;
    int tile_cells;
};

struct KernelSet {
    void *insert;
    void *pack0;
    void *pack1;
    void *stage0;
    void *stage1;
    void *update;
    void *topo;
    void *sys_dt;
    void *sys_end;
    void *pair;
    void *scan_local0;
    void *scan_local1;
    void *scan_tiles;
    size_t (*stage_smem)(int block_beads);  // dynamic shared memory of the stage kernels
};

KernelSet kernel_set(int dim, int precision);

// message returned by gcr_last_error() on the calling thread (gcr_abi.cu)
void set_last_error(const char *msg);

// gcr_lists.cu
cudaError_t launch_reference_lists(int dim, const SysP &p, int64_t n_grid, int64_t grid_window,
                                   int64_t *where_is_bead, int64_t *grid_list, int64_t grid_depth1,
                                   int64_t *nbor_list, int64_t nbor_depth1, int *d_err, cudaStream_t st);
cudaError_t launch_order_params(int dim, int precision, const SysP &p, const int32_t *chain_start,
                                double *d_out, cudaStream_t st);
cudaError_t launch_chain_starts(const int32_t *chain, int n, int n_chains, int32_t *chain_start, int *d_err,
                                cudaStream_t st);
cudaError_t launch_cell_assignment(int dim, const SysP &p, int32_t *cell_of_bead, cudaStream_t st);
cudaError_t launch_philox_noise(int dim, uint64_t seed, int64_t step, int64_t n, int do_trans,
                                int do_rot, double *out, cudaStream_t st);

}  // namespace gcr
