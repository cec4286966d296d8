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
    int *cnt;      // beads binned per cell (the sort reads and zeroes it)
    int *ncell;    // beads per cell at the last list build
    int *items;    // bead ids per cell, `depth` slots per cell
    int *nbr;      // neighbour list: slot k of bead g at nbr[k * list_stride + g]
    int *ncount;   // neighbours per bead
    double *xref;  // positions at the last list build, FP64 [bead][dim]
    void *xi;      // translational noise of the current step per bead, FT [bead][dim]
    void *fp;      // pair force per bead (bead order), FT [bead][dim]
    int *work;     // flagged systems of the coming list build (k_lists_plan)
    int n_slots;
    int64_t list_stride;
    int list_depth;
    int depth;
    int log_depth;
    int tile_beads;
    int tile_cells;
    int order;     // SRK order of the context: 2 or 4
    // cross lists of coupled populations: slot k of row r at xnbr[k * xstride + r]
    // (row r = x_off + c * n + bead for cross partner c), xcount[r] partners
    int *xnbr;
    int *xcount;
    int64_t xstride;
    // periodic images crossed by each bead since admission, int32 [bead][dim]
    // (the real updates count them; unwrapped = pos + L * img)
    int *img;
    // row tiles of the cell-staged pair kernel: slot k owns tiles
    // row_prefix[k] .. row_prefix[k+1]-1 (row_prefix[n_slots] = all tiles);
    // tile r of a system is segment r % segments of row r / segments
    const int *row_prefix;
    int cell_stage_cap;  // beads a CTA of the cell-staged pair kernel copies into shared memory
    // motors (allocated with the first motor population): where_active of every
    // bead (chains: motors attached, -1 + count; motors: the bead it pushes or
    // -1), and per chain bead the pushes and the where_active change of the
    // current stage (written by k_motor, consumed and zeroed by k_stage)
    int *act;
    int *mpush;
    int *mdelta;
    // rest length of each bead's chain, FP64 [bead]: rest_lengths[chain_id],
    // written for every armed system at each run start (the host may change
    // rest lengths between calls), so that the stage kernels stage it with
    // one load instead of the chain-id load and the dependent gather
    double *restb;
};

struct KernelSet {
    void *bin0;     // cell binning of pos / pos1 for a list build
    void *bin1;
    void *sort;     // per-cell sort of the binned ids (zeroes the counts)
    void *build0;   // neighbour lists from pos / pos1
    void *build1;
    void *pair0;    // pair forces at pos / pos1
    void *pair1;
    void *stage0;
    void *stage1;
    void *stage0f;  // stages 0 and 1 that sum the pair forces themselves (no k_pair launch)
    void *stage1f;
    void *update;
    void *rigid0;   // rigid-rod projection: predictor (pos -> pos1) and corrector (pos1 -> pos)
    void *rigid1;
    // SRK4: lists and pair forces at pos2, the four stages, their projections
    void *bin2;
    void *build2;
    void *pair2;
    void *stage4[4];
    void *rigid4[4];
    void *topo;
    void *sys_dt;
    void *sys_end;
    void *sys_mark;  // flag one resident system (or all) for a list build
    void *run_check;  // run start: flag the armed systems whose lists no longer cover their positions
    void *lists_plan;  // compact the systems that take part in a list build
    void *pair_cross[3];  // pair forces at pos / pos1 / pos2 with the other populations' (coupled systems)
    void *pair_cells[2];  // cell-staged pair forces at pos / pos1 (pair_mode 2)
    void *motor[2];       // motor decisions of stage 0 / 1 (graphs with a motor population)
    size_t (*pair_cells_smem)(int cap);  // their dynamic shared memory for `cap` staged beads
    int pair_cells_rows;  // cell rows a row tile stages (3 in 2D, 9 in 3D)
    int max_row_cells;    // cells of a row tile, at most
    size_t (*stage_smem)(int block_beads);  // dynamic shared memory of the stage kernels
    size_t (*pair_smem)(int block_beads);   // dynamic shared memory of the pair kernels
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
// k_observe<FT>(BatchArgs, int dim): the in-graph order-parameter series, one 1024-thread CTA per slot
void *observe_kernel(int precision);
// chain_start[n_chains + 1]; d_err[0] |= 4 on bad chain ids, d_err[1] = longest chain
cudaError_t launch_chain_starts(const int32_t *chain, int n, int n_chains, int32_t *chain_start, int *d_err,
                                cudaStream_t st);
cudaError_t launch_cell_assignment(int dim, const SysP &p, int32_t *cell_of_bead, cudaStream_t st);
cudaError_t launch_export_list(const int *nbr, const int *ncount, int64_t stride, int list_depth, int n,
                               int32_t *counts, int32_t *partners, int partners_depth, unsigned long long *total,
                               cudaStream_t st);
// gcr_observables.cu
cudaError_t launch_chain_frames(int dim, int precision, const SysP &p, const int32_t *chain_start, double *com,
                                double *phi, cudaStream_t st);
cudaError_t launch_pair_corr(const double *com, const double *phi, int n_chains, double L, double binsize, int n_bins,
                             int kind, unsigned long long *counts, unsigned long long *sums, int sm_count,
                             cudaStream_t st);
// out[n][dim] = pos + L * img (unwrapped positions of one system)
cudaError_t launch_unwrap(int dim, const double *pos, const int *img, int n, double L, double *out, cudaStream_t st);
cudaError_t launch_philox_noise(int dim, uint64_t seed, int64_t step, int64_t n, int do_trans,
                                int do_rot, double *out, cudaStream_t st);

}  // namespace gcr
