// gcr_abi.cu -- the C ABI of libgcr.so (declared in include/gcr.h).
//
// A context owns the scratch of many resident systems and one CUDA graph of
// `steps_per_graph` SRK2 steps.  The graph's kernels are persistent and read
// the system descriptors and tile tables from device memory, so admitting or
// evicting a system (continuous batching) never re-captures the graph.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/gcr.h"
#include "gcr_device.cuh"
#include "gcr_kernels.h"

using namespace gcr;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define GCR_CUDA(call)                                                                             \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(e_ == cudaErrorMemoryAllocation ? GCR_ERR_OOM : GCR_ERR_CUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

// first-fit allocator of integer ranges [0, capacity)
struct RangeAlloc {
    int64_t capacity = 0;
    std::map<int64_t, int64_t> free_;  // offset -> length
    void init(int64_t cap)
    {
        capacity = cap;
        free_.clear();
        if (cap > 0) free_[0] = cap;
    }
    int64_t alloc(int64_t n)
    {
        if (n <= 0) return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                int64_t off = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[off + n] = len - n;
                return off;
            }
        }
        return -1;
    }
    void release(int64_t off, int64_t n)
    {
        if (n <= 0) return;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Slot {
    bool used = false;
    gcr_system_desc desc{};
    gcr_system_buffers buf{};
    int64_t bead_off = 0, cell_off = 0, chain_off = 0;
    int64_t n_cells = 0;        // cells of the current grid
    int64_t n_cells_alloc = 0;  // cells reserved at admission
    int64_t nc = 1;             // current GPU cells per side
    int64_t longest = 0;        // beads of the longest chain
    int group = -1;             // coupled group (index into gcr_ctx::groups) or -1
    // a motor population (gcr_set_motors): the chains it pushes and how
    int motor_chain = -1;
    double mparams[5] = {0, 0, 0, 0, 0};
    int motor_hold = 1;
};

// populations coupled in one box (gcr_couple)
struct Group {
    int n = 0;  // 0: dissolved
    int32_t slots[kMaxPops] = {-1, -1, -1, -1};
    int32_t fixed[kMaxPops] = {0, 0, 0, 0};
    double cross[kMaxPops][kMaxPops][4] = {};  // [i][j]: force on member i from member j
};

int ilog2(int v)
{
    int l = 0;
    while ((1 << l) < v) l++;
    return l;
}

}  // namespace

namespace gcr {
void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }
}  // namespace gcr

struct gcr_ctx {
    gcr_config cfg{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    int sm_count = 0;
    KernelSet ks{};
    // device arrays
    SysP *dP = nullptr;
    SysS *dS = nullptr;
    Tile *d_bead_tiles = nullptr;
    Tile *d_cell_tiles = nullptr;
    int *d_row_prefix = nullptr;  // row tiles of the cell-staged pair kernel per slot, prefix [S + 1]
    int *d_ntiles = nullptr;  // [0] bead tiles, [1] cell tiles
    uint8_t *topo = nullptr;
    int *cnt = nullptr;
    int *ncell = nullptr;
    int *items = nullptr;
    int *nbr = nullptr;
    int *ncount = nullptr;
    double *xref = nullptr;
    int *img = nullptr;  // periodic images crossed per bead and axis since admission
    double *restb = nullptr;  // rest length of each bead's chain (refreshed at every run start)
    int *work = nullptr;
    void *xi = nullptr;
    void *fp = nullptr;
    double *pos2 = nullptr;  // SRK4 scratch: second virtual update
    void *faux = nullptr;    // SRK4 scratch: stage forces of systems without a caller buffer
    size_t stage_smem = 0;
    size_t pair_cells_smem = 0;
    size_t pair_smem = 0;
    int32_t *chain_starts = nullptr;
    int *d_err = nullptr;
    double *d_out = nullptr;
    int64_t max_bead_tiles = 0, max_cell_tiles = 0;
    // host mirrors
    std::vector<Slot> slots;
    std::vector<SysP> hP;
    std::vector<SysS> hS;
    std::vector<Tile> h_bead_tiles, h_cell_tiles;
    std::vector<int> h_row_prefix;
    RangeAlloc beads, cells, chains;
    BatchArgs args{};
    int grid_update = 1, grid_sys = 1, grid_pair = 1, grid_bin = 1, grid_sort = 1, grid_build = 1;
    int grid_stage0 = 1, grid_stage1 = 1, grid_stage4[4] = {1, 1, 1, 1};
    int grid_stage0f = 1, grid_stage1f = 1, grid_pair_cells = 1;
    cudaGraphExec_t graph = nullptr;
    bool graph_rigid = false;  // the graph holds the rigid-rod projection kernels
    bool graph_obs = false;    // the graph holds the series kernel
    bool graph_cross = false;  // the graph holds the cross-population pair kernels
    bool graph_motor = false;  // the graph holds the motor kernels
    int *act = nullptr;        // motors: where_active per bead, pushes and changes per stage (lazy)
    int *mpush = nullptr;
    int *mdelta = nullptr;
    std::vector<Group> groups;
    int *xnbr = nullptr;       // cross lists of coupled populations
    int *xcount = nullptr;
    int64_t x_rows = 0;        // rows allocated (the slot stride of xnbr)
    void *observe = nullptr;   // k_observe of the context's precision
    bool pdl = true;           // programmatic dependent launch of the step kernels
    bool tiles_dirty = true;
};

namespace {

int kernel_grid(const gcr_ctx *c, void *fn, int block, int64_t max_tiles, size_t smem = 0)
{
    // ctas_per_sm < 0: one CTA per tile (the hardware scheduler streams the
    // tiles; CTAs past the live tile count exit at once)
    if (c->cfg.ctas_per_sm < 0) return (int)std::max<int64_t>(max_tiles, 1);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, smem) != cudaSuccess || occ < 1) occ = 1;
    if (c->cfg.ctas_per_sm > 0) occ = std::min(occ, c->cfg.ctas_per_sm);
    int64_t g = (int64_t)c->sm_count * occ;
    g = std::min<int64_t>(g, std::max<int64_t>(max_tiles, 1));
    return (int)std::max<int64_t>(g, 1);
}

int rebuild_tiles(gcr_ctx *c)
{
    c->h_bead_tiles.clear();
    c->h_cell_tiles.clear();
    c->h_row_prefix.assign(c->slots.size() + 1, 0);
    int64_t rows = 0;
    const int tb = c->cfg.block_beads, tcl = c->cfg.block_cells;
    for (int s = 0; s < (int)c->slots.size(); s++) {
        const Slot &sl = c->slots[s];
        if (!sl.used) continue;
        // a fixed population never moves: only the list kernels visit it
        if (!c->hP[s].fixed)
            for (int64_t b = 0; b < sl.desc.n_beads; b += tb) c->h_bead_tiles.push_back(Tile{s, (int32_t)b});
        if (sl.desc.calc_wca)
            for (int64_t q = 0; q < sl.n_cells; q += tcl) c->h_cell_tiles.push_back(Tile{s, (int32_t)q});
    }
    for (int s = 0; s < (int)c->slots.size(); s++) {
        c->h_row_prefix[s] = (int)rows;
        if (c->slots[s].used) rows += c->hP[s].n_row_tiles;
    }
    if (rows > INT32_MAX / 2) return fail(GCR_ERR_CAPACITY, "too many row tiles");
    c->h_row_prefix[c->slots.size()] = (int)rows;
    GCR_CUDA(cudaMemcpyAsync(c->dP, c->hP.data(), sizeof(SysP) * c->hP.size(), cudaMemcpyHostToDevice,
                             c->stream));
    if ((int64_t)c->h_bead_tiles.size() > c->max_bead_tiles || (int64_t)c->h_cell_tiles.size() > c->max_cell_tiles)
        return fail(GCR_ERR_CAPACITY, "tile table capacity exceeded");
    int nt[2] = {(int)c->h_bead_tiles.size(), (int)c->h_cell_tiles.size()};
    if (nt[0]) GCR_CUDA(cudaMemcpyAsync(c->d_bead_tiles, c->h_bead_tiles.data(), nt[0] * sizeof(Tile),
                                        cudaMemcpyHostToDevice, c->stream));
    if (nt[1]) GCR_CUDA(cudaMemcpyAsync(c->d_cell_tiles, c->h_cell_tiles.data(), nt[1] * sizeof(Tile),
                                        cudaMemcpyHostToDevice, c->stream));
    GCR_CUDA(cudaMemcpyAsync(c->d_row_prefix, c->h_row_prefix.data(), c->h_row_prefix.size() * sizeof(int),
                             cudaMemcpyHostToDevice, c->stream));
    GCR_CUDA(cudaMemcpyAsync(c->d_ntiles, nt, sizeof(nt), cudaMemcpyHostToDevice, c->stream));
    // the host arrays must outlive the asynchronous copies
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    c->tiles_dirty = false;
    return GCR_OK;
}

// checks a descriptor; derives the GPU cell grid (cells of side >= (r_cut +
// skin) * cell_factor, at least 3 per side) and the skin actually used
int validate_desc(const gcr_config &cfg, const gcr_system_desc *d, int64_t *nc_out, double *skin_out = nullptr)
{
    if (!d) return fail(GCR_ERR_BAD_ARG, "null descriptor");
    if (d->n_beads <= 0 || d->n_beads > (int64_t)INT32_MAX / 2) return fail(GCR_ERR_BAD_ARG, "n_beads out of range");
    if (d->n_chains <= 0 || d->n_chains > d->n_beads) return fail(GCR_ERR_BAD_ARG, "n_chains out of range");
    if (!(d->L > 0.0) || !std::isfinite(d->L)) return fail(GCR_ERR_BAD_ARG, "box side L must be positive");
    if (!(d->radius > 0.0)) return fail(GCR_ERR_BAD_ARG, "radius must be positive");
    if (d->spring_params[3] != 0.0) return fail(GCR_ERR_BAD_ARG, "FENE springs are not supported");
    if (d->active_params[1] > 0.0) return fail(GCR_ERR_BAD_ARG, "active sliding is not supported");
    if (!(d->skin >= 0.0) || !std::isfinite(d->skin)) return fail(GCR_ERR_BAD_ARG, "skin must be >= 0");
    if (!std::isfinite(d->rigid_rod)) return fail(GCR_ERR_BAD_ARG, "rigid_rod must be finite");
    int64_t nc = 1;
    double skin = d->skin;
    if (d->calc_wca) {
        double rc = d->wca_params[3];
        double cf = d->cell_factor >= 1.0 ? d->cell_factor : 1.0;
        if (!(rc > 0.0)) return fail(GCR_ERR_BAD_ARG, "pair cutoff must be positive");
        if (d->L < 3.0 * rc * cf)
            return fail(GCR_ERR_BAD_ARG, "box side must be at least 3 pair cutoffs for the GPU cell grid");
        // a box too small for the skin keeps 3 cells per side with a smaller skin
        if ((rc + skin) * cf * 3.0 > d->L) skin = d->L / (3.0 * cf) - rc;
        skin = skin > 0.0 ? skin : 0.0;
        const double side = (rc + skin) * cf;
        nc = (int64_t)std::floor(d->L / side);
        nc = nc < 3 ? 3 : nc;
        // h = L/nc must not fall below the list radius through rounding
        while (nc > 3 && d->L / (double)nc < rc + skin) nc--;
        if (d->L / (double)nc < rc + skin) skin = d->L / (double)nc - rc;
        skin = skin > 0.0 ? skin : 0.0;
        int64_t cells = 1;
        for (int i = 0; i < cfg.dim; i++) cells *= nc;
        if (cells > (int64_t)INT32_MAX / 2) return fail(GCR_ERR_BAD_ARG, "too many GPU cells");
    }
    *nc_out = nc;
    if (skin_out) *skin_out = skin;
    return GCR_OK;
}

// row tiles of the cell-staged pair kernel: segments of T cells of each
// row of the GPU grid, T chosen so that a segment holds about one CTA's
// worth (block_beads) of beads at the system's mean cell occupancy
void row_tiling(const gcr_ctx *c, const gcr_system_desc &d, int64_t nc, SysP &p)
{
    p.row_cells = 0;
    p.n_row_tiles = 0;
    if (!d.calc_wca || p.fixed || nc < 3) return;
    int64_t cells = 1, rows = 1;
    for (int i = 0; i < c->cfg.dim; i++) cells *= nc;
    for (int i = 1; i < c->cfg.dim; i++) rows *= nc;
    const double per_cell = (double)d.n_beads / (double)cells;
    int64_t T = (int64_t)std::floor((double)c->cfg.block_beads / std::max(per_cell, 1e-3));
    T = std::max<int64_t>(1, std::min<int64_t>(T, c->ks.max_row_cells));
    p.row_cells = (int32_t)T;
    p.n_row_tiles = (int32_t)(rows * ((nc + T - 1) / T));
}

void fill_sysp(const gcr_ctx *c, const Slot &sl, int64_t nc, double skin, SysP &p)
{
    const gcr_system_desc &d = sl.desc;
    std::memset(&p, 0, sizeof(p));
    p.pos = sl.buf.pos;
    p.pos1 = sl.buf.pos1;
    p.tan = sl.buf.tangent;
    p.frc = sl.buf.forces;
    p.chain = sl.buf.chain_id;
    p.rest = sl.buf.rest_lengths;
    p.chain_start = c->chain_starts + sl.chain_off;
    const size_t ft = c->cfg.precision == GCR_FP64 ? 8 : 4;
    p.pos2 = c->pos2 ? c->pos2 + (size_t)sl.bead_off * c->cfg.dim : nullptr;
    p.faux = sl.buf.forces_aux ? sl.buf.forces_aux
                               : (c->faux ? (void *)((char *)c->faux + (size_t)sl.bead_off * c->cfg.dim * ft) : nullptr);
    p.bead_off = sl.bead_off;
    p.cell_off = sl.cell_off;
    p.n = (int32_t)d.n_beads;
    p.n_chains = (int32_t)d.n_chains;
    p.nc = (int32_t)nc;
    p.n_cells = (int32_t)sl.n_cells;
    p.n_bead_tiles = (int32_t)((d.n_beads + c->cfg.block_beads - 1) / c->cfg.block_beads);
    p.n_cell_tiles = (int32_t)((sl.n_cells + c->cfg.block_cells - 1) / c->cfg.block_cells);
    row_tiling(c, d, nc, p);
    p.L = d.L;
    p.half_L = d.L / 2.0;
    p.h = d.L / (double)nc;
    p.inv_h = (double)nc / d.L;
    p.k = d.spring_params[0];
    p.kappa = d.spring_params[1];
    p.theta0 = d.spring_params[2];
    p.calc_springs = d.calc_springs ? 1 : 0;
    p.get_orient = (d.calc_springs && d.spring_params[4] != 0.0) ? 1 : 0;
    p.calc_bend = (d.calc_springs && d.spring_params[1] != 0.0) ? 1 : 0;
    p.calc_wca = d.calc_wca ? 1 : 0;
    p.p0 = d.wca_params[0];
    p.p1 = d.wca_params[1];
    p.shift = d.wca_params[2];
    p.rc2 = d.wca_params[3] * d.wca_params[3];
    // list radius with a relative margin of 1e-6 in r^2, above the rounding of
    // the FP32 pair test, so that every pair that test accepts is listed
    p.rl2 = (d.wca_params[3] + skin) * (d.wca_params[3] + skin) * (1.0 + 1e-6);
    p.half_skin2 = 0.25 * skin * skin;
    p.n_nearby = d.n_nearby;
    p.self_propel = d.self_propel ? 1 : 0;
    p.v0 = d.active_params[0];
    double ang = d.active_params[2];
    p.rotate_prop = (ang != 0.0 && c->cfg.dim == 2) ? 1 : 0;
    p.cos_a = std::cos(ang);
    p.sin_a = std::sin(ang);
    p.D = d.D;
    p.Dr = d.Dr;
    p.radius = d.radius;
    p.sqrt2D = std::sqrt(2.0 * d.D);
    p.dtmax = d.dtmax;
    p.mdps = d.max_dist_per_step;
    p.rk = d.rk_cheat;
    // SRK.py:364: the projection acts only when some chain has more than 2 beads
    p.rigid = (d.rigid_rod != 0.0 && sl.longest > 2) ? d.rigid_rod : 0.0;
    p.seed = d.seed;
}

// the coupling fields of every resident system from the context's groups,
// and the cross-list rows they need; *moved: the cross-list buffer was
// reallocated (graphs captured with the old one must go)
int apply_groups(gcr_ctx *c, bool *moved)
{
    *moved = false;
    const int dim = c->cfg.dim;
    for (size_t s = 0; s < c->slots.size(); s++) {
        const Slot &sl = c->slots[s];
        if (!sl.used) continue;
        SysP &p = c->hP[s];
        p.fixed = 0;
        p.grp_n = 0;
        p.n_cross = 0;
        p.x_off = 0;
        for (int k = 0; k < kMaxPops; k++) p.grp[k] = -1;
        for (int k = 0; k < kMaxPops - 1; k++) {
            p.cross_q[k] = -1;
            p.cross_w[k] = 1;
            p.cross_p0[k] = p.cross_p1[k] = p.cross_shift[k] = p.cross_rc2[k] = p.cross_rl2[k] = 0.0;
        }
        p.pos1 = sl.buf.pos1;
        p.pos2 = c->pos2 ? c->pos2 + (size_t)sl.bead_off * dim : nullptr;
        p.motor = 0;
        p.motor_k = -1;
        p.motor_hold = 0;
        p.pushed = 0;
        p.push_force = 0.0;
        for (int k = 0; k < 5; k++) p.mparams[k] = 0.0;
    }
    int64_t rows = 0;
    for (const Group &g : c->groups) {
        for (int a = 0; a < g.n; a++) {
            SysP &p = c->hP[g.slots[a]];
            p.grp_n = g.n;
            for (int k = 0; k < g.n; k++) p.grp[k] = g.slots[k];
            p.fixed = g.fixed[a] ? 1 : 0;
            if (p.fixed) {
                // stage positions of a population that never moves
                p.pos1 = p.pos;
                p.pos2 = p.pos;
                continue;
            }
            const double skin_a = 2.0 * std::sqrt(p.half_skin2);
            // the other populations in the order their forces are added
            // (pop_index_diff = 1, 2, ..., SRK.py:287-294)
            // a motor population's cross list to the chains it pushes holds
            // its candidate beads (radius w[3]), not a force
            const Slot &sa = c->slots[g.slots[a]];
            for (int ii = 1; ii < g.n; ii++) {
                const int b = (a + ii) % g.n;
                const double *w = g.cross[a][b];
                const bool pushes = sa.motor_chain >= 0 && sa.motor_chain == g.slots[b] && !g.fixed[b];
                if (!(w[3] > 0.0) || (!pushes && w[0] == 0.0 && w[1] == 0.0)) continue;
                const SysP &q = c->hP[g.slots[b]];
                const int k = p.n_cross++;
                if (pushes) {
                    SysP &ch = c->hP[g.slots[b]];
                    p.motor = 1;
                    p.motor_k = k;
                    p.motor_hold = sa.motor_hold;
                    for (int e = 0; e < 5; e++) p.mparams[e] = sa.mparams[e];
                    ch.pushed = 1;
                    ch.push_force = sa.mparams[2];
                }
                p.cross_q[k] = g.slots[b];
                p.cross_p0[k] = w[0];
                p.cross_p1[k] = w[1];
                p.cross_shift[k] = w[2];
                p.cross_rc2[k] = w[3] * w[3];
                // both populations' beads stay within half their skins of the
                // build positions, so pairs within this radius cover r_cut
                const double rl = w[3] + 0.5 * (skin_a + 2.0 * std::sqrt(q.half_skin2));
                p.cross_rl2[k] = rl * rl * (1.0 + 1e-6);
                p.cross_w[k] = std::max(1, (int)std::ceil(rl * q.inv_h));
            }
            p.x_off = rows;
            rows += (int64_t)p.n_cross * p.n;
        }
    }
    if (rows > c->x_rows) {
        GCR_CUDA(cudaStreamSynchronize(c->stream));
        if (c->xnbr) cudaFree(c->xnbr);
        if (c->xcount) cudaFree(c->xcount);
        c->xnbr = nullptr;
        c->xcount = nullptr;
        c->x_rows = 0;
        cudaError_t e = cudaMalloc(&c->xnbr, sizeof(int) * (size_t)rows * (size_t)c->cfg.list_depth);
        if (e == cudaSuccess) e = cudaMalloc(&c->xcount, sizeof(int) * (size_t)rows);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->xcount, 0, sizeof(int) * (size_t)rows, c->stream);
        if (e != cudaSuccess) {
            if (c->xnbr) cudaFree(c->xnbr);
            if (c->xcount) cudaFree(c->xcount);
            c->xnbr = nullptr;
            c->xcount = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? GCR_ERR_OOM : GCR_ERR_CUDA, "cross-list allocation");
        }
        c->x_rows = rows;
        *moved = true;
    }
    c->args.xnbr = c->xnbr;
    c->args.xcount = c->xcount;
    c->args.xstride = c->x_rows;
    return GCR_OK;
}

// some resident system is a motor population pushing chains
bool any_motor(const gcr_ctx *c)
{
    for (size_t s = 0; s < c->slots.size(); s++)
        if (c->slots[s].used && c->hP[s].motor) return true;
    return false;
}

// some resident system feels another population's pair force
bool any_cross(const gcr_ctx *c)
{
    for (size_t s = 0; s < c->slots.size(); s++)
        if (c->slots[s].used && c->hP[s].n_cross > 0) return true;
    return false;
}

// drop the captured graph (the next gcr_run captures a new one)
int drop_graph(gcr_ctx *c)
{
    if (!c->graph) return GCR_OK;
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    return GCR_OK;
}

// dissolve group g: its members step on their own again
int dissolve(gcr_ctx *c, int g)
{
    if (g < 0 || g >= (int)c->groups.size()) return GCR_OK;
    Group &gr = c->groups[g];
    for (int k = 0; k < gr.n; k++)
        if (gr.slots[k] >= 0 && gr.slots[k] < (int)c->slots.size()) c->slots[gr.slots[k]].group = -1;
    gr = Group();
    return GCR_OK;
}

// some resident system uses the rigid-rod projection
bool any_rigid(const gcr_ctx *c)
{
    for (size_t s = 0; s < c->slots.size(); s++)
        if (c->slots[s].used && c->hP[s].rigid != 0.0) return true;
    return false;
}

// some resident system's call records a series (the host mirror of the
// state table is current after every gcr_call_begin)
bool any_series(const gcr_ctx *c)
{
    for (size_t s = 0; s < c->slots.size(); s++)
        if (c->slots[s].used && c->hS[s].series) return true;
    return false;
}

// a step kernel, with programmatic dependent launch: it may be scheduled
// while the previous kernel on the stream drains, and waits for it in its
// first statement (pdl_wait), so only the launch latency overlaps.  Off with
// GCR_PDL=0 in the environment.
int launch_args(gcr_ctx *c, void *fn, int grid, int block, size_t smem, void **a)
{
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(block);
    lc.dynamicSmemBytes = smem;
    lc.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = c->pdl ? 1 : 0;
    lc.attrs = at;
    lc.numAttrs = 1;
    GCR_CUDA(cudaLaunchKernelExC(&lc, fn, a));
    return GCR_OK;
}

int launch(gcr_ctx *c, void *fn, int grid, int block, size_t smem = 0)
{
    void *a[] = {&c->args};
    return launch_args(c, fn, grid, block, smem, a);
}

int launch_sys(gcr_ctx *c, void *fn)
{
    int n = (int)c->slots.size();
    void *a[] = {&c->args, &n};
    return launch_args(c, fn, c->grid_sys, 128, 0, a);
}

// one stage's neighbour lists (flagged systems only): plan, bin, per-cell
// sort, build
int enqueue_lists(gcr_ctx *c, int which)
{
    int rc;
    const int bb = c->cfg.block_beads, bc = c->cfg.block_cells;
    void *bin = which == 0 ? c->ks.bin0 : (which == 1 ? c->ks.bin1 : c->ks.bin2);
    void *build = which == 0 ? c->ks.build0 : (which == 1 ? c->ks.build1 : c->ks.build2);
    if ((rc = launch(c, c->ks.lists_plan, 1, 1024))) return rc;
    if ((rc = launch(c, bin, c->grid_bin, bb))) return rc;
    if ((rc = launch(c, c->ks.sort, c->grid_sort, bc))) return rc;
    return launch(c, build, c->grid_build, bb);
}

// the in-graph order-parameter series: one 1024-thread CTA per slot
int launch_observe(gcr_ctx *c)
{
    int dim = c->cfg.dim;
    void *a[] = {&c->args, &dim};
    return launch_args(c, c->observe, (int)c->slots.size(), 1024, 0, a);
}

// one SRK4 step (SRK.py:166-215): four force evaluations at pos, pos1, pos2,
// pos1, each with its lists; the virtual updates alternate pos1 / pos2
int enqueue_step4(gcr_ctx *c)
{
    int rc;
    const int bb = c->cfg.block_beads;
    static const int reads[4] = {0, 1, 2, 1};
    for (int k = 0; k < 4; k++) {
        if ((rc = enqueue_lists(c, reads[k]))) return rc;
        void *pair = c->graph_cross ? c->ks.pair_cross[reads[k]]
                                    : (reads[k] == 0 ? c->ks.pair0 : (reads[k] == 1 ? c->ks.pair1 : c->ks.pair2));
        if ((rc = launch(c, pair, c->grid_pair, bb, c->pair_smem))) return rc;
        if ((rc = launch(c, c->ks.stage4[k], c->grid_stage4[k], bb, c->stage_smem))) return rc;
        if (k < 3 && c->graph_rigid && (rc = launch(c, c->ks.rigid4[k], c->grid_update, bb))) return rc;
    }
    if ((rc = launch_sys(c, c->ks.sys_dt))) return rc;
    if ((rc = launch(c, c->ks.update, c->grid_update, bb))) return rc;
    if (c->graph_rigid && (rc = launch(c, c->ks.rigid4[3], c->grid_update, bb))) return rc;
    if ((rc = launch_sys(c, c->ks.sys_end))) return rc;
    return c->graph_obs ? launch_observe(c) : GCR_OK;
}

// pair_mode of an SRK2 graph: 1 and 2 only without coupled populations,
// whose cross forces only k_pair adds
int pair_mode(const gcr_ctx *c, bool cross) { return (c->cfg.srk_order == 2 && !cross) ? c->cfg.pair_mode : 0; }
bool fused_pair(const gcr_ctx *c, bool cross) { return pair_mode(c, cross) == 1; }

// SRK2 stage s (0 predictor, 1 corrector): the pair forces, then the stage
int enqueue_pair(gcr_ctx *c, int s, bool cross)
{
    const int mode = pair_mode(c, cross);
    if (mode == 1) return GCR_OK;
    if (mode == 2) return launch(c, c->ks.pair_cells[s], c->grid_pair_cells, c->cfg.block_beads, c->pair_cells_smem);
    void *pair = cross ? c->ks.pair_cross[s] : (s == 0 ? c->ks.pair0 : c->ks.pair1);
    return launch(c, pair, c->grid_pair, c->cfg.block_beads, c->pair_smem);
}

int enqueue_stage(gcr_ctx *c, int s, bool cross)
{
    const bool f = fused_pair(c, cross);
    void *stage = s == 0 ? (f ? c->ks.stage0f : c->ks.stage0) : (f ? c->ks.stage1f : c->ks.stage1);
    const int grid = s == 0 ? (f ? c->grid_stage0f : c->grid_stage0) : (f ? c->grid_stage1f : c->grid_stage1);
    return launch(c, stage, grid, c->cfg.block_beads, c->stage_smem);
}

int enqueue_step(gcr_ctx *c)
{
    int rc;
    const int bb = c->cfg.block_beads;
    if (c->cfg.srk_order == 4) return enqueue_step4(c);
    if ((rc = enqueue_lists(c, 0))) return rc;
    if ((rc = enqueue_pair(c, 0, c->graph_cross))) return rc;
    if (c->graph_motor && (rc = launch(c, c->ks.motor[0], c->grid_update, bb))) return rc;
    if ((rc = enqueue_stage(c, 0, c->graph_cross))) return rc;
    if (c->graph_rigid && (rc = launch(c, c->ks.rigid0, c->grid_update, bb))) return rc;
    if ((rc = enqueue_lists(c, 1))) return rc;
    if ((rc = enqueue_pair(c, 1, c->graph_cross))) return rc;
    if (c->graph_motor && (rc = launch(c, c->ks.motor[1], c->grid_update, bb))) return rc;
    if ((rc = enqueue_stage(c, 1, c->graph_cross))) return rc;
    if ((rc = launch_sys(c, c->ks.sys_dt))) return rc;
    if ((rc = launch(c, c->ks.update, c->grid_update, bb))) return rc;
    if (c->graph_rigid && (rc = launch(c, c->ks.rigid1, c->grid_update, bb))) return rc;
    if ((rc = launch_sys(c, c->ks.sys_end))) return rc;
    return c->graph_obs ? launch_observe(c) : GCR_OK;
}

// start of a run: flag the armed systems whose neighbour lists no longer
// cover their positions (the host may have moved beads between calls); the
// others keep their lists
int enqueue_run_start(gcr_ctx *c)
{
    return launch(c, c->ks.run_check, c->grid_update, c->cfg.block_beads);
}

// a list build of `slot` before its next pair forces, from zeroed cell
// counts: admission, a new descriptor (grid, cutoff, skin, exclusions), a
// coupling change, and re-arming after a stop (a build that overflowed its
// cells leaves their counts set)
int mark_rebuild(gcr_ctx *c, int slot)
{
    const Slot &sl = c->slots[slot];
    if (sl.n_cells_alloc > 0)
        GCR_CUDA(cudaMemsetAsync(c->cnt + sl.cell_off, 0, sizeof(int) * (size_t)sl.n_cells_alloc, c->stream));
    int n = (int)c->slots.size();
    void *a[] = {&c->args, &n, &slot};
    GCR_CUDA(cudaLaunchKernel(c->ks.sys_mark, dim3(c->grid_sys), dim3(128), a, 0, c->stream));
    return GCR_OK;
}

int build_graph(gcr_ctx *c)
{
    // the projection and series kernels are in the graph only while some
    // system uses them
    const bool rigid = any_rigid(c), obs = any_series(c), cross = any_cross(c), motor = any_motor(c);
    if (c->graph && (rigid != c->graph_rigid || obs != c->graph_obs || cross != c->graph_cross ||
                     motor != c->graph_motor)) {
        GCR_CUDA(cudaStreamSynchronize(c->stream));
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    if (c->graph) return GCR_OK;
    c->graph_rigid = rigid;
    c->graph_obs = obs;
    c->graph_cross = cross;
    c->graph_motor = motor;
    cudaGraph_t g = nullptr;
    GCR_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = GCR_OK;
    for (int s = 0; s < c->cfg.steps_per_graph && rc == GCR_OK; s++) rc = enqueue_step(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc != GCR_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(GCR_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(GCR_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return GCR_OK;
}

bool valid_slot(const gcr_ctx *c, int32_t slot)
{
    return c && slot >= 0 && slot < (int32_t)c->slots.size() && c->slots[slot].used;
}

}  // namespace

extern "C" {

const char *gcr_last_error(void) { return g_last_error.c_str(); }

int gcr_version(void) { return 1; }

int gcr_footprint(const gcr_config *cfg, const gcr_system_desc *desc, int64_t *cells_out, int64_t *bytes_out)
{
    if (!cfg) return fail(GCR_ERR_BAD_ARG, "null config");
    int64_t nc = 1;
    int rc = validate_desc(*cfg, desc, &nc);
    if (rc) return rc;
    int64_t cells = 0;
    if (desc->calc_wca) {
        cells = 1;
        for (int i = 0; i < cfg->dim; i++) cells *= nc;
    }
    const int64_t n = desc->n_beads, d = cfg->dim;
    const int64_t ft = cfg->precision == GCR_FP64 ? 8 : 4;
    const int64_t ld = cfg->list_depth > 0 ? cfg->list_depth : (cfg->dim == 2 ? 32 : 96);
    int64_t bytes = n * d * (8 + 8 + ft + ft) + n * 4 + desc->n_chains * 8     // caller-owned state
                    + n * (1 + 2 * d * ft + 8) + 4 * (desc->n_chains + 1)      // topo, fp, xi, rest, chain starts
                    + n * (4 * ld + 4 + 8 * d)                                 // neighbour list, xref
                    + cells * (8 + (int64_t)cfg->cell_depth * 4)               // counts, slots
                    + (cfg->srk_order == 4 ? n * d * (8 + ft) : 0);            // SRK4: pos2, stage forces
    if (cells_out) *cells_out = cells;
    if (bytes_out) *bytes_out = bytes;
    return GCR_OK;
}

int gcr_create(const gcr_config *cfg_in, void *cuda_stream, gcr_ctx **out)
{
    if (!cfg_in || !out) return fail(GCR_ERR_BAD_ARG, "null argument");
    gcr_config cfg = *cfg_in;
    if (cfg.dim != 2 && cfg.dim != 3) return fail(GCR_ERR_BAD_ARG, "dim must be 2 or 3");
    if (cfg.precision != GCR_FP64 && cfg.precision != GCR_MIXED) return fail(GCR_ERR_BAD_ARG, "bad precision");
    if (cfg.cell_depth != 8 && cfg.cell_depth != 16 && cfg.cell_depth != 32 && cfg.cell_depth != 64 &&
        cfg.cell_depth != 128)
        return fail(GCR_ERR_BAD_ARG, "cell_depth must be 8, 16, 32, 64 or 128");
    if (cfg.block_beads < 64 || cfg.block_beads > 512 || cfg.block_beads % 32)
        return fail(GCR_ERR_BAD_ARG, "block_beads must be a multiple of 32 in [64, 512]");
    if (cfg.block_cells < 64 || cfg.block_cells > 512 || cfg.block_cells % 32)
        return fail(GCR_ERR_BAD_ARG, "block_cells must be a multiple of 32 in [64, 512]");
    if (cfg.steps_per_graph < 1 || cfg.steps_per_graph > 64)
        return fail(GCR_ERR_BAD_ARG, "steps_per_graph must be in [1, 64]");
    if (cfg.bead_capacity <= 0 || cfg.system_capacity <= 0 || cfg.cell_capacity < 0)
        return fail(GCR_ERR_BAD_ARG, "capacities must be positive");
    if (cfg.list_depth == 0) cfg.list_depth = cfg.dim == 2 ? 32 : 96;
    if (cfg.list_depth < 4 || cfg.list_depth > 1024) return fail(GCR_ERR_BAD_ARG, "list_depth must be in [4, 1024]");
    if (cfg.srk_order == 0) cfg.srk_order = 2;
    if (cfg.pair_mode < 0 || cfg.pair_mode > 2) return fail(GCR_ERR_BAD_ARG, "pair_mode must be 0, 1 or 2");
    if (cfg.srk_order != 2 && cfg.srk_order != 4) return fail(GCR_ERR_BAD_ARG, "srk_order must be 2 or 4");

    gcr_ctx *c = new (std::nothrow) gcr_ctx();
    if (!c) return fail(GCR_ERR_OOM, "host allocation");
    c->cfg = cfg;
    auto cleanup = [&](int code) {
        gcr_destroy(c);
        return code;
    };
    if (cudaGetDevice(&c->device) != cudaSuccess) return cleanup(fail(GCR_ERR_CUDA, "no CUDA device"));
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    if (cuda_stream) {
        c->stream = (cudaStream_t)cuda_stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
            return cleanup(fail(GCR_ERR_CUDA, "stream creation"));
        c->own_stream = true;
    }
    c->ks = kernel_set(cfg.dim, cfg.precision);
    c->observe = observe_kernel(cfg.precision);
    {
        const char *e = std::getenv("GCR_PDL");
        c->pdl = !(e && e[0] == '0');
    }
    const int64_t S = cfg.system_capacity;
    c->max_bead_tiles = cfg.bead_capacity / cfg.block_beads + S;
    c->max_cell_tiles = cfg.cell_capacity / cfg.block_cells + S;
    const int64_t slots_total = cfg.cell_capacity * (int64_t)cfg.cell_depth;
    const size_t cells_alloc = (size_t)std::max<int64_t>(cfg.cell_capacity, 1);
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&c->dP, sizeof(SysP) * S);
    e = e ? e : cudaMalloc(&c->dS, sizeof(SysS) * S);
    e = e ? e : cudaMalloc(&c->d_bead_tiles, sizeof(Tile) * c->max_bead_tiles);
    e = e ? e : cudaMalloc(&c->d_cell_tiles, sizeof(Tile) * c->max_cell_tiles);
    e = e ? e : cudaMalloc(&c->d_ntiles, sizeof(int) * 2);
    e = e ? e : cudaMalloc(&c->d_row_prefix, sizeof(int) * (size_t)(S + 1));
    e = e ? e : cudaMemsetAsync(c->d_row_prefix, 0, sizeof(int) * (size_t)(S + 1), c->stream);
    e = e ? e : cudaMalloc(&c->topo, (size_t)cfg.bead_capacity);
    e = e ? e : cudaMalloc(&c->cnt, sizeof(int) * cells_alloc);
    e = e ? e : cudaMalloc(&c->ncell, sizeof(int) * cells_alloc);
    e = e ? e : cudaMalloc(&c->items, sizeof(int) * std::max<int64_t>(slots_total, 1));
    e = e ? e : cudaMalloc(&c->nbr, sizeof(int) * (size_t)cfg.bead_capacity * (size_t)cfg.list_depth);
    e = e ? e : cudaMalloc(&c->ncount, sizeof(int) * (size_t)cfg.bead_capacity);
    e = e ? e : cudaMalloc(&c->xref, sizeof(double) * (size_t)cfg.bead_capacity * cfg.dim);
    e = e ? e : cudaMalloc(&c->img, sizeof(int) * (size_t)cfg.bead_capacity * cfg.dim);
    e = e ? e : cudaMalloc(&c->restb, sizeof(double) * (size_t)cfg.bead_capacity);
    e = e ? e : cudaMalloc(&c->work, sizeof(int) * (size_t)(3 + 3 * (S + 1)));
    e = e ? e : cudaMalloc(&c->xi, (size_t)cfg.bead_capacity * cfg.dim * (cfg.precision == GCR_FP64 ? 8 : 4));
    e = e ? e : cudaMalloc(&c->fp, (size_t)cfg.bead_capacity * cfg.dim * (cfg.precision == GCR_FP64 ? 8 : 4));
    e = e ? e : cudaMalloc(&c->chain_starts, sizeof(int32_t) * (cfg.bead_capacity + S));
    e = e ? e : cudaMalloc(&c->d_err, 2 * sizeof(int));
    e = e ? e : cudaMalloc(&c->d_out, sizeof(double) * 8);
    if (cfg.srk_order == 4) {
        e = e ? e : cudaMalloc(&c->pos2, sizeof(double) * (size_t)cfg.bead_capacity * cfg.dim);
        e = e ? e : cudaMalloc(&c->faux, (size_t)cfg.bead_capacity * cfg.dim * (cfg.precision == GCR_FP64 ? 8 : 4));
    }
    if (e != cudaSuccess)
        return cleanup(fail(e == cudaErrorMemoryAllocation ? GCR_ERR_OOM : GCR_ERR_CUDA,
                            std::string("device allocation: ") + cudaGetErrorString(e)));
    cudaMemsetAsync(c->dS, 0, sizeof(SysS) * S, c->stream);
    cudaMemsetAsync(c->d_ntiles, 0, sizeof(int) * 2, c->stream);
    cudaMemsetAsync(c->cnt, 0, sizeof(int) * cells_alloc, c->stream);
    cudaMemsetAsync(c->ncell, 0, sizeof(int) * cells_alloc, c->stream);
    cudaMemsetAsync(c->ncount, 0, sizeof(int) * (size_t)cfg.bead_capacity, c->stream);
    cudaMemsetAsync(c->img, 0, sizeof(int) * (size_t)cfg.bead_capacity * cfg.dim, c->stream);
    cudaMemsetAsync(c->work, 0, sizeof(int) * (size_t)(3 + 3 * (S + 1)), c->stream);
    c->slots.assign(S, Slot());
    c->hP.assign(S, SysP());
    c->hS.assign(S, SysS());
    c->beads.init(cfg.bead_capacity);
    c->cells.init(cfg.cell_capacity);
    c->chains.init(cfg.bead_capacity + S);
    BatchArgs &a = c->args;
    a.P = c->dP;
    a.S = c->dS;
    a.bead_tiles = c->d_bead_tiles;
    a.n_bead_tiles = c->d_ntiles;
    a.cell_tiles = c->d_cell_tiles;
    a.n_cell_tiles = c->d_ntiles + 1;
    a.topo = c->topo;
    a.cnt = c->cnt;
    a.ncell = c->ncell;
    a.items = c->items;
    a.nbr = c->nbr;
    a.ncount = c->ncount;
    a.xref = c->xref;
    a.img = c->img;
    a.restb = c->restb;
    a.row_prefix = c->d_row_prefix;
    // staging capacity of the cell-staged pair kernel: twice the beads of a
    // row tile and its neighbour rows at the mean occupancy (the row tiling
    // aims at block_beads beads per row); a denser tile reads global memory
    a.cell_stage_cap = 2 * c->ks.pair_cells_rows * cfg.block_beads;
    a.xi = c->xi;
    a.fp = c->fp;
    a.work = c->work;
    a.n_slots = (int)S;
    a.list_stride = cfg.bead_capacity;
    a.list_depth = cfg.list_depth;
    a.depth = cfg.cell_depth;
    a.log_depth = ilog2(cfg.cell_depth);
    a.tile_beads = cfg.block_beads;
    a.tile_cells = cfg.block_cells;
    a.order = cfg.srk_order;
    c->stage_smem = c->ks.stage_smem(cfg.block_beads);
    if (c->stage_smem > 48 * 1024) {
        cudaFuncSetAttribute(c->ks.stage0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->stage_smem);
        cudaFuncSetAttribute(c->ks.stage1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->stage_smem);
        cudaFuncSetAttribute(c->ks.stage0f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->stage_smem);
        cudaFuncSetAttribute(c->ks.stage1f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->stage_smem);
        for (int k = 0; k < 4; k++)
            cudaFuncSetAttribute(c->ks.stage4[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->stage_smem);
    }
    for (int k = 0; k < 4; k++)
        c->grid_stage4[k] = kernel_grid(c, c->ks.stage4[k], cfg.block_beads, c->max_bead_tiles, c->stage_smem);
    c->grid_stage0 = kernel_grid(c, c->ks.stage0, cfg.block_beads, c->max_bead_tiles, c->stage_smem);
    c->grid_stage1 = kernel_grid(c, c->ks.stage1, cfg.block_beads, c->max_bead_tiles, c->stage_smem);
    c->grid_stage0f = kernel_grid(c, c->ks.stage0f, cfg.block_beads, c->max_bead_tiles, c->stage_smem);
    c->grid_stage1f = kernel_grid(c, c->ks.stage1f, cfg.block_beads, c->max_bead_tiles, c->stage_smem);
    c->pair_cells_smem = c->ks.pair_cells_smem(a.cell_stage_cap);
    if (c->pair_cells_smem > 48 * 1024)
        for (int k = 0; k < 2; k++)
            cudaFuncSetAttribute(c->ks.pair_cells[k], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)c->pair_cells_smem);
    // row tiles: at most cells/3 rows, plus cells/T <= 2 beads/block_beads (or cells/128) segments
    c->grid_pair_cells = kernel_grid(c, c->ks.pair_cells[0], cfg.block_beads,
                                     cfg.cell_capacity / 3 + cfg.cell_capacity / 128 +
                                         2 * cfg.bead_capacity / cfg.block_beads + S,
                                     c->pair_cells_smem);
    c->grid_update = kernel_grid(c, c->ks.update, cfg.block_beads, c->max_bead_tiles);
    c->pair_smem = c->ks.pair_smem(cfg.block_beads);
    c->grid_pair = kernel_grid(c, c->ks.pair0, cfg.block_beads, c->max_bead_tiles, c->pair_smem);
    c->grid_bin = kernel_grid(c, c->ks.bin0, cfg.block_beads, c->max_bead_tiles);
    c->grid_sort = kernel_grid(c, c->ks.sort, cfg.block_cells, c->max_cell_tiles);
    c->grid_build = kernel_grid(c, c->ks.build0, cfg.block_beads, c->max_bead_tiles);
    c->grid_sys = (int)((S + 127) / 128);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return cleanup(fail(GCR_ERR_CUDA, "initialisation"));
    *out = c;
    return GCR_OK;
}

int gcr_destroy(gcr_ctx *c)
{
    if (!c) return GCR_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    void *ptrs[] = {c->dP, c->dS, c->d_bead_tiles, c->d_cell_tiles, c->d_ntiles, c->d_row_prefix, c->topo, c->cnt,
                    c->ncell,
                    c->items, c->nbr, c->ncount, c->xref, c->work, c->xi, c->fp, c->chain_starts, c->d_err,
                    c->d_out, c->pos2, c->faux, c->xnbr, c->xcount, c->img, c->act, c->mpush, c->mdelta, c->restb};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GCR_OK;
}

int gcr_admit(gcr_ctx *c, const gcr_system_desc *desc, const gcr_system_buffers *buf, int32_t *slot_out)
{
    if (!c || !desc || !buf || !slot_out) return fail(GCR_ERR_BAD_ARG, "null argument");
    if (!buf->pos || !buf->pos1 || !buf->tangent || !buf->forces || !buf->chain_id || !buf->rest_lengths)
        return fail(GCR_ERR_BAD_ARG, "all state buffers must be bound");
    int64_t nc = 1;
    double skin = 0.0;
    int rc = validate_desc(c->cfg, desc, &nc, &skin);
    if (rc) return rc;
    int slot = -1;
    for (int s = 0; s < (int)c->slots.size(); s++)
        if (!c->slots[s].used) {
            slot = s;
            break;
        }
    if (slot < 0) return fail(GCR_ERR_CAPACITY, "no free system slot");
    int64_t n_cells = 0;
    if (desc->calc_wca) {
        n_cells = 1;
        for (int i = 0; i < c->cfg.dim; i++) n_cells *= nc;
    }
    int64_t boff = c->beads.alloc(desc->n_beads);
    if (boff < 0) return fail(GCR_ERR_CAPACITY, "bead capacity exhausted");
    int64_t coff = n_cells ? c->cells.alloc(n_cells) : 0;
    if (coff < 0) {
        c->beads.release(boff, desc->n_beads);
        return fail(GCR_ERR_CAPACITY, "cell capacity exhausted");
    }
    int64_t choff = c->chains.alloc(desc->n_chains + 1);
    if (choff < 0) {
        c->beads.release(boff, desc->n_beads);
        if (n_cells) c->cells.release(coff, n_cells);
        return fail(GCR_ERR_CAPACITY, "chain capacity exhausted");
    }
    Slot &sl = c->slots[slot];
    sl.used = true;
    sl.desc = *desc;
    sl.buf = *buf;
    sl.bead_off = boff;
    sl.cell_off = coff;
    sl.chain_off = choff;
    sl.n_cells = n_cells;
    sl.n_cells_alloc = n_cells;
    sl.nc = nc;
    fill_sysp(c, sl, nc, skin, c->hP[slot]);
    SysS &s = c->hS[slot];
    std::memset(&s, 0, sizeof(s));
    s.dt = desc->dtmax;
    s.step = desc->step;
    s.max_steps = 0;
    s.max_dt_usable = -1.0;
    GCR_CUDA(cudaMemcpyAsync(c->dP + slot, &c->hP[slot], sizeof(SysP), cudaMemcpyHostToDevice, c->stream));
    GCR_CUDA(cudaMemcpyAsync(c->dS + slot, &s, sizeof(SysS), cudaMemcpyHostToDevice, c->stream));
    int n = (int)desc->n_beads;
    void *targs[] = {(void *)&buf->chain_id, &n, nullptr};
    uint8_t *tp = c->topo + boff;
    targs[2] = &tp;
    GCR_CUDA(cudaMemsetAsync(c->d_err, 0, 2 * sizeof(int), c->stream));
    // image counters start at 0: unwrapped positions are measured from admission
    GCR_CUDA(cudaMemsetAsync(c->img + (size_t)boff * c->cfg.dim, 0, sizeof(int) * (size_t)n * c->cfg.dim, c->stream));
    GCR_CUDA(cudaLaunchKernel(c->ks.topo, dim3((n + 255) / 256), dim3(256), targs, 0, c->stream));
    GCR_CUDA(launch_chain_starts(buf->chain_id, n, (int)desc->n_chains, c->chain_starts + choff, c->d_err,
                                 c->stream));
    int err[2] = {0, 0};
    GCR_CUDA(cudaMemcpyAsync(err, c->d_err, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    if (err[0]) {
        c->beads.release(boff, desc->n_beads);
        if (n_cells) c->cells.release(coff, n_cells);
        c->chains.release(choff, desc->n_chains + 1);
        sl = Slot();
        return fail(GCR_ERR_BAD_ARG, "chain ids must run 0, 1, ..., n_chains - 1 in order (contiguous chains)");
    }
    sl.longest = err[1];
    fill_sysp(c, sl, nc, skin, c->hP[slot]);
    GCR_CUDA(cudaMemcpyAsync(c->dP + slot, &c->hP[slot], sizeof(SysP), cudaMemcpyHostToDevice, c->stream));
    // its first stage builds the lists, from zeroed counts in its cells
    rc = mark_rebuild(c, slot);
    if (rc) return rc;
    rc = rebuild_tiles(c);
    if (rc) return rc;
    *slot_out = slot;
    return GCR_OK;
}

int gcr_evict(gcr_ctx *c, int32_t slot)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    Slot &sl = c->slots[slot];
    // make sure no queued work still uses the slot's scratch
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    if (sl.group >= 0) {
        // its coupled populations step on their own again
        const Group members = c->groups[sl.group];
        dissolve(c, sl.group);
        int rc = drop_graph(c);
        if (rc) return rc;
        bool moved = false;
        rc = apply_groups(c, &moved);
        if (rc) return rc;
        for (int k = 0; k < members.n; k++)
            if (members.slots[k] != slot && (rc = mark_rebuild(c, members.slots[k]))) return rc;
    }
    c->beads.release(sl.bead_off, sl.desc.n_beads);
    if (sl.n_cells_alloc) c->cells.release(sl.cell_off, sl.n_cells_alloc);
    c->chains.release(sl.chain_off, sl.desc.n_chains + 1);
    sl = Slot();
    for (Slot &o : c->slots)
        if (o.motor_chain == slot) o.motor_chain = -1;
    SysS &s = c->hS[slot];
    std::memset(&s, 0, sizeof(s));
    GCR_CUDA(cudaMemcpyAsync(c->dS + slot, &s, sizeof(SysS), cudaMemcpyHostToDevice, c->stream));
    return rebuild_tiles(c);
}

int gcr_update_desc(gcr_ctx *c, int32_t slot, const gcr_system_desc *desc)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    Slot &sl = c->slots[slot];
    if (desc->n_beads != sl.desc.n_beads || desc->n_chains != sl.desc.n_chains)
        return fail(GCR_ERR_BAD_ARG, "bead and chain counts of a resident system cannot change");
    int64_t nc = 1;
    double skin = 0.0;
    int rc = validate_desc(c->cfg, desc, &nc, &skin);
    if (rc) return rc;
    if (sl.group >= 0) {
        // a coupled population keeps what gcr_couple checked: its cells
        // (the others' cross lists read them) and the shared box
        const Group &g = c->groups[sl.group];
        if (!desc->calc_wca) return fail(GCR_ERR_BAD_ARG, "a coupled population keeps its WCA force");
        for (int k = 0; k < g.n; k++)
            if (g.slots[k] != slot && c->slots[g.slots[k]].desc.L != desc->L)
                return fail(GCR_ERR_BAD_ARG, "coupled populations share L");
    }
    // the current grid stays while its cells cover the list radius (a new
    // descriptor marks the system for a list build, so a grid change between
    // calls is safe)
    if (desc->calc_wca && sl.desc.calc_wca && desc->L == sl.desc.L && sl.nc >= 3 &&
        desc->L / (double)sl.nc >= desc->wca_params[3] + skin)
        nc = sl.nc;
    int64_t n_cells = 0;
    if (desc->calc_wca) {
        n_cells = 1;
        for (int i = 0; i < c->cfg.dim; i++) n_cells *= nc;
    }
    if (n_cells > sl.n_cells_alloc)
        return fail(GCR_ERR_CAPACITY, "the new GPU cell grid needs more cells than were reserved at admission");
    // in-flight work reads the descriptor table
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    if (n_cells != sl.n_cells) c->tiles_dirty = true;
    sl.desc = *desc;
    sl.n_cells = n_cells;
    sl.nc = nc;
    fill_sysp(c, sl, nc, skin, c->hP[slot]);
    if (sl.group >= 0) {
        // the partners' cross-list radii and windows follow the new skin and grid
        bool moved = false;
        rc = apply_groups(c, &moved);
        if (rc) return rc;
        if (moved && (rc = drop_graph(c))) return rc;
        GCR_CUDA(cudaMemcpyAsync(c->dP, c->hP.data(), sizeof(SysP) * c->hP.size(), cudaMemcpyHostToDevice,
                                 c->stream));
    } else {
        GCR_CUDA(cudaMemcpyAsync(c->dP + slot, &c->hP[slot], sizeof(SysP), cudaMemcpyHostToDevice, c->stream));
    }
    // the lists follow the new cutoff, skin, exclusions and grid (coupled:
    // the partners' cross lists too)
    if (sl.group >= 0) {
        const Group &g = c->groups[sl.group];
        for (int k = 0; k < g.n; k++)
            if ((rc = mark_rebuild(c, g.slots[k]))) return rc;
    } else if ((rc = mark_rebuild(c, slot))) {
        return rc;
    }
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_couple(gcr_ctx *c, int32_t n, const int32_t *slots, const int32_t *fixed, const double *cross_wca)
{
    if (!c || !slots || !fixed || !cross_wca) return fail(GCR_ERR_BAD_ARG, "null argument");
    if (n < 2 || n > kMaxPops) return fail(GCR_ERR_BAD_ARG, "2 to 4 populations can be coupled");
    int g_old = -2;
    int movers = 0;
    for (int a = 0; a < n; a++) {
        if (!valid_slot(c, slots[a])) return fail(GCR_ERR_BAD_ARG, "invalid slot");
        for (int b = 0; b < a; b++)
            if (slots[b] == slots[a]) return fail(GCR_ERR_BAD_ARG, "a slot appears twice");
        const Slot &sl = c->slots[slots[a]];
        if (!sl.desc.calc_wca) return fail(GCR_ERR_BAD_ARG, "every coupled population needs its WCA force");
        if (sl.desc.L != c->slots[slots[0]].desc.L) return fail(GCR_ERR_BAD_ARG, "coupled populations share L");
        const int g = sl.group;
        if (g_old == -2) g_old = g;
        if (g != g_old || (g >= 0 && c->groups[g].n != n))
            return fail(GCR_ERR_BAD_ARG, "a slot is coupled to other populations (gcr_decouple first)");
        if (!fixed[a]) movers++;
        for (int b = 0; b < n; b++)
            for (int k = 0; k < 4; k++)
                if (!std::isfinite(cross_wca[((size_t)a * n + b) * 4 + k]))
                    return fail(GCR_ERR_BAD_ARG, "cross parameters must be finite");
    }
    if (movers == 0) return fail(GCR_ERR_BAD_ARG, "at least one coupled population must move");
    if (g_old >= 0) {
        // the same members again: their order must match
        for (int a = 0; a < n; a++)
            if (c->groups[g_old].slots[a] != slots[a])
                return fail(GCR_ERR_BAD_ARG, "re-coupling must list the members in the same order");
    }
    int rc = drop_graph(c);
    if (rc) return rc;
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    int g = g_old;
    if (g < 0) {
        for (int k = 0; k < (int)c->groups.size(); k++)
            if (c->groups[k].n == 0) {
                g = k;
                break;
            }
        if (g < 0) {
            c->groups.push_back(Group());
            g = (int)c->groups.size() - 1;
        }
    }
    Group &gr = c->groups[g];
    gr = Group();
    gr.n = n;
    for (int a = 0; a < n; a++) {
        gr.slots[a] = slots[a];
        gr.fixed[a] = fixed[a] ? 1 : 0;
        c->slots[slots[a]].group = g;
        for (int b = 0; b < n; b++)
            for (int k = 0; k < 4; k++) gr.cross[a][b][k] = a == b ? 0.0 : cross_wca[((size_t)a * n + b) * 4 + k];
    }
    bool moved = false;
    rc = apply_groups(c, &moved);
    if (rc) {
        dissolve(c, g);
        apply_groups(c, &moved);
        return rc;
    }
    c->tiles_dirty = true;
    for (int a = 0; a < n; a++)
        if ((rc = mark_rebuild(c, slots[a]))) return rc;
    return rebuild_tiles(c);
}

int gcr_decouple(gcr_ctx *c, int32_t slot)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    const int g = c->slots[slot].group;
    if (g < 0) return GCR_OK;
    int rc = drop_graph(c);
    if (rc) return rc;
    const Group members = c->groups[g];
    dissolve(c, g);
    bool moved = false;
    rc = apply_groups(c, &moved);
    if (rc) return rc;
    c->tiles_dirty = true;
    for (int k = 0; k < members.n; k++)
        if ((rc = mark_rebuild(c, members.slots[k]))) return rc;
    return rebuild_tiles(c);
}

int gcr_set_motors(gcr_ctx *c, int32_t motor_slot, int32_t chain_slot, const double *params, int32_t hold)
{
    if (!valid_slot(c, motor_slot)) return fail(GCR_ERR_BAD_ARG, "invalid motor slot");
    if (c->cfg.srk_order != 2) return fail(GCR_ERR_BAD_ARG, "motors are stepped by SRK2 contexts");
    Slot &ms = c->slots[motor_slot];
    if (chain_slot >= 0) {
        if (!valid_slot(c, chain_slot) || chain_slot == motor_slot)
            return fail(GCR_ERR_BAD_ARG, "invalid chain slot");
        if (!params) return fail(GCR_ERR_BAD_ARG, "null params");
        for (int k = 0; k < 5; k++)
            if (!std::isfinite(params[k])) return fail(GCR_ERR_BAD_ARG, "motor parameters must be finite");
        if (!(params[0] >= 0.0)) return fail(GCR_ERR_BAD_ARG, "motor_max_dist_sq must be >= 0");
        if (ms.desc.calc_springs || ms.desc.self_propel || ms.desc.n_chains != ms.desc.n_beads)
            return fail(GCR_ERR_BAD_ARG, "motors are single beads without springs or propulsion");
        for (const Slot &o : c->slots)
            if (&o != &ms && o.used && o.motor_chain == chain_slot)
                return fail(GCR_ERR_BAD_ARG, "the chains are pushed by another motor population");
    }
    int rc = drop_graph(c);
    if (rc) return rc;
    if (chain_slot >= 0 && !c->act) {
        const size_t n = (size_t)c->cfg.bead_capacity;
        cudaError_t e = cudaMalloc(&c->act, sizeof(int) * n);
        e = e ? e : cudaMalloc(&c->mpush, sizeof(int) * n);
        e = e ? e : cudaMalloc(&c->mdelta, sizeof(int) * n);
        e = e ? e : cudaMemsetAsync(c->act, 0xff, sizeof(int) * n, c->stream);  // -1
        e = e ? e : cudaMemsetAsync(c->mpush, 0, sizeof(int) * n, c->stream);
        e = e ? e : cudaMemsetAsync(c->mdelta, 0, sizeof(int) * n, c->stream);
        if (e != cudaSuccess) {
            for (int **q : {&c->act, &c->mpush, &c->mdelta}) {
                if (*q) cudaFree(*q);
                *q = nullptr;
            }
            return fail(e == cudaErrorMemoryAllocation ? GCR_ERR_OOM : GCR_ERR_CUDA, "motor arrays");
        }
        c->args.act = c->act;
        c->args.mpush = c->mpush;
        c->args.mdelta = c->mdelta;
    }
    const int old_chain = ms.motor_chain;
    ms.motor_chain = chain_slot;
    if (chain_slot >= 0) {
        for (int k = 0; k < 5; k++) ms.mparams[k] = params[k];
        ms.motor_hold = hold ? 1 : 0;
    }
    bool moved = false;
    if ((rc = apply_groups(c, &moved))) return rc;
    c->tiles_dirty = true;
    for (int32_t s : {motor_slot, chain_slot, (int32_t)old_chain})
        if (s >= 0 && valid_slot(c, s) && (rc = mark_rebuild(c, s))) return rc;
    return rebuild_tiles(c);
}

int gcr_where_active(gcr_ctx *c, int32_t slot, int32_t *dst)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    if (!dst) return fail(GCR_ERR_BAD_ARG, "null destination");
    if (!c->act) return fail(GCR_ERR_BAD_ARG, "no motor population was set");
    const Slot &sl = c->slots[slot];
    GCR_CUDA(cudaMemcpyAsync(dst, c->act + sl.bead_off, sizeof(int) * (size_t)sl.desc.n_beads,
                             cudaMemcpyDeviceToDevice, c->stream));
    return GCR_OK;
}

namespace {
int check_call(const gcr_call *call)
{
    if (!call) return fail(GCR_ERR_BAD_ARG, "null call");
    if (call->noise && call->noise_steps <= 0) return fail(GCR_ERR_BAD_ARG, "injected noise without steps");
    if (call->noise && call->max_steps < 0) return fail(GCR_ERR_BAD_ARG, "injected noise needs a step limit");
    if (call->noise && call->max_steps > call->noise_steps)
        return fail(GCR_ERR_BAD_ARG, "fewer injected noise steps than the step limit");
    if (call->series && (call->series_every <= 0 || call->series_capacity <= 0 || call->series_phase < 0))
        return fail(GCR_ERR_BAD_ARG, "a series needs series_every > 0, series_phase >= 0, series_capacity > 0");
    return GCR_OK;
}

// arm one system for a call; true when its last call ended in a stop (a
// fatal flag), after which its lists are rebuilt from zeroed cell counts
bool arm(SysS &s, const gcr_call *call)
{
    const bool stopped = (s.flags & kFlagFatal) != 0;
    // dt <= 0: the system keeps the dt its last step chose (status.dt of the
    // reference, which carries from call to call)
    if (call->dt > 0.0) s.dt = call->dt;
    s.dt_next = s.dt;
    s.dt_used = 0.0;
    s.elapsed = 0.0;
    s.max_f2 = 0ull;
    s.steps_done = 0;
    s.max_steps = call->max_steps;
    s.max_dt_usable = call->max_dt_usable;
    s.noise = call->noise;
    s.noise_steps = call->noise_steps;
    s.series = call->series;
    s.series_every = call->series ? call->series_every : 0;
    s.series_phase = call->series ? call->series_phase : 0;
    s.series_cap = call->series ? call->series_capacity : 0;
    s.series_rows = 0;
    s.series_mark = 0;
    s.flags = 0;
    s.active = ((0 < s.max_steps || s.max_steps < 0) && (0.0 < s.max_dt_usable || s.max_dt_usable < 0.0)) ? 1 : 0;
    return stopped;
}
}  // namespace

int gcr_call_begin_batch(gcr_ctx *c, int32_t n, const int32_t *slots, const gcr_call *calls)
{
    if (!c || n < 0 || (n > 0 && (!slots || !calls))) return fail(GCR_ERR_BAD_ARG, "bad argument");
    for (int i = 0; i < n; i++) {
        if (!valid_slot(c, slots[i])) return fail(GCR_ERR_BAD_ARG, "invalid slot");
        int rc = check_call(calls + i);
        if (rc) return rc;
    }
    const int S = (int)c->slots.size();
    // the device table holds the step counters: fetch it, arm, write it back
    GCR_CUDA(cudaMemcpyAsync(c->hS.data(), c->dS, sizeof(SysS) * S, cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    std::vector<int> stopped;
    for (int i = 0; i < n; i++)
        if (arm(c->hS[slots[i]], calls + i)) stopped.push_back(slots[i]);
    GCR_CUDA(cudaMemcpyAsync(c->dS, c->hS.data(), sizeof(SysS) * S, cudaMemcpyHostToDevice, c->stream));
    for (int sl : stopped) {
        int rc = mark_rebuild(c, sl);
        if (rc) return rc;
    }
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_call_begin(gcr_ctx *c, int32_t slot, const gcr_call *call)
{
    if (!valid_slot(c, slot) || !call) return fail(GCR_ERR_BAD_ARG, "invalid slot or call");
    int rc = check_call(call);
    if (rc) return rc;
    SysS &s = c->hS[slot];
    // the device copy holds the current step counter: fetch it first
    GCR_CUDA(cudaMemcpyAsync(&s, c->dS + slot, sizeof(SysS), cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    const bool stopped = arm(s, call);
    GCR_CUDA(cudaMemcpyAsync(c->dS + slot, &s, sizeof(SysS), cudaMemcpyHostToDevice, c->stream));
    if (stopped && (rc = mark_rebuild(c, slot))) return rc;
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_run(gcr_ctx *c, int64_t max_steps, int32_t sync_every)
{
    if (!c) return fail(GCR_ERR_BAD_ARG, "null context");
    if (max_steps <= 0) return GCR_OK;
    if (c->tiles_dirty) {
        int rc = rebuild_tiles(c);
        if (rc) return rc;
    }
    int rc = build_graph(c);
    if (rc) return rc;
    rc = enqueue_run_start(c);
    if (rc) return rc;
    const int64_t spg = c->cfg.steps_per_graph;
    const int64_t graphs = (max_steps + spg - 1) / spg;
    for (int64_t g = 0; g < graphs; g++) {
        GCR_CUDA(cudaGraphLaunch(c->graph, c->stream));
        if (sync_every > 0 && (g + 1) % sync_every == 0 && g + 1 < graphs) {
            int32_t n = 0;
            rc = gcr_count_active(c, &n);
            if (rc) return rc;
            if (n == 0) break;
        }
    }
    GCR_CUDA(cudaGetLastError());
    return GCR_OK;
}

int gcr_profile_steps(gcr_ctx *c, int32_t n_steps, float *ms_out)
{
    if (!c || !ms_out || n_steps <= 0) return fail(GCR_ERR_BAD_ARG, "bad argument");
    if (c->cfg.srk_order != 2) return fail(GCR_ERR_BAD_ARG, "per-group profiling covers SRK2 contexts");
    if (c->tiles_dirty) {
        int rc = rebuild_tiles(c);
        if (rc) return rc;
    }
    int rc = enqueue_run_start(c);
    if (rc) return rc;
    // groups: lists(pos), pair(pos), stage 0, lists(pos1), pair(pos1),
    // stage 1 + dt rule, update + bookkeeping
    const int G = 7;
    std::vector<cudaEvent_t> ev((size_t)n_steps * (G + 1), nullptr);
    for (auto &e : ev) GCR_CUDA(cudaEventCreate(&e));
    const int bb = c->cfg.block_beads;
    const bool rigid = any_rigid(c), cross = any_cross(c);
    for (int s = 0; s < n_steps && rc == GCR_OK; s++) {
        cudaEvent_t *e = ev.data() + (size_t)s * (G + 1);
        GCR_CUDA(cudaEventRecord(e[0], c->stream));
        rc = enqueue_lists(c, 0);
        GCR_CUDA(cudaEventRecord(e[1], c->stream));
        if (!rc) rc = enqueue_pair(c, 0, cross);  // nothing with fused stages
        if (!rc && any_motor(c)) rc = launch(c, c->ks.motor[0], c->grid_update, bb);
        GCR_CUDA(cudaEventRecord(e[2], c->stream));
        if (!rc) rc = enqueue_stage(c, 0, cross);
        if (!rc && rigid) rc = launch(c, c->ks.rigid0, c->grid_update, bb);
        GCR_CUDA(cudaEventRecord(e[3], c->stream));
        if (!rc) rc = enqueue_lists(c, 1);
        GCR_CUDA(cudaEventRecord(e[4], c->stream));
        if (!rc) rc = enqueue_pair(c, 1, cross);
        if (!rc && any_motor(c)) rc = launch(c, c->ks.motor[1], c->grid_update, bb);
        GCR_CUDA(cudaEventRecord(e[5], c->stream));
        if (!rc) rc = enqueue_stage(c, 1, cross);
        if (!rc) rc = launch_sys(c, c->ks.sys_dt);
        GCR_CUDA(cudaEventRecord(e[6], c->stream));
        if (!rc) rc = launch(c, c->ks.update, c->grid_update, bb);
        if (!rc && rigid) rc = launch(c, c->ks.rigid1, c->grid_update, bb);
        if (!rc) rc = launch_sys(c, c->ks.sys_end);
        GCR_CUDA(cudaEventRecord(e[7], c->stream));
    }
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < G; k++) ms_out[k] = 0.f;
    for (int s = 0; s < n_steps; s++)
        for (int k = 0; k < G; k++) {
            float ms = 0.f;
            GCR_CUDA(cudaEventElapsedTime(&ms, ev[(size_t)s * (G + 1) + k], ev[(size_t)s * (G + 1) + k + 1]));
            ms_out[k] += ms;
        }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}

int gcr_unwrapped_positions(gcr_ctx *c, int32_t slot, double *out)
{
    if (!valid_slot(c, slot) || !out) return fail(GCR_ERR_BAD_ARG, "bad argument");
    const Slot &sl = c->slots[slot];
    GCR_CUDA(launch_unwrap(c->cfg.dim, sl.buf.pos, c->img + (size_t)sl.bead_off * c->cfg.dim, (int)sl.desc.n_beads,
                           sl.desc.L, out, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_reset_images(gcr_ctx *c, int32_t slot)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    const Slot &sl = c->slots[slot];
    GCR_CUDA(cudaMemsetAsync(c->img + (size_t)sl.bead_off * c->cfg.dim, 0,
                             sizeof(int) * (size_t)sl.desc.n_beads * c->cfg.dim, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_synchronize(gcr_ctx *c)
{
    if (!c) return fail(GCR_ERR_BAD_ARG, "null context");
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_count_active(gcr_ctx *c, int32_t *n_out)
{
    if (!c || !n_out) return fail(GCR_ERR_BAD_ARG, "null argument");
    const int S = (int)c->slots.size();
    GCR_CUDA(cudaMemcpyAsync(c->hS.data(), c->dS, sizeof(SysS) * S, cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    int n = 0;
    for (int s = 0; s < S; s++)
        if (c->slots[s].used && c->hS[s].active) n++;
    *n_out = n;
    return GCR_OK;
}

namespace {
void fill_status(const SysS &s, gcr_status *out)
{
    out->dt = s.dt;
    out->dt_used = s.elapsed;
    out->max_forces_strength = s.mfs;
    out->steps_done = s.steps_done;
    out->step = s.step;
    out->flags = s.flags;
    out->active = s.active;
    out->list_builds = s.list_builds;
    out->series_rows = s.series_rows;
}
}  // namespace

int gcr_get_statuses(gcr_ctx *c, int32_t n, const int32_t *slots, gcr_status *out)
{
    if (!c || n < 0 || (n > 0 && (!slots || !out))) return fail(GCR_ERR_BAD_ARG, "bad argument");
    for (int i = 0; i < n; i++)
        if (!valid_slot(c, slots[i])) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    const int S = (int)c->slots.size();
    GCR_CUDA(cudaMemcpyAsync(c->hS.data(), c->dS, sizeof(SysS) * S, cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < n; i++) fill_status(c->hS[slots[i]], out + i);
    return GCR_OK;
}

int gcr_get_status(gcr_ctx *c, int32_t slot, gcr_status *out)
{
    if (!valid_slot(c, slot) || !out) return fail(GCR_ERR_BAD_ARG, "invalid slot or output");
    SysS &s = c->hS[slot];
    GCR_CUDA(cudaMemcpyAsync(&s, c->dS + slot, sizeof(SysS), cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    fill_status(s, out);
    return GCR_OK;
}

int gcr_order_params(gcr_ctx *c, int32_t slot, double out[3])
{
    if (!valid_slot(c, slot) || !out) return fail(GCR_ERR_BAD_ARG, "invalid slot or output");
    if (c->cfg.dim != 2) return fail(GCR_ERR_BAD_ARG, "order parameters are defined for 2D systems");
    const Slot &sl = c->slots[slot];
    GCR_CUDA(launch_order_params(c->cfg.dim, c->cfg.precision, c->hP[slot], c->chain_starts + sl.chain_off,
                                 c->d_out, c->stream));
    GCR_CUDA(cudaMemcpyAsync(out, c->d_out, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_reference_lists(gcr_ctx *c, int32_t slot, int64_t n_grid, int64_t grid_window, int64_t *where_is_bead,
                        int64_t *grid_list, int64_t grid_depth1, int64_t *nbor_list, int64_t nbor_depth1,
                        int32_t mode)
{
    if (!valid_slot(c, slot) || !where_is_bead) return fail(GCR_ERR_BAD_ARG, "invalid slot or output");
    if (n_grid < 1 || grid_window < 1) return fail(GCR_ERR_BAD_ARG, "bad grid");
    if (grid_list && grid_depth1 < 3) return fail(GCR_ERR_BAD_ARG, "grid depth too small");
    if (nbor_list && nbor_depth1 < 2) return fail(GCR_ERR_BAD_ARG, "neighbour depth too small");
    if (mode == 1 && !grid_list) return fail(GCR_ERR_BAD_ARG, "the cell-window neighbour list needs grid_list");
    GCR_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    SysP p = c->hP[slot];
    // mode 0: the rule of SRK.py:450 (all-pairs when N < n_grid^dim),
    // 1: cell window (populations.update_nbor_list_with_pop2), 2: all pairs
    int64_t n_pow = 1;
    for (int i = 0; i < c->cfg.dim; i++) n_pow *= n_grid;
    bool few = (mode == 2) || (mode == 0 && p.n < n_pow) || !grid_list;
    if (few && nbor_list && p.n > 200000)
        return fail(GCR_ERR_BAD_ARG, "the all-pairs neighbour builder is limited to 200000 beads");
    GCR_CUDA(launch_reference_lists(c->cfg.dim, p, n_grid, grid_window, where_is_bead, grid_list, grid_depth1,
                                    few ? nullptr : nbor_list, nbor_depth1, c->d_err, c->stream));
    if (few && nbor_list)
        GCR_CUDA(launch_reference_lists(c->cfg.dim, p, n_grid, grid_window, where_is_bead, nullptr, grid_depth1,
                                        nbor_list, nbor_depth1, c->d_err, c->stream));
    int err = 0;
    GCR_CUDA(cudaMemcpyAsync(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    if (err) return fail(GCR_ERR_OVERFLOW, err & 1 ? "grid_list depth too small" : "nbor_list depth too small");
    return GCR_OK;
}

int gcr_cell_assignment(gcr_ctx *c, int32_t slot, int32_t *cell_of_bead, int32_t *n_cells_side)
{
    if (!valid_slot(c, slot) || !cell_of_bead) return fail(GCR_ERR_BAD_ARG, "invalid slot or output");
    GCR_CUDA(launch_cell_assignment(c->cfg.dim, c->hP[slot], cell_of_bead, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    if (n_cells_side) *n_cells_side = c->hP[slot].nc;
    return GCR_OK;
}

int gcr_neighbour_list(gcr_ctx *c, int32_t slot, int32_t *counts, int32_t *partners, int32_t partners_depth,
                       double *build_pos, int64_t *entries)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    if (partners && partners_depth < c->cfg.list_depth)
        return fail(GCR_ERR_BAD_ARG, "partners_depth is smaller than the context's list_depth");
    const Slot &sl = c->slots[slot];
    unsigned long long *total = reinterpret_cast<unsigned long long *>(c->d_out);
    GCR_CUDA(cudaMemsetAsync(total, 0, sizeof(unsigned long long), c->stream));
    GCR_CUDA(launch_export_list(c->nbr + sl.bead_off, c->ncount + sl.bead_off, c->cfg.bead_capacity,
                                c->cfg.list_depth, (int)sl.desc.n_beads, counts, partners, partners_depth, total,
                                c->stream));
    if (build_pos)
        GCR_CUDA(cudaMemcpyAsync(build_pos, c->xref + (size_t)sl.bead_off * c->cfg.dim,
                                 sizeof(double) * (size_t)sl.desc.n_beads * c->cfg.dim, cudaMemcpyDeviceToDevice,
                                 c->stream));
    unsigned long long h = 0;
    GCR_CUDA(cudaMemcpyAsync(&h, total, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    if (entries) *entries = (int64_t)h;
    return GCR_OK;
}

int gcr_chain_frames(gcr_ctx *c, int32_t slot, double *com, double *phi)
{
    if (!valid_slot(c, slot)) return fail(GCR_ERR_BAD_ARG, "invalid slot");
    const Slot &sl = c->slots[slot];
    GCR_CUDA(launch_chain_frames(c->cfg.dim, c->cfg.precision, c->hP[slot], c->chain_starts + sl.chain_off, com, phi,
                                 c->stream));
    GCR_CUDA(cudaStreamSynchronize(c->stream));
    return GCR_OK;
}

int gcr_pair_correlation(gcr_ctx *c, int32_t slot, int32_t kind, double binsize, double *out, int32_t max_rows,
                         int32_t *n_rows)
{
    if (!valid_slot(c, slot) || !out || !n_rows) return fail(GCR_ERR_BAD_ARG, "invalid slot or output");
    if (c->cfg.dim != 2) return fail(GCR_ERR_BAD_ARG, "the pair correlations are defined for 2D systems");
    if (kind < 0 || kind > 2) return fail(GCR_ERR_BAD_ARG, "kind must be 0 (g(r)), 1 (Cvv) or 2 (Cnn)");
    if (!(binsize > 0.0) || !std::isfinite(binsize)) return fail(GCR_ERR_BAD_ARG, "binsize must be positive");
    const SysP &p = c->hP[slot];
    // bins of np.arange(0, int(L/2) * sqrt(2), binsize)
    const double stop = (double)(int64_t)(p.L / 2.0) * std::sqrt(2.0);
    const int64_t n_bins = (int64_t)std::ceil(stop / binsize);
    if (n_bins < 1 || n_bins > 12000) return fail(GCR_ERR_BAD_ARG, "binsize gives more than 12000 bins");
    const int nc = p.n_chains;
    if (kind != 0 && (int64_t)nc * (nc - 1) > ((int64_t)1 << 31))
        return fail(GCR_ERR_BAD_ARG, "Cvv / Cnn are limited to about 46000 chains (fixed-point sums)");
    double *com = nullptr, *phi = nullptr;
    unsigned long long *hist = nullptr;
    // analysis call, not the step: its scratch is allocated here and freed below
    cudaError_t e = cudaMalloc(&com, sizeof(double) * 2 * (size_t)nc);
    if (e == cudaSuccess) e = cudaMalloc(&phi, sizeof(double) * 2 * (size_t)nc);
    if (e == cudaSuccess) e = cudaMalloc(&hist, sizeof(unsigned long long) * 2 * (size_t)n_bins);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * 2 * (size_t)n_bins, c->stream);
    if (e == cudaSuccess)
        e = launch_chain_frames(2, c->cfg.precision, p, c->chain_starts + c->slots[slot].chain_off, com, phi, c->stream);
    if (e == cudaSuccess)
        e = launch_pair_corr(com, phi, nc, p.L, binsize, (int)n_bins, kind, hist, hist + n_bins, c->sm_count, c->stream);
    std::vector<unsigned long long> h((size_t)(2 * n_bins));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), hist, sizeof(unsigned long long) * 2 * (size_t)n_bins, cudaMemcpyDeviceToHost,
                            c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(com);
    cudaFree(phi);
    cudaFree(hist);
    if (e != cudaSuccess) return fail(GCR_ERR_CUDA, std::string("pair correlation: ") + cudaGetErrorString(e));
    // normalisation of correlation_func (analysis.py:229-237), rows with r < L/2
    double total = 0.0;
    for (int64_t b = 0; b < n_bins; b++) total += (double)h[b];
    const double density = total / (p.L * p.L);
    int32_t rows = 0;
    for (int64_t b = 0; b < n_bins; b++) {
        const double r = (double)b * binsize;
        if (!(r < p.L / 2.0)) continue;
        if (rows >= max_rows) return fail(GCR_ERR_CAPACITY, "out has fewer rows than the correlation");
        double v;
        if (kind == 0) {
            v = (double)h[b] / (density * 2.0 * M_PI * binsize * (r + binsize / 2.0));
        } else {
            const double sum = (double)(long long)h[n_bins + b] / 4294967296.0;
            v = sum / (double)std::max<unsigned long long>(h[b], 1ull);
        }
        out[2 * rows] = r;
        out[2 * rows + 1] = v;
        rows++;
    }
    *n_rows = rows;
    return GCR_OK;
}

int gcr_philox_noise(int32_t dim, uint64_t seed, int64_t step, int64_t n, int32_t do_trans, int32_t do_rot,
                     double *out, void *cuda_stream)
{
    if ((dim != 2 && dim != 3) || n < 0 || !out) return fail(GCR_ERR_BAD_ARG, "bad argument");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    GCR_CUDA(launch_philox_noise(dim, seed, step, n, do_trans, do_rot, out, st));
    GCR_CUDA(cudaStreamSynchronize(st));
    return GCR_OK;
}

}  // extern "C"
