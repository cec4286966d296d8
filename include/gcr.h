/*
 * gcr.h -- C ABI of libgcr.so, the B200 (sm_100a) hot path of the
 * gliding-collective-rotation Brownian-dynamics step.
 *
 * One context (gcr_ctx) owns the device scratch for up to `system_capacity`
 * independent bead-spring-chain systems with `bead_capacity` beads in total.
 * Bead state (positions, tangents, forces, chain ids, rest lengths) lives in
 * caller-owned device buffers that are bound to a slot at admission; the
 * library never frees them.  A context is bound to one CUDA stream and is not
 * thread-safe; separate contexts may be used concurrently.
 *
 * Every function returns GCR_OK (0) or a negative GCR_ERR_* code; no C++
 * exception crosses this boundary.  gcr_last_error() gives a message for the
 * last failure on the calling thread.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   gcr_run / gcr_call_begin  <- updates.SRK2_force_calc   updates.py:132-267
 *                                (the SRK.SRK_jit loop      SRK.py:13-484; SRK2, and SRK4
 *                                with gcr_config.srk_order = 4)
 *   pair rule                 <- force_rules.central_pair_force_rule = forces.WCA
 *                                                           force_rules.py:3, forces.py:13-15
 *   gcr_system_desc packing   <- populations.make_WCA_params populations.py:48-58,
 *                                Chain_Collection.spring_params populations.py:345-353,
 *                                Chain_Collection.active_params populations.py:355-358,
 *                                SRK2_force_calc time_vals / pop_consts updates.py:138-162
 *   gcr_reference_lists       <- updates.update_grid_list_mini updates.py:502-522 and
 *                                updates.update_nbor_list   updates.py:586-669
 *   gcr_system_desc.rigid_rod <- updates.project_updates_for_rigid_rod updates.py:347-499
 *                                (applied as SRK.py:364-378 applies it)
 *   gcr_couple                <- SRK2_force_calc over several populations updates.py:146-247,
 *                                interpop_forces updates.py:274-312, cross-population pair
 *                                forces SRK.py:229-245, 287-294
 *   gcr_set_motors            <- forces.calc_motor_push forces.py:248-283 with the motor_push
 *                                parameters of Chain_Collection.interactions populations.py:276-287,
 *                                Motor_Population diffusion SRK.py:389-395
 *   gcr_where_active          <- pop.where_active (SRK.py:132, forces.py:267-279)
 *   gcr_order_params          <- output_methods.calc_avg_phi_chain output_methods.py:492-510,
 *                                analysis.polar_orderparameter analysis.py:315-328,
 *                                analysis.nematic_orderparameter analysis.py:294-313
 */
#ifndef GCR_H
#define GCR_H

#include <stdint.h>

#if defined(__GNUC__)
#define GCR_API __attribute__((visibility("default")))
#else
#define GCR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GCR_OK 0
#define GCR_ERR_BAD_ARG (-1)
#define GCR_ERR_CUDA (-2)
#define GCR_ERR_OOM (-3)
#define GCR_ERR_NONFINITE (-4)
#define GCR_ERR_TIMEOUT (-5)
#define GCR_ERR_CAPACITY (-6)
#define GCR_ERR_STATE (-7)
#define GCR_ERR_OVERFLOW (-8)

/* precision of forces, tangents and SRK arithmetic (positions are FP64) */
#define GCR_FP64 0
#define GCR_MIXED 1

/* per-system device status flags */
#define GCR_FLAG_CELL_OVERFLOW 1   /* more beads in a cell than cell_depth */
#define GCR_FLAG_NONFINITE 2       /* a non-finite force or position */
#define GCR_FLAG_NEXT_OVERFLOW 4   /* reserved (no longer raised) */
#define GCR_FLAG_LIST_CORRUPT 8    /* an inconsistent cell or neighbour list was detected and not used */
#define GCR_FLAG_LIST_OVERFLOW 16  /* more list partners of a bead than list_depth */
#define GCR_FLAG_SERIES_FULL 32    /* the order-parameter series buffer was full (rows dropped; not fatal) */

typedef struct gcr_ctx gcr_ctx;

typedef struct {
    int32_t dim;              /* 2 or 3 (every system of a context has it) */
    int32_t precision;        /* GCR_FP64 or GCR_MIXED */
    int64_t bead_capacity;    /* beads over all resident systems */
    int32_t system_capacity;  /* resident systems */
    int64_t cell_capacity;    /* GPU cells over all resident systems */
    int32_t cell_depth;       /* bead slots per GPU cell: 8, 16, 32, 64 or 128 */
    int32_t block_beads;      /* threads per CTA of bead kernels (64..512) */
    int32_t block_cells;      /* threads per CTA of the cell kernel (64..512) */
    int32_t steps_per_graph;  /* SRK2 steps per captured CUDA graph (1..64) */
    int32_t ctas_per_sm;      /* persistent CTAs per SM (0 = from occupancy, <0 = one CTA per tile) */
    int32_t list_depth;       /* neighbour-list slots per bead, 4..1024 (0 = 32 in 2D, 96 in 3D) */
    int32_t srk_order;        /* config.SRK_order: 2 (0 = 2) or 4 (SRK.py:144-215, 296-321) */
    int32_t pair_mode;        /* pair forces of SRK2 contexts while no system is coupled to another
                                 population (SRK4 and coupled systems always use 0):
                                 0: a pair kernel walks each bead's neighbour list;
                                 1: the stage kernels walk the lists themselves (no pair launch;
                                    the same bits as 0);
                                 2: a cell-staged pair kernel: each CTA copies a row of cells and
                                    its neighbour cells into shared memory and sums over them (the
                                    same pairs as 0, summed cell by cell: FP rounding differs) */
} gcr_config;

/* One system.  The packed arrays follow the reference's packing exactly. */
typedef struct {
    int64_t n_beads;
    int64_t n_chains;
    double L;                   /* periodic box side */
    double spring_params[6];    /* [k, kappa, theta0, FENE(=0), get_orientations, FENE_tol] */
    double wca_params[4];       /* [12 eps r^6, 12 eps r^12, shift, r_cut] */
    double active_params[3];    /* [v0, sliding_partner_maxdist(=0), v_tan_angle] */
    int32_t calc_springs;       /* "springs" force present and chains longer than 1 */
    int32_t calc_wca;           /* "WCA" force present */
    int32_t self_propel;        /* "self-propulsion" present and b_calc_active_forces */
    int32_t n_nearby;           /* n_nearby_beads_dont_repel (<0: whole chain) */
    double D, Dr, radius;       /* pop_consts [D, Dr, repel_d_max] */
    double dtmax, max_dist_per_step, rk_cheat;
    uint64_t seed;              /* Philox key */
    int64_t step;               /* global index of the next step (Philox counter) */
    double cell_factor;         /* GPU cell side >= (r_cut + skin) * cell_factor (>= 1) */
    double skin;                /* Verlet skin (>= 0): the neighbour list holds the pairs within
                                   r_cut + skin and is rebuilt once a bead has moved skin / 2;
                                   reduced to L/3 - r_cut when the box is too small for it */
    double rigid_rod;           /* rigid_rod_projection_factor (populations.py:325-329): each chain's
                                   update is blended with that of a rigid rod of its rest length;
                                   0 = off; applied only when the longest chain has more than 2 beads
                                   (SRK.py:364) */
} gcr_system_desc;

/* Caller-owned device buffers of one system (bound, not copied). */
typedef struct {
    double *pos;                /* [n, dim] FP64 */
    double *pos1;               /* [n, dim] FP64 predictor positions */
    void *tangent;              /* [n, dim] FP64 or FP32 (precision) */
    void *forces;               /* [n, dim] FP64 or FP32 (precision) */
    const int32_t *chain_id;    /* [n] chain index; chains are contiguous ranges */
    const double *rest_lengths; /* [n_chains] */
    void *forces_aux;           /* SRK4: [n, dim] FP64 or FP32, the force of the last stage
                                   (pop.forces_aux); NULL: library scratch.  Unused by SRK2 */
} gcr_system_buffers;

/* Limits and inputs of one SRK2_force_calc call for one system. */
typedef struct {
    int64_t max_steps;          /* next_output_step - stepnum (<0: unlimited) */
    double max_dt_usable;       /* next_save_time - t; negative: unlimited (SRK.py:128-129) */
    double dt;                  /* status.dt: predictor dt of the first step (<= 0: keep the
                                   system's current dt, i.e. carry it over from its last call) */
    const double *noise;        /* injected noise_vec snapshots [noise_steps][n][2*dim],
                                   device memory, or NULL for the Philox stream */
    int64_t noise_steps;
    double *series;             /* device buffer of series_capacity rows (step, time elapsed in
                                   the call, P, S, director angle): a row is appended on the
                                   device after each step k of the call with
                                   (k + series_phase) % series_every == 0, the order parameters
                                   of gcr_order_params (global_op-chiral.py:24-30); NULL: none */
    int64_t series_every;
    int64_t series_phase;
    int64_t series_capacity;
} gcr_call;

/* What SRK2_force_calc writes back (shared_arr[0], updates.py:249-256). */
typedef struct {
    double dt;                  /* most recent dt */
    double dt_used;             /* time elapsed in the call */
    double max_forces_strength; /* sqrt(2D) + max|F0+F1| / (2 r) of the last step */
    int64_t steps_done;         /* steps completed in the call */
    int64_t step;               /* global index of the next step */
    int32_t flags;              /* GCR_FLAG_* */
    int32_t active;             /* still running (limits not reached) */
    int64_t list_builds;        /* neighbour-list builds since admission */
    int64_t series_rows;        /* rows appended to the call's series */
} gcr_status;

/* ---- context ---------------------------------------------------------- */
GCR_API int gcr_create(const gcr_config *cfg, void *cuda_stream, gcr_ctx **out);
GCR_API int gcr_destroy(gcr_ctx *ctx);
GCR_API const char *gcr_last_error(void);
GCR_API int gcr_version(void);

/* ---- systems ---------------------------------------------------------- */
/* Admit a system: reserves scratch, derives the GPU cell grid, uploads its
 * descriptor.  Fails with GCR_ERR_CAPACITY when beads, cells or slots do not
 * fit (the caller queues it). */
GCR_API int gcr_admit(gcr_ctx *ctx, const gcr_system_desc *desc, const gcr_system_buffers *buf,
              int32_t *slot_out);
GCR_API int gcr_evict(gcr_ctx *ctx, int32_t slot);
/* Replace the parameters of a resident system (same bead and chain counts).
 * A changed pair cutoff or skin keeps the GPU cell grid while its cells still
 * cover r_cut + skin, else re-derives it within the cells reserved at
 * admission (GCR_ERR_CAPACITY beyond them: evict and re-admit). */
GCR_API int gcr_update_desc(gcr_ctx *ctx, int32_t slot, const gcr_system_desc *desc);
/* Arm a resident system for the next gcr_run (one SRK2_force_calc call). */
GCR_API int gcr_call_begin(gcr_ctx *ctx, int32_t slot, const gcr_call *call);
/* Arm `n` resident systems at once (one copy of the state table each way). */
GCR_API int gcr_call_begin_batch(gcr_ctx *ctx, int32_t n, const int32_t *slots, const gcr_call *calls);
/* Cells and bytes a system of this description would occupy. */
GCR_API int gcr_footprint(const gcr_config *cfg, const gcr_system_desc *desc, int64_t *cells_out,
                  int64_t *bytes_out);

/* ---- several populations in one box ------------------------------------ */
#define GCR_MAX_POPULATIONS 4
/* Couple 2..4 resident systems as the populations of one box, listed in the
 * reference's population order (config.pop_name_list): the multi-population
 * updates.SRK2_force_calc (updates.py:146-247) with the SRK loop's
 * cross-population pair forces (SRK.py:229-245, 287-294).  From the next
 * gcr_run the members
 *   - step under one dt: the max-force rule (SRK.py:323-353) over the largest
 *     sqrt(2D) + pref max|F|/r of the moving members, the max over every
 *     thread's shared_arr[:,3];
 *   - rebuild their neighbour lists together;
 *   - each moving member i feels, after its own pair force, the WCA force of
 *     each other member j, taken j = i+1, i+2, ... (mod n) as the reference
 *     adds them, with parameters cross_wca[(i*n + j)*4 + 0..3] = [p0, p1,
 *     shift, r_cut] of forces.WCA (interpop_forces, updates.py:274-312: the
 *     mean of the two WCA parameter sets unless a special interaction says
 *     otherwise); r_cut <= 0 or p0 = p1 = 0 means no force.
 * fixed[i] != 0 (pop.fixed): member i never moves and feels no force, but
 * still acts on the others.  Every member needs calc_wca and the same L (also
 * through later gcr_update_desc calls); the dt rule takes dtmax,
 * max_dist_per_step and rk_cheat from the first moving member (time_vals are
 * one array for every population in the reference).  The moving members are
 * armed together with the same limits for each call.  Calling it again with
 * the same members in the same order replaces fixed and cross_wca. */
GCR_API int gcr_couple(gcr_ctx *ctx, int32_t n, const int32_t *slots, const int32_t *fixed,
                       const double *cross_wca);
/* Dissolve the coupled group that holds `slot` (no-op when there is none);
 * evicting a member does the same. */
GCR_API int gcr_decouple(gcr_ctx *ctx, int32_t slot);
/* Motors (Motor_Population, populations.py:617-661; forces.calc_motor_push,
 * forces.py:248-283; its diffusion, SRK.py:389-395).  `motor_slot` holds the
 * motors as single beads (chains of 1, springs and propulsion off, calc_wca
 * with p0 = p1 = 0 so that they are binned, D = D_motors); it pushes the
 * beads of `chain_slot`, a moving member of the same coupled group whose
 * cross entry (motor from chains) in gcr_couple has r_cut = the list radius
 * of the reference's chain-motor lists (grid_window * Lx / n_grid) and p0 =
 * p1 = 0.  params = [motor_max_dist_sq, b_one_motor_per_bead, imparts_force,
 * k_on, k_off] as Chain_Collection.interactions packs them
 * (populations.py:276-287); hold = b_motors_dont_diffuse_while_pushing.
 * Each SRK2 stage a motor walks the chain beads within the list radius in
 * ascending id, detaches with probability k_off, attaches with probability
 * k_on when within motor_max_dist and then pushes that bead once by
 * imparts_force along its tangent; where_active is -1 at the start of each
 * step.  Draws are keyed Philox (seed of the motor system) instead of the
 * reference's unseeded sequential np.random.random().  SRK2 contexts only;
 * chain_slot = -1 turns the slot back into a plain population. */
GCR_API int gcr_set_motors(gcr_ctx *ctx, int32_t motor_slot, int32_t chain_slot, const double *params,
                           int32_t hold);
/* where_active of a resident system (pop.where_active: chains, the motors
 * attached minus one; motors, the bead pushed or -1) as int32 [n_beads] into
 * device memory `dst` on the context stream; GCR_ERR_BAD_ARG before any
 * motor population was set. */
GCR_API int gcr_where_active(gcr_ctx *ctx, int32_t slot, int32_t *dst);

/* ---- stepping --------------------------------------------------------- */
/* Advance every armed system until its limits are reached or `max_steps`
 * steps have been launched, through captured CUDA graphs of
 * steps_per_graph steps.  `sync_every` graphs between checks of whether any
 * system is still running (0: never check; run exactly ceil(max_steps /
 * steps_per_graph) graphs).  Asynchronous on the context stream unless a
 * check is made. */
GCR_API int gcr_run(gcr_ctx *ctx, int64_t max_steps, int32_t sync_every);
/* Copy the status of a system to the host (synchronises the stream). */
GCR_API int gcr_get_status(gcr_ctx *ctx, int32_t slot, gcr_status *out);
/* The statuses of `n` resident systems `slots` at once, out[n] (host): one
 * copy of the state table (synchronises the stream).  Like gcr_get_status,
 * the write-back of updates.SRK2_force_calc (updates.py:249-256), for many
 * systems at the end of a serving round. */
GCR_API int gcr_get_statuses(gcr_ctx *ctx, int32_t n, const int32_t *slots, gcr_status *out);
/* Number of armed systems still running (synchronises the stream). */
GCR_API int gcr_count_active(gcr_ctx *ctx, int32_t *n_out);
GCR_API int gcr_synchronize(gcr_ctx *ctx);
/* Run `n_steps` steps launching the step kernels one by one (not through
 * the graph) with CUDA events between groups on the context stream;
 * ms_out[0..6] receive the total milliseconds of: cell list of pos (scans and
 * pack), pair forces at pos, stage 0, cell list of pos1, pair forces at
 * pos1, stage 1 with the dt rule, update with the step bookkeeping.  For
 * profiling; the results equal gcr_run's.  SRK2 contexts only. */
GCR_API int gcr_profile_steps(gcr_ctx *ctx, int32_t n_steps, float *ms_out);

/* ---- observables and exports ------------------------------------------ */
/* [P, S, director_angle] of one system from its tangents, FP64 (host out). */
GCR_API int gcr_order_params(gcr_ctx *ctx, int32_t slot, double out[3]);
/* The reference's cell and neighbour lists of one system, built on the
 * device from its current positions: where_is_bead int64 [n,3], grid_list
 * int64 [n_grid, n_grid, nz, grid_depth1], nbor_list int64 [n, nbor_depth1]
 * (device buffers).  Returns GCR_ERR_OVERFLOW when a depth is too small
 * (the reference then doubles it).  mode 0 picks the neighbour builder as
 * SRK.py:450 does (all pairs when n < n_grid^dim), 1 the cell-window builder
 * (updates.update_nbor_list, as populations.py:164 calls it), 2 all pairs
 * (updates.update_nbor_list_few). */
GCR_API int gcr_reference_lists(gcr_ctx *ctx, int32_t slot, int64_t n_grid, int64_t grid_window,
                        int64_t *where_is_bead, int64_t *grid_list, int64_t grid_depth1,
                        int64_t *nbor_list, int64_t nbor_depth1, int32_t mode);
/* The GPU cell table of one system after binning its current positions:
 * cell index per bead (int32 [n], device) and the grid side (host). */
GCR_API int gcr_cell_assignment(gcr_ctx *ctx, int32_t slot, int32_t *cell_of_bead, int32_t *n_cells_side);
/* Per-chain frames of a resident system: com[n_chains][dim] (device, or
 * NULL) the chain centre exactly as analysis.chain_COM computes it
 * (analysis.py:288-292: the head plus the summed separations head - x_i,
 * wrapped); phi[n_chains][2] (device, or NULL) the mean chain angle of
 * output_methods.calc_avg_phi_chain (output_methods.py:492-510) with n-fold
 * symmetry 1 and 2 (azimuth of the tangents' x, y components). */
GCR_API int gcr_chain_frames(gcr_ctx *ctx, int32_t slot, double *com, double *phi);
/* Pair correlation over chain centres, analysis.correlation_func
 * (analysis.py:203-241) with the pair function of g_of_r (kind 0, norm
 * 'all'), Cvv (1) or Cnn (2, norm 'bin'), analysis.py:243-275: bins of
 * `binsize` over [0, int(L/2) sqrt(2)) (at most 12000 bins), rows (r, value)
 * with r < L/2 written to out[max_rows][2] (host); *n_rows their number.
 * 2D systems. */
GCR_API int gcr_pair_correlation(gcr_ctx *ctx, int32_t slot, int32_t kind, double binsize, double *out,
                                 int32_t max_rows, int32_t *n_rows);
/* The neighbour list of a resident system as of its last build (no
 * counterpart in the reference, whose nbor_list gcr_reference_lists gives):
 * counts[n] (device, or NULL) partners per bead; partners[n][partners_depth]
 * (device, or NULL; partners_depth >= the context's list_depth) their bead
 * ids in ascending order (the summation order); build_pos[n][dim] (device, or NULL) the FP64
 * positions the list was built from; *entries (host, or NULL) the total. */
GCR_API int gcr_neighbour_list(gcr_ctx *ctx, int32_t slot, int32_t *counts, int32_t *partners,
                               int32_t partners_depth, double *build_pos, int64_t *entries);
/* Unwrapped positions of a resident system, out[n][dim] (device): pos + L *
 * the periodic images each bead crossed in the real updates since its
 * admission or the last gcr_reset_images -- the displacement record of the
 * mean-squared displacement (no counterpart in the reference, whose
 * analysis unwraps between saved states).  Synchronises the stream. */
GCR_API int gcr_unwrapped_positions(gcr_ctx *ctx, int32_t slot, double *out);
GCR_API int gcr_reset_images(gcr_ctx *ctx, int32_t slot);
/* Standard normals of the Philox stream the step draws: [n][2*dim] noise_vec
 * layout for one step (device out). */
GCR_API int gcr_philox_noise(int32_t dim, uint64_t seed, int64_t step, int64_t n, int32_t do_trans,
                     int32_t do_rot, double *out, void *cuda_stream);

/* ---- without device allocation ---------------------------------------- */
/* No counterpart in the reference.  The order parameters of one 2D system
 * (what gcr_order_params computes) from caller-owned device arrays --
 * tangents [n_beads][2] (FP64 for GCR_FP64, FP32 for GCR_MIXED) and chain
 * ids [n_beads] running 0..n_chains-1 in contiguous ranges -- without a
 * context and without allocating device memory: for callers that cannot
 * call cudaMalloc/cudaFree (an analysis hook sampling a system while other
 * work is queued on the device, since cudaFree waits for the whole device;
 * an application that hands out all device memory from its own pool).  Its
 * scratch is a static device array of about 1 MiB held by every GPU that
 * loads the library until the process exits, sized for at most
 * GCR_NOALLOC_MAX_CHAINS chains; more chains return GCR_ERR_CAPACITY.  The
 * first call on a device, with that device current, looks up that array's
 * device address (cudaGetSymbolAddress) and keeps it for the life of the
 * process (a cudaDeviceReset after that call is not supported).  Chain ids
 * that do not run 0..n_chains-1 as described return GCR_ERR_BAD_ARG.  Calls
 * that overlap on the GPU race on the shared scratch.  The call waits for
 * `cuda_stream` before it returns; out = [P, S, director] (host). */
#define GCR_NOALLOC_MAX_CHAINS 262144
GCR_API int gcr_order_params_noalloc(int32_t dim, int32_t precision, const void *tangent,
                                     const int32_t *chain_id, int64_t n_beads, int64_t n_chains,
                                     double out[3], void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* GCR_H */
