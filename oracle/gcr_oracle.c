/*
 * gcr_oracle.c -- CPU restatement of the gliding-collective-rotation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path and the CPU baseline timed beside it.  Nothing in the product package
 * links, loads or calls it.
 *
 * It restates, loop for loop, the reference's Numba hot path:
 *   SRK_jit                    SRK.py:13-484   (SRK2 and SRK4 branches)
 *   thread_wait                SRK.py:487-495  (-> OpenMP barrier)
 *   WCA                        forces.py:13-15
 *   inbounds_diff              forces.py:44-55
 *   central_pair_force         forces.py:57-145 (WCA rule, no active sliding)
 *   self_propel                forces.py:206-224
 *   project_updates_for_rigid_rod  updates.py:347-499
 *   calc_chain_spring_forces   forces.py:285-403 (Hookean branch)
 *   update_grid_list_mini      updates.py:502-522
 *   update_grid_list           updates.py:525-583 (overwrite / append modes)
 *   update_nbor_list           updates.py:586-669
 *   update_nbor_list_few       updates.py:672-734
 *   chunk_chain                updates.py:323-344
 *   calc_avg_phi_chain         output_methods.py:492-510
 *   polar_orderparameter       analysis.py:315-328
 *   nematic_orderparameter     analysis.py:294-313
 * and the random streams the reference consumes:
 *   MT19937 (Matsumoto & Nishimura 1998) with the 53-bit double and the
 *   Marsaglia polar Gaussian with one cached deviate -- the stream that
 *   Numba's np.random.standard_normal and numpy's RandomState produce.
 * plus the counter-based Philox4x32-10 stream (Salmon et al., SC'11) that the
 * CUDA path draws, keyed exactly as the CUDA path keys it.
 *
 * Arithmetic is IEEE double without contraction (built with
 * -ffp-contract=off); integer power follows Numba's exponentiation by
 * squaring.  Arrays use the reference's numpy layouts: float64 [N,dim],
 * int64 chain ids, grid_list int64 [n,n,nz,1+depth], nbor_list int64
 * [N,1+depth].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define GCRO_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* Random streams                                                      */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t mt[624];
    int idx;
    int has_gauss;
    double gauss;
} gcro_mt;

GCRO_EXPORT void gcro_mt_seed(gcro_mt *s, uint32_t seed)
{
    /* init_genrand of the 1998 MT19937 reference implementation */
    s->mt[0] = seed;
    for (int i = 1; i < 624; i++)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
    s->has_gauss = 0;
    s->gauss = 0.0;
}

static uint32_t mt_next(gcro_mt *s)
{
    if (s->idx >= 624) {
        for (int i = 0; i < 624; i++) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = s->mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            s->mt[i] = v;
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

static double mt_double(gcro_mt *s)
{
    /* 53-bit resolution double in [0,1) from two 32-bit draws */
    uint32_t a = mt_next(s) >> 5, b = mt_next(s) >> 6;
    return ((double)a * 67108864.0 + (double)b) / 9007199254740992.0;
}

GCRO_EXPORT double gcro_mt_normal(gcro_mt *s)
{
    /* Marsaglia polar method, second deviate cached */
    if (s->has_gauss) {
        s->has_gauss = 0;
        return s->gauss;
    }
    double x1, x2, r2;
    do {
        x1 = 2.0 * mt_double(s) - 1.0;
        x2 = 2.0 * mt_double(s) - 1.0;
        r2 = x1 * x1 + x2 * x2;
    } while (r2 >= 1.0 || r2 == 0.0);
    double f = sqrt(-2.0 * log(r2) / r2);
    s->gauss = f * x1;
    s->has_gauss = 1;
    return f * x2;
}

GCRO_EXPORT void gcro_mt_normals(uint32_t seed, int64_t n, double *out)
{
    gcro_mt s;
    gcro_mt_seed(&s, seed);
    for (int64_t i = 0; i < n; i++) out[i] = gcro_mt_normal(&s);
}

/* Philox4x32-10: round function and key schedule from Salmon, Moraes, Dror
 * and Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11). */
static void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Two standard normals from one Philox block, as the CUDA path draws them:
 * counter = (bead, step lo, step hi, stream), key = (seed lo, seed hi);
 * u1 in (0,1] and u2 in [0,1) with 53 bits each; Box-Muller. */
GCRO_EXPORT void gcro_philox_pair(uint64_t seed, uint32_t bead, int64_t step, uint32_t stream,
                                  double out[2])
{
    uint32_t ctr[4] = {bead, (uint32_t)((uint64_t)step & 0xffffffffu),
                       (uint32_t)((uint64_t)step >> 32), stream};
    uint32_t key[2] = {(uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32)};
    uint32_t r[4];
    philox4x32_10(ctr, key, r);
    const double two_m53 = 1.1102230246251565e-16; /* 2^-53 */
    uint64_t a = ((uint64_t)r[0] << 21) ^ (uint64_t)(r[1] >> 11);
    uint64_t b = ((uint64_t)r[2] << 21) ^ (uint64_t)(r[3] >> 11);
    a &= ((uint64_t)1 << 53) - 1;
    b &= ((uint64_t)1 << 53) - 1;
    double u1 = ((double)a + 1.0) * two_m53;  /* (0,1] */
    double u2 = (double)b * two_m53;          /* [0,1) */
    double rad = sqrt(-2.0 * log(u1));
    double ang = 6.283185307179586 * u2;
    out[0] = rad * cos(ang);
    out[1] = rad * sin(ang);
}

/* Two uniforms in [0, 1) for the motor decisions of (motor, bead) at a
 * stage of a step (53 bits each, as the normals above): u[0] for k_off,
 * u[1] for k_on.  Keyed Philox stands in for the reference's sequential
 * np.random.random() draws (forces.py:268, 275), which nothing seeds. */
GCRO_EXPORT void gcro_motor_uniforms(uint64_t seed, uint32_t motor, uint32_t bead, int64_t step, int stage,
                                     double u[2])
{
    uint32_t ctr[4] = {motor, bead, (uint32_t)((uint64_t)step & 0xffffffffu),
                       ((uint32_t)((uint64_t)step >> 32) & 0xffffu) | ((uint32_t)stage << 16)};
    uint32_t key[2] = {(uint32_t)(seed & 0xffffffffu) ^ 0x6d6f746fu, (uint32_t)(seed >> 32)};
    uint32_t r[4];
    philox4x32_10(ctr, key, r);
    const double two_m53 = 1.1102230246251565e-16;
    uint64_t a = (((uint64_t)r[0] << 21) ^ (uint64_t)(r[1] >> 11)) & (((uint64_t)1 << 53) - 1);
    uint64_t b = (((uint64_t)r[2] << 21) ^ (uint64_t)(r[3] >> 11)) & (((uint64_t)1 << 53) - 1);
    u[0] = (double)a * two_m53;
    u[1] = (double)b * two_m53;
}

/* Fill noise_vec [N, 2*dim] for one step from the Philox stream.
 * Translational components use streams 0..; rotational ones 2... */
GCRO_EXPORT void gcro_philox_noise(uint64_t seed, int64_t step, int dim, int64_t n,
                                   int do_trans, int do_rot, double *noise)
{
    for (int64_t b = 0; b < n; b++) {
        double z[4];
        double *row = noise + b * 2 * dim;
        if (do_trans) {
            gcro_philox_pair(seed, (uint32_t)b, step, 0u, z);
            if (dim == 3) gcro_philox_pair(seed, (uint32_t)b, step, 1u, z + 2);
            for (int i = 0; i < dim; i++) row[i] = z[i];
        }
        if (do_rot) {
            gcro_philox_pair(seed, (uint32_t)b, step, 2u, z);
            if (dim == 3) gcro_philox_pair(seed, (uint32_t)b, step, 3u, z + 2);
            for (int i = 0; i < dim; i++) row[dim + i] = z[i];
        }
    }
}

/* ------------------------------------------------------------------ */
/* Small arithmetic helpers with the reference's semantics             */
/* ------------------------------------------------------------------ */

/* Python float modulo (floor-mod, result has the sign of the divisor). */
static inline double py_mod(double x, double m)
{
    double r = fmod(x, m);
    if (r != 0.0) {
        if ((m < 0) != (r < 0)) r += m;
    } else {
        r = copysign(0.0, m);
    }
    return r;
}

/* Python float floor division (CPython float_floor_div / divmod). */
static inline double py_floordiv(double x, double m)
{
    double mod = fmod(x, m);
    double div = (x - mod) / m;
    if (mod != 0.0) {
        if ((m < 0) != (mod < 0)) div -= 1.0;
    }
    double fd;
    if (div != 0.0) {
        fd = floor(div);
        if (div - fd > 0.5) fd += 1.0;
    } else {
        fd = copysign(0.0, x / m);
    }
    return fd;
}

/* x ** (-n) by squaring, as Numba lowers integer powers. */
static inline double ipow_neg(double x, int n)
{
    double r = 1.0, a = x;
    int e = n;
    while (e) {
        if (e & 1) r *= a;
        e >>= 1;
        a *= a;
    }
    return 1.0 / r;
}

/* forces.inbounds_diff (forces.py:44-55) */
static inline double inbounds_diff(const double *a, const double *b, double hb, double L,
                                   double *out, int dim)
{
    double ds = 0.0;
    for (int i = 0; i < dim; i++) {
        out[i] = a[i] - b[i];
        if (out[i] < -hb)
            out[i] += L;
        else if (out[i] >= hb)
            out[i] -= L;
        ds += out[i] * out[i];
    }
    return ds;
}

/* ------------------------------------------------------------------ */
/* Parameters and state                                                */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t dim;
    int32_t n_threads;
    double L;
    int64_t n_beads;
    int64_t n_chains;
    /* force switches derived as SRK.py:58-97 derives them */
    int32_t calc_springs;
    int32_t calc_wca;
    int32_t self_propel;
    int32_t noise_mode;     /* 0 = MT19937 (reference RNG), 1 = injected, 2 = Philox */
    double spring[6];       /* populations.py:345-353 */
    double wca[4];          /* populations.py:48-58 */
    double active[3];       /* populations.py:355-358 */
    double D, Dr, radius;
    double rigid_rod;       /* rigid_rod_projection_factor (populations.py:325-329) */
    int64_t n_nearby;
    int64_t longest_chain_length;
    double grid_factor;
    /* time_vals, updates.py:144-146 */
    double dt, dtmax, max_dist_per_step, rk_cheat, max_dt_usable;
    int64_t steps_until_update, n_steps_update, max_steps;
    /* Philox key and the global step index of the first step of this call */
    uint64_t seed;
    int64_t step0;
    /* config.SRK_order: 2 (or 0) = SRK2, 4 = SRK4 */
    int64_t srk_order;
} gcro_params;

typedef struct {
    double *pos, *pos1, *noise, *tangent, *forces;
    int64_t *where_active;
    int64_t *where_is_bead;   /* [N,3] */
    const int64_t *chain_id;  /* [N]   */
    const double *rest_lengths; /* [n_chains] */
    int64_t *grid_list;       /* [n, n, nz, depth1] */
    int64_t n_grid, n_grid_z, grid_depth1;
    int64_t *nbor_list;       /* [N, depth1] */
    int64_t nbor_depth1;
    /* injected noise: [n_steps][N][2*dim] snapshots of noise_vec */
    const double *noise_inject;
    int64_t noise_inject_steps;
    /* MT19937 state per thread (n_threads entries) */
    gcro_mt *mt;
    /* SRK4: the force of the current stage (pop.forces_aux, populations.py:149-154) */
    double *forces_aux;
} gcro_state;

/* shared_arr row layout, SRK.py: 0 dt, 1 elapsed, 2 steps, 3 max force,
 * 4 barrier counter, 5 list-overflow flag */
typedef struct {
    double dt, dt_used_total, steps, max_forces_strength, counter, flag;
} gcro_result;

/* ------------------------------------------------------------------ */
/* Forces                                                              */
/* ------------------------------------------------------------------ */

/* forces.calc_chain_spring_forces (forces.py:285-403), Hookean branch.
 * Operates on a chain-aligned chunk [0,n) of the arrays. */
static void spring_forces(const double *pos, double *tangent_list, const int64_t *chain_id,
                          double *forces, int64_t n, double L, const double *sp,
                          const double *rest_lengths, int dim)
{
    double half_L = L / 2.0;
    int b_calc_f_bend = (sp[1] != 0.0);
    int64_t max_b1 = n - 1;
    int b_get_orientations = (sp[4] != 0.0);
    double tangents[2][3] = {{0}};
    int new_chain = 1;
    int ti = 0, tj = 1;
    int64_t ci = 0;
    double chain_a = 0.0;

    for (int64_t b1 = 0; b1 < n; b1++) {
        if (new_chain) {
            ti = 0;
            tj = 1;
            ci = chain_id[b1];
            chain_a = rest_lengths[ci];
        }
        int end_of_chain;
        if (b1 == max_b1)
            end_of_chain = 1;
        else if (chain_id[b1 + 1] != ci)
            end_of_chain = 1;
        else
            end_of_chain = 0;
        if (!end_of_chain) {
            double dist_sq = inbounds_diff(pos + b1 * dim, pos + (b1 + 1) * dim, half_L, L,
                                           tangents[ti], dim);
            if (dist_sq != 0.0) {
                double inv_dist = 1.0 / sqrt(dist_sq);
                double f_spring_mag = sp[0] * (chain_a * inv_dist - 1.0);
                for (int i = 0; i < dim; i++) {
                    double f = tangents[ti][i] * f_spring_mag;
                    forces[b1 * dim + i] += f;
                    forces[(b1 + 1) * dim + i] -= f;
                    tangents[ti][i] *= inv_dist;
                }
            }
        }
        if (b_get_orientations || b_calc_f_bend) {
            if (new_chain) {
                if (b_get_orientations)
                    for (int i = 0; i < dim; i++) tangent_list[b1 * dim + i] = tangents[ti][i];
            } else if (end_of_chain) {
                if (b_get_orientations)
                    for (int i = 0; i < dim; i++) tangent_list[b1 * dim + i] = tangents[tj][i];
            } else {
                double c = 0.0;
                for (int i = 0; i < dim; i++) c += tangents[ti][i] * tangents[tj][i];
                if (-1.0 < c && c < 1.0) {
                    if (b_calc_f_bend) {
                        double phi = acos(c);
                        if (sp[2] != 0.0) {
                            double cr = -tangents[ti][0] * tangents[tj][1] +
                                        tangents[ti][1] * tangents[tj][0];
                            double sg = (cr > 0) - (cr < 0);
                            phi += sp[2] * sg;
                        }
                        phi *= sp[1] / sqrt(1.0 - c * c);
                        for (int i = 0; i < dim; i++) {
                            double fwd = phi * (c * tangents[tj][i] - tangents[ti][i]);
                            double bwd = phi * (tangents[tj][i] - c * tangents[ti][i]);
                            forces[b1 * dim + i] += fwd + bwd;
                            forces[(b1 - 1) * dim + i] -= fwd;
                            forces[(b1 + 1) * dim + i] -= bwd;
                        }
                    }
                    if (b_get_orientations) {
                        double coeff = 1.0 / sqrt(2.0 * (1.0 + c));
                        for (int i = 0; i < dim; i++)
                            tangent_list[b1 * dim + i] = coeff * (tangents[ti][i] + tangents[tj][i]);
                    }
                } else {
                    if (b_get_orientations)
                        for (int i = 0; i < dim; i++) tangent_list[b1 * dim + i] = tangents[ti][i];
                }
            }
        }
        tj = ti;
        ti = 1 - ti;
        new_chain = end_of_chain;
    }
}

/* forces.central_pair_force (forces.py:57-145) with force_rule = forces.WCA
 * (forces.py:13-15), same population, thread chunk [start, start+n). */
static void pair_forces(int64_t start, const double *pos_chunk, const int64_t *nbor, int64_t nbd1,
                        double *forces_chunk, int64_t n, double L, const double *pos2,
                        const double *wp, double pbc_w, int dim)
{
    double half_L = L / 2.0;
    double rc_sq = wp[3] * wp[3];
    double pbc_wR = L - pbc_w;
    int64_t end = start + n;
    double seps[3];
    for (int64_t b1 = 0; b1 < n; b1++) {
        int flags[3];
        for (int i = 0; i < dim; i++) {
            double x = pos_chunk[b1 * dim + i];
            flags[i] = !(pbc_w <= x && x < pbc_wR);
        }
        int64_t true_b1 = b1 + start;
        const int64_t *row = nbor + b1 * nbd1;
        for (int64_t j = 0; j < row[0]; j++) {
            int64_t b2 = row[1 + j];
            if (true_b1 <= b2 && b2 < end) continue;
            int same_thread = (true_b1 > b2 && b2 >= start);
            double ds = 0.0;
            for (int i = 0; i < dim; i++) {
                double sep = pos2[b2 * dim + i] - pos_chunk[b1 * dim + i];
                if (flags[i]) {
                    if (sep < -half_L)
                        sep += L;
                    else if (sep >= half_L)
                        sep -= L;
                }
                seps[i] = sep;
                ds += sep * sep;
            }
            if (0.0 < ds && ds <= rc_sq) {
                if (wp[2] != 0.0) {
                    double mag = sqrt(ds);
                    double nm = mag + wp[2];
                    if (nm < 0.0) nm = 0.0;
                    double rescale = nm / mag;
                    for (int i = 0; i < dim; i++) seps[i] *= rescale;
                    ds = nm * nm;
                }
                double coeff = ipow_neg(ds, 4) * (wp[0] - wp[1] * ipow_neg(ds, 3));
                if (same_thread) {
                    int64_t b2l = b2 - start;
                    for (int i = 0; i < dim; i++) {
                        double f = seps[i] * coeff;
                        forces_chunk[b1 * dim + i] += f;
                        forces_chunk[b2l * dim + i] -= f;
                    }
                } else {
                    for (int i = 0; i < dim; i++) forces_chunk[b1 * dim + i] += seps[i] * coeff;
                }
            }
        }
    }
}

/* forces.self_propel (forces.py:206-224) */
static void self_propel(double *forces, const double *tangent, int64_t n, const double *ap, int dim)
{
    double v0 = ap[0], ang = ap[2];
    if (ang == 0.0 || dim != 2) {
        for (int64_t b = 0; b < n; b++)
            for (int i = 0; i < dim; i++) forces[b * dim + i] += v0 * tangent[b * dim + i];
    } else {
        double sn = sin(ang), cs = cos(ang);
        for (int64_t b = 0; b < n; b++) {
            double tx = tangent[b * dim], ty = tangent[b * dim + 1];
            forces[b * dim] += v0 * (cs * tx - sn * ty);
            forces[b * dim + 1] += v0 * (sn * tx + cs * ty);
        }
    }
}

/* Public single-call wrappers for unit tests (whole array = one chunk). */
GCRO_EXPORT void gcro_spring_forces(const double *pos, double *tangent_list, const int64_t *chain_id,
                                    double *forces, int64_t n, double L, const double *spring_params,
                                    const double *rest_lengths, int dim)
{
    spring_forces(pos, tangent_list, chain_id, forces, n, L, spring_params, rest_lengths, dim);
}

GCRO_EXPORT void gcro_pair_forces(const double *pos, const int64_t *nbor, int64_t nbd1, double *forces,
                                  int64_t n, double L, const double *wca_params, double pbc_w, int dim)
{
    pair_forces(0, pos, nbor, nbd1, forces, n, L, pos, wca_params, pbc_w, dim);
}

GCRO_EXPORT void gcro_self_propel(double *forces, const double *tangent, int64_t n,
                                  const double *active_params, int dim)
{
    self_propel(forces, tangent, n, active_params, dim);
}

/* ------------------------------------------------------------------ */
/* Cell and neighbour lists                                            */
/* ------------------------------------------------------------------ */

#define GL(g, gx, gy, gz, k) \
    (g)->grid_list[((((gx) * (g)->n_grid + (gy)) * (g)->n_grid_z + (gz)) * (g)->grid_depth1) + (k)]

/* updates.update_grid_list_mini (updates.py:502-522) over all beads of the
 * population for the x-slab [start_gx, end_gx).  Returns 1 on success. */
static int grid_list_mini(gcro_state *g, int64_t n_beads, int64_t start_gx, int64_t end_gx)
{
    int64_t depth_less_one = g->grid_depth1 - 2;
    for (int64_t gx = start_gx; gx < end_gx; gx++)
        for (int64_t gy = 0; gy < g->n_grid; gy++)
            for (int64_t gz = 0; gz < g->n_grid_z; gz++) GL(g, gx, gy, gz, 0) = 0;
    for (int64_t bi = 0; bi < n_beads; bi++) {
        const int64_t *w = g->where_is_bead + bi * 3;
        /* A bead at exactly x == L (floor-mod of a tiny negative number)
         * has cell index n_grid; the reference then writes outside its
         * array.  Such a bead is left out of every cell here. */
        if (start_gx <= w[0] && w[0] < end_gx && w[1] >= 0 && w[1] < g->n_grid && w[2] >= 0 &&
            w[2] < g->n_grid_z) {
            int64_t *cell = &GL(g, w[0], w[1], w[2], 0);
            cell[0] += 1;
            if (cell[0] < depth_less_one)
                cell[cell[0]] = bi;
            else
                return 0;
        }
    }
    return 1;
}

/* updates.update_grid_list (updates.py:525-583), as populations.py:104-112
 * calls it (overwrite / append modes and the incremental mode). */
GCRO_EXPORT int gcro_update_grid_list(gcro_state *g, const double *pos, int64_t n, double L, int dim,
                                      int append_mode, int overwrite, int64_t start)
{
    int64_t ng = g->n_grid, ngz = g->n_grid_z;
    double spacing = L / (double)ng;
    for (int64_t bi = 0; bi < n; bi++) {
        for (int i = 0; i < dim; i++)
            g->where_is_bead[bi * 3 + i] = (int64_t)py_floordiv(pos[bi * dim + i], spacing);
        if (dim == 2) g->where_is_bead[bi * 3 + 2] = 0;
    }
    if (append_mode || overwrite) {
        for (int64_t bi = 0; bi < n; bi++) g->where_is_bead[bi * 3] = -g->where_is_bead[bi * 3] - 1;
        if (overwrite)
            for (int64_t c = 0; c < ng * ng * ngz; c++) g->grid_list[c * g->grid_depth1] = 0;
    } else {
        start = 0;
        for (int64_t gx = 0; gx < ng; gx++)
            for (int64_t gy = 0; gy < ng; gy++)
                for (int64_t gz = 0; gz < ngz; gz++) {
                    int64_t *cell = &GL(g, gx, gy, gz, 0);
                    int64_t gxyz[3] = {gx, gy, gz};
                    int64_t num_here_now = 0;
                    int64_t cnt = cell[0];
                    for (int64_t k = 0; k < cnt; k++) {
                        int64_t bi = cell[1 + k];
                        int moved = 0;
                        for (int i = 0; i < dim; i++)
                            if (g->where_is_bead[bi * 3 + i] != gxyz[i]) {
                                moved = 1;
                                break;
                            }
                        if (moved) {
                            cell[1 + num_here_now] = bi;
                            num_here_now++;
                        } else {
                            g->where_is_bead[bi * 3] = -g->where_is_bead[bi * 3] - 1;
                        }
                    }
                    cell[0] = num_here_now;
                }
    }
    int64_t depth = g->grid_depth1;
    for (int64_t bi = 0; bi < n; bi++) {
        int64_t *w = g->where_is_bead + bi * 3;
        if (w[0] < 0) {
            w[0] = -w[0] - 1;
            if (w[0] >= ng || w[1] < 0 || w[1] >= ng || w[2] < 0 || w[2] >= ngz) continue;
            int64_t *cell = &GL(g, w[0], w[1], w[2], 0);
            if (cell[0] < depth - 2)
                cell[1 + cell[0]] = start + bi;
            else
                return 0;
            cell[0] += 1;
        }
    }
    return 1;
}

/* updates.update_nbor_list (updates.py:586-669) for a chunk starting at
 * `start` (same population).  Returns 1 on success, 0 on overflow. */
static int nbor_list_cells(int64_t start, const double *pos1, const int64_t *wib1, int64_t *nb,
                           int64_t nbd1, int64_t n, const int64_t *chain_id, const double *pos2,
                           const gcro_state *g, int64_t n_nearby, double L, int64_t gw, int dim)
{
    int b3d = (dim == 3);
    int64_t ng = g->n_grid;
    double hgrid = (double)gw * L / (double)ng;
    double max_dist_sq = hgrid * hgrid;
    double half_L = L / 2.0;
    for (int64_t b1 = 0; b1 < n; b1++) nb[b1 * nbd1] = 0;
    int64_t dg_start = -(gw < ng / 2 ? gw : ng / 2);
    int64_t dg_end = (1 + gw < ng + dg_start) ? 1 + gw : ng + dg_start;
    for (int64_t b1 = 0; b1 < n; b1++) {
        int64_t b1u = b1 + start;
        int flags[3];
        for (int i = 0; i < dim; i++) {
            int64_t w = wib1[b1 * 3 + i];
            flags[i] = (w < gw + 1) || (w >= ng - (gw + 1));
        }
        int64_t gy0 = dg_start + wib1[b1 * 3 + 1], gy1 = wib1[b1 * 3 + 1] + dg_end;
        int64_t gz0, gz1;
        if (b3d) {
            gz0 = dg_start + wib1[b1 * 3 + 2];
            gz1 = wib1[b1 * 3 + 2] + dg_end;
        } else {
            gz0 = 0;
            gz1 = 1;
        }
        for (int64_t gx2r = dg_start + wib1[b1 * 3]; gx2r < wib1[b1 * 3] + dg_end; gx2r++) {
            int64_t gx2 = gx2r;
            if (flags[0]) gx2 = ((gx2 % ng) + ng) % ng;
            for (int64_t gy2r = gy0; gy2r < gy1; gy2r++) {
                int64_t gy2 = gy2r;
                if (flags[1]) gy2 = ((gy2 % ng) + ng) % ng;
                for (int64_t gz2r = gz0; gz2r < gz1; gz2r++) {
                    int64_t gz2 = gz2r;
                    if (b3d && flags[2]) gz2 = ((gz2 % ng) + ng) % ng;
                    const int64_t *cell = &g->grid_list[(((gx2 * ng + gy2) * g->n_grid_z + gz2) * g->grid_depth1)];
                    int64_t cnt = cell[0];
                    for (int64_t k = 0; k < cnt; k++) {
                        int64_t b2 = cell[1 + k];
                        if (chain_id[b1u] == chain_id[b2]) {
                            if (n_nearby < 0) continue;
                            int64_t d = b1u - b2;
                            if (d < 0) d = -d;
                            if (d <= n_nearby) continue;
                        }
                        double dist_sq = 0.0;
                        for (int i = 0; i < dim; i++) {
                            double sep = pos2[b2 * dim + i] - pos1[b1 * dim + i];
                            if (flags[i]) {
                                if (sep < -half_L)
                                    sep += L;
                                else if (sep >= half_L)
                                    sep -= L;
                            }
                            dist_sq += sep * sep;
                        }
                        if (dist_sq <= max_dist_sq) {
                            int64_t *row = nb + b1 * nbd1;
                            if (row[0] + 1 >= nbd1) {
                                row[0] = -1;
                                return 0;
                            }
                            row[0] += 1;
                            row[row[0]] = b2;
                        }
                    }
                }
            }
        }
    }
    return 1;
}

/* updates.update_nbor_list_few (updates.py:672-734) */
static int nbor_list_few(int64_t start, const double *pos1, const int64_t *wib1, int64_t *nb,
                         int64_t nbd1, int64_t n, const int64_t *chain_id, const double *pos2,
                         const int64_t *wib2, int64_t n2, int64_t n_nearby, double L, int64_t ng,
                         int64_t gw, int dim)
{
    double hgrid = (double)gw * L / (double)ng;
    double max_dist_sq = hgrid * hgrid;
    double half_L = L / 2.0;
    double half_ng = (double)ng / 2.0;
    for (int64_t b1 = 0; b1 < n; b1++) nb[b1 * nbd1] = 0;
    for (int64_t b1 = 0; b1 < n; b1++) {
        for (int64_t b2 = 0; b2 < n2; b2++) {
            int use = 1;
            for (int i = 0; i < dim; i++) {
                double dg = (double)(wib2[b2 * 3 + i] - wib1[b1 * 3 + i]);
                if (dg < -half_ng)
                    dg += (double)ng;
                else if (dg >= half_ng)
                    dg -= (double)ng;
                if (fabs(dg) > (double)gw) {
                    use = 0;
                    break;
                }
            }
            if (!use) continue;
            int64_t b1u = b1 + start;
            if (chain_id[b1u] == chain_id[b2]) {
                if (n_nearby < 0) continue;
                int64_t d = b1u - b2;
                if (d < 0) d = -d;
                if (d <= n_nearby) continue;
            }
            double dist_sq = 0.0;
            for (int i = 0; i < dim; i++) {
                double sep = pos2[b2 * dim + i] - pos1[b1 * dim + i];
                if (sep < -half_L)
                    sep += L;
                else if (sep >= half_L)
                    sep -= L;
                dist_sq += sep * sep;
            }
            if (dist_sq <= max_dist_sq) {
                int64_t *row = nb + b1 * nbd1;
                if (row[0] + 1 >= nbd1) {
                    row[0] = -1;
                    return 0;
                }
                row[0] += 1;
                row[row[0]] = b2;
            }
        }
    }
    return 1;
}

/* populations.update_nbor_list_with_pop2 core (populations.py:156-180) for
 * the whole population: one updates.update_nbor_list call.  Returns 1 on
 * success; on overflow the caller doubles the depth and calls again. */
GCRO_EXPORT int gcro_update_nbor_list(gcro_state *g, const double *pos, int64_t n, double L,
                                      int64_t n_nearby, int64_t gw, int dim)
{
    return nbor_list_cells(0, pos, g->where_is_bead, g->nbor_list, g->nbor_depth1, n, g->chain_id, pos,
                           g, n_nearby, L, gw, dim);
}

GCRO_EXPORT int gcro_update_nbor_list_few(gcro_state *g, const double *pos, int64_t n, double L,
                                          int64_t n_nearby, int64_t gw, int dim)
{
    return nbor_list_few(0, pos, g->where_is_bead, g->nbor_list, g->nbor_depth1, n, g->chain_id, pos,
                         g->where_is_bead, n, n_nearby, L, g->n_grid, gw, dim);
}

/* ------------------------------------------------------------------ */
/* updates.chunk_chain (updates.py:323-344)                            */
/* ------------------------------------------------------------------ */

GCRO_EXPORT int gcro_chunk_chain(int64_t n_threads, int64_t total, const int64_t *chain_id,
                                 int64_t *split /* [n_threads-1] */)
{
    int64_t chunklen = (total + n_threads - 1) / n_threads;
    int64_t first = 0;
    int64_t sii = 0;
    while (first < total && sii < n_threads - 1) {
        if (first > 0) {
            split[sii] = first;
            sii++;
        }
        int64_t test = (sii + 1) * chunklen - 1;
        if (test < first) test = first;
        if (test > total - 1) test = total - 1;
        int64_t last_ci = chain_id[test];
        while (test < total) {
            if (chain_id[test] != last_ci) break;
            test++;
        }
        first = test;
    }
    return (int)sii; /* entries of split that were set */
}

/* ------------------------------------------------------------------ */
/* SRK.SRK_jit (SRK.py:13-484), SRK2, one population                   */
/* ------------------------------------------------------------------ */

/* updates.project_updates_for_rigid_rod (updates.py:347-499) on one
 * thread's chunk of n beads (chains are contiguous, sorted bead ranges, as
 * the reference's phonebook lists them): each chain's update (forces over
 * radius plus noise) is blended with the translation and rotation a rigid
 * rod of the chain's rest length would see, and the chain's current
 * deviation from that rod is removed.  rtn = (prev + update) mod L.  The
 * arithmetic follows the reference expression by expression, including its
 * 2D per-component torque and its 3D rotation term, which carries no
 * distance factor.  A one-bead chain in 3D (moment of inertia 0) gets no
 * rotation term; the reference divides by zero there. */
static void project_rigid(double *rtn, const double *prev, const double *F, const double *noise, int64_t n,
                          const int64_t *chain_id, const double *rest_lengths, double pf, double L, double dt,
                          double D, double radius, int dim, double *upd, double *ool, double *dist)
{
    const double half = 0.5 * L;
    const double dt_over_r = dt / radius;
    const double s2 = sqrt(2.0 * D * dt);
    int64_t b0 = 0;
    while (b0 < n) {
        int64_t b1 = b0 + 1;
        while (b1 < n && chain_id[b1] == chain_id[b0]) b1++;
        const int64_t len = b1 - b0;
        const double rest = rest_lengths[chain_id[b0]];
        const double half_clm1 = (double)(len - 1) / 2.0;
        double inertia = 0.0;
        for (int64_t k = 0; k < len; k++) dist[k] = rest * ((double)k - half_clm1);
        for (int64_t k = 0; k < len; k++)
            for (int i = 0; i < dim; i++) inertia += dist[k] * dist[k];
        for (int64_t k = 0; k < len; k++)
            for (int i = 0; i < dim; i++) {
                double u = dt_over_r * F[(b0 + k) * dim + i];
                if (s2 != 0.0) u += s2 * noise[(b0 + k) * 2 * dim + i];
                upd[k * dim + i] = u;
            }
        double mean[3] = {0.0, 0.0, 0.0}, com[3] = {0.0, 0.0, 0.0}, rh[3] = {0.0, 0.0, 0.0};
        for (int64_t k = 0; k < len; k++)
            for (int i = 0; i < dim; i++) mean[i] += upd[k * dim + i];
        for (int i = 0; i < dim; i++) mean[i] /= (double)len;
        double r_mag = 0.0;
        for (int64_t k = 0; k < len; k++)
            for (int i = 0; i < dim; i++) {
                double sep = prev[(b0 + k) * dim + i] - prev[b0 * dim + i];
                if (sep < -half)
                    sep += L;
                else if (sep > half)
                    sep -= L;
                com[i] += sep;
                if (k == len - 1) {
                    rh[i] = sep;
                    r_mag += sep * sep;
                }
            }
        for (int i = 0; i < dim; i++) com[i] = py_mod(prev[b0 * dim + i] + com[i] / (double)len, L);
        if (r_mag > 0) {
            r_mag = sqrt(r_mag);
            for (int i = 0; i < dim; i++) rh[i] /= r_mag;
        }
        for (int64_t k = 0; k < len; k++)
            for (int i = 0; i < dim; i++) {
                double sep = prev[(b0 + k) * dim + i] - (com[i] + rh[i] * dist[k]);
                if (sep < -half)
                    sep += L;
                else if (sep >= half)
                    sep -= L;
                ool[k * dim + i] = sep;
            }
        const double keep = 1. - pf;
        if (dim == 2) {
            double tq[2] = {0.0, 0.0};
            for (int64_t k = 0; k < len; k++)
                for (int i = 0; i < 2; i++) tq[i] += (double)(2 * i - 1) * rh[1 - i] * upd[k * 2 + i] * dist[k];
            if (inertia != 0)
                for (int i = 0; i < 2; i++) tq[i] /= inertia;
            for (int64_t k = 0; k < len; k++)
                for (int i = 0; i < 2; i++) {
                    double u = upd[k * 2 + i] * keep;
                    u += pf * (-ool[k * 2 + i] + mean[i] + (tq[i] * dist[k] * (double)(2 * i - 1) * rh[1 - i]));
                    rtn[(b0 + k) * 2 + i] = py_mod(prev[(b0 + k) * 2 + i] + u, L);
                }
        } else {
            double tq[3] = {0.0, 0.0, 0.0};
            for (int64_t k = 0; k < len; k++) {
                const double *u = upd + k * 3;
                tq[0] += rh[1] * u[2] - rh[2] * u[1];
                tq[1] += rh[2] * u[0] - rh[0] * u[2];
                tq[2] += rh[0] * u[1] - rh[1] * u[0];
            }
            for (int i = 0; i < 3; i++) tq[i] = r_mag * tq[i];
            const double q = inertia != 0 ? r_mag / inertia : 0.0;
            double rot[3];
            rot[0] = q * (tq[1] * rh[2] - tq[2] * rh[1]);
            rot[1] = q * (tq[2] * rh[0] - tq[0] * rh[2]);
            rot[2] = q * (tq[0] * rh[1] - tq[1] * rh[0]);
            for (int64_t k = 0; k < len; k++)
                for (int i = 0; i < 3; i++) {
                    double u = upd[k * 3 + i] * keep;
                    u += pf * (-ool[k * 3 + i] + mean[i] + rot[i]);
                    rtn[(b0 + k) * 3 + i] = py_mod(prev[(b0 + k) * 3 + i] + u, L);
                }
        }
        b0 = b1;
    }
}

/* the projection on its own, for the golden vectors of its direct calls */
GCRO_EXPORT void gcro_project_rigid(double *rtn, const double *prev, const double *F, const double *noise, int64_t n,
                                    const int64_t *chain_id, const double *rest_lengths, double pf, double L,
                                    double dt, double D, double radius, int dim)
{
    double *scratch = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * 7);
    project_rigid(rtn, prev, F, noise, n, chain_id, rest_lengths, pf, L, dt, D, radius, dim, scratch,
                  scratch + 3 * (n > 0 ? n : 1), scratch + 6 * (n > 0 ? n : 1));
    free(scratch);
}

static double draw_normal(gcro_state *st, int tid)
{
    return gcro_mt_normal(&st->mt[tid]);
}

GCRO_EXPORT int gcro_srk2_run(const gcro_params *p, gcro_state *st, gcro_result *out)
{
    const int dim = p->dim;
    const int64_t N = p->n_beads;
    const double L = p->L;
    int T = p->n_threads > 0 ? p->n_threads : 1;
    /* SRK.py:364: the projection replaces the plain update */
    const int rigid = p->rigid_rod != 0.0 && p->longest_chain_length > 2;
    const int srk4 = p->srk_order == 4;
    const int n_stages = srk4 ? 4 : 2;
    if (srk4 && !st->forces_aux) return -2;

    /* chunk boundaries: chain-aligned (updates.py:192-199, 323-344) */
    int64_t *bounds = (int64_t *)malloc(sizeof(int64_t) * (T + 1));
    {
        bounds[0] = 0;
        if (T > 1) {
            int64_t *split = (int64_t *)calloc((size_t)(T - 1), sizeof(int64_t));
            gcro_chunk_chain(T, N, st->chain_id, split);
            /* numpy.array_split with these indices (unset entries are the
             * uninitialised tail of np.empty in the reference; here they
             * are left at the array end) */
            for (int t = 0; t < T - 1; t++) bounds[t + 1] = split[t] > 0 ? split[t] : N;
            free(split);
        }
        bounds[T] = N;
        for (int t = 1; t <= T; t++)
            if (bounds[t] < bounds[t - 1]) bounds[t] = bounds[t - 1];
    }
    double (*shared)[6] = calloc((size_t)T, sizeof(double[6]));
    for (int t = 0; t < T; t++) shared[t][0] = p->dt;

    int64_t ng = st->n_grid;
    double grid_spacing = L / (double)ng;
    double nbor_length_scale = p->calc_wca ? p->wca[3] : 0.0;
    int64_t grid_window = (int64_t)ceil(p->grid_factor * nbor_length_scale / grid_spacing);
    if (grid_window < 1) grid_window = 1;
    double pbc_width = (double)grid_window * L / (double)ng;
    int64_t n_pow = 1;
    for (int i = 0; i < dim; i++) n_pow *= ng;
    int use_few = (N < n_pow);
    int b_get_orientations = p->calc_springs ? (p->spring[4] != 0.0) : 0;
    int64_t inject_step = 0;
    int rc = 0;

#pragma omp parallel num_threads(T)
    {
        int t = omp_get_thread_num();
        int64_t s0 = bounds[t], s1 = bounds[t + 1], n = s1 - s0;
        double *pos = st->pos + s0 * dim, *pos1 = st->pos1 + s0 * dim;
        double *noise = st->noise + s0 * 2 * dim, *tan = st->tangent + s0 * dim;
        double *F = st->forces + s0 * dim;
        double *Fa = srk4 ? st->forces_aux + s0 * dim : NULL;
        int64_t *nb = st->nbor_list + s0 * st->nbor_depth1;
        int64_t *wib = st->where_is_bead + s0 * 3;
        int64_t gchunk = (ng + T - 1) / T;
        int64_t start_gx = t * gchunk;
        int64_t end_gx = (t + 1) * gchunk < ng ? (t + 1) * gchunk : ng;
        double dt = p->dt;
        double dt_for_update = dt;
        int64_t steps_until = p->steps_until_update;
        double *rscratch = rigid ? (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * 7) : NULL;
        shared[t][4] = 0;

        while ((shared[t][2] < (double)p->max_steps || p->max_steps < 0) &&
               (shared[t][1] < p->max_dt_usable || p->max_dt_usable < 0) && shared[t][5] >= 0) {
            int64_t local_step = (int64_t)shared[t][2];
            for (int64_t b = 0; b < n; b++) st->where_active[s0 + b] = -1;
            /* noise: SRK.py:134-142 */
            if (p->noise_mode == 0) {
                if (p->D > 0)
                    for (int64_t b = 0; b < n; b++)
                        for (int i = 0; i < dim; i++) noise[b * 2 * dim + i] = draw_normal(st, t);
                if (p->Dr > 0)
                    for (int64_t b = 0; b < n; b++)
                        for (int i = dim; i < 2 * dim; i++) noise[b * 2 * dim + i] = draw_normal(st, t);
            } else if (p->noise_mode == 1) {
                int64_t k = local_step < st->noise_inject_steps ? local_step : st->noise_inject_steps - 1;
                const double *src = st->noise_inject + (k * N + s0) * 2 * dim;
                for (int64_t b = 0; b < n * 2 * dim; b++) noise[b] = src[b];
            } else {
                for (int64_t b = 0; b < n; b++) {
                    double z[4];
                    double *row = noise + b * 2 * dim;
                    int64_t gs = p->step0 + local_step;
                    if (p->D > 0) {
                        gcro_philox_pair(p->seed, (uint32_t)(s0 + b), gs, 0u, z);
                        if (dim == 3) gcro_philox_pair(p->seed, (uint32_t)(s0 + b), gs, 1u, z + 2);
                        for (int i = 0; i < dim; i++) row[i] = z[i];
                    }
                    if (p->Dr > 0) {
                        gcro_philox_pair(p->seed, (uint32_t)(s0 + b), gs, 2u, z);
                        if (dim == 3) gcro_philox_pair(p->seed, (uint32_t)(s0 + b), gs, 3u, z + 2);
                        for (int i = 0; i < dim; i++) row[dim + i] = z[i];
                    }
                }
            }
            /* SRK.py:144-160: the forces of SRK2 (both stages) or of the
             * SRK4 stages are wiped */
            for (int64_t b = 0; b < n * dim; b++) (srk4 ? Fa : F)[b] = 0.0;
            shared[t][5] = 0;

            for (int stage = 0; stage < n_stages; stage++) {
                /* SRK.py:166-215: where forces are taken and updates written */
                double *X = stage == 0 ? pos : pos1;
                double *Xfull = stage == 0 ? st->pos : st->pos1;
                double *W = srk4 ? (stage == 3 ? pos : pos1) : (stage == 0 ? pos1 : pos);
                double pref = srk4 ? 1.0 : (stage == 0 ? 1.0 : 0.5);
                double rescale = stage <= 1 ? 0.5 : 1.0;
                double *Fs = srk4 ? Fa : F;  /* write_to_forces */
                if (srk4 && stage > 0)
                    for (int64_t b = 0; b < n * dim; b++) Fa[b] = 0.0;
#pragma omp barrier
                if (p->calc_springs)
                    spring_forces(X, tan, st->chain_id + s0, Fs, n, L, p->spring, st->rest_lengths, dim);
#pragma omp barrier
                if (p->calc_wca)
                    pair_forces(s0, X, nb, st->nbor_depth1, Fs, n, L, Xfull, p->wca, pbc_width, dim);
                if (p->self_propel) self_propel(Fs, tan, n, p->active, dim);
                if (srk4) {
                    /* SRK.py:296-321: weighted sum of the four stage forces */
                    const double mult = (stage == 0 || stage == 3) ? 1. / 6. : 1. / 3.;
                    if (stage == 0)
                        for (int64_t b = 0; b < n * dim; b++) F[b] = Fa[b] * mult;
                    else
                        for (int64_t b = 0; b < n * dim; b++) F[b] += Fa[b] * mult;
                }
                if (stage == n_stages - 1) {
                    shared[t][3] = sqrt(2.0 * p->D);
                    if (n > 0) {
                        double m = -1.0;
                        for (int64_t b = 0; b < n; b++) {
                            double s = 0.0;
                            for (int i = 0; i < dim; i++) s += F[b * dim + i] * F[b * dim + i];
                            if (s > m) m = s;
                        }
                        shared[t][3] += pref * sqrt(m) / p->radius;
                    }
                    shared[t][2] += 1;
                }
#pragma omp barrier
                if (stage == n_stages - 1) {
                    double mfs = shared[0][3];
                    for (int u = 1; u < T; u++)
                        if (shared[u][3] > mfs) mfs = shared[u][3];
                    if (mfs == 0.0)
                        dt = p->dtmax;
                    else {
                        double c = p->max_dist_per_step / mfs;
                        dt = p->dtmax < c ? p->dtmax : c;
                    }
                    double dt_used = p->rk_cheat * dt;
                    if (p->max_dt_usable > 0) {
                        double lim = p->max_dt_usable - shared[t][1];
                        if (lim < dt_used) dt_used = lim;
                    }
                    shared[t][0] = dt;
                    shared[t][1] += dt_used;
                    dt_for_update = dt_used;
                } else {
                    dt_for_update = dt;
                }
                /* SRK.py:355-362; the SRK4 real update uses the weighted sum */
                double dt_eff = srk4 ? dt_for_update * rescale * pref : dt_for_update * pref;
                double s2 = sqrt(2.0 * dt_for_update * p->D);
                const double *Fu = (srk4 && stage < 3) ? Fa : F;
                if (n > 0 && rigid) {
                    /* read at check_force_at_pos: pos in the first stage, pos1
                     * after it (SRK.py:166-215, 365-371) */
                    project_rigid(W, X, Fu, noise, n, st->chain_id + s0, st->rest_lengths, p->rigid_rod, L, dt_eff,
                                  p->D, p->radius, dim, rscratch, rscratch + 3 * n, rscratch + 6 * n);
                } else if (n > 0) {
                    dt_eff /= p->radius;
                    for (int64_t b = 0; b < n; b++)
                        for (int i = 0; i < dim; i++) {
                            double tmp = pos[b * dim + i] + dt_eff * Fu[b * dim + i];
                            if (s2 != 0.0) tmp += s2 * noise[b * 2 * dim + i];
                            W[b * dim + i] = py_mod(tmp, L);
                        }
                }
            }
            /* rotational diffusion: SRK.py:399-423 */
            if (p->Dr > 0 && !b_get_orientations) {
                double sq = sqrt(2.0 * dt_for_update * p->Dr) * 3.141592653589793;
                for (int64_t b = 0; b < n; b++) {
                    double *xr = noise + b * 2 * dim + dim;
                    double *tb = tan + b * dim;
                    double proj = 0.0;
                    for (int i = 0; i < dim; i++) proj += xr[i] * tb[i];
                    for (int i = 0; i < dim; i++) xr[i] -= proj * tb[i];
                    double mag = 0.0;
                    for (int i = 0; i < dim; i++) {
                        double v = tb[i] + sq * xr[i];
                        mag += v * v;
                        tb[i] = v;
                    }
                    mag = sqrt(mag);
                    for (int i = 0; i < dim; i++) tb[i] /= mag;
                }
            }
            /* periodic rebuild: SRK.py:428-484 */
            if (shared[t][2] >= (double)steps_until) {
                for (int64_t b = 0; b < n; b++)
                    for (int i = 0; i < dim; i++)
                        wib[b * 3 + i] = (int64_t)py_floordiv(pos[b * dim + i], grid_spacing);
#pragma omp barrier
                for (int ii = 0; ii < 2; ii++) {
                    int success = 1;
                    if (ii == 0) {
                        success = grid_list_mini(st, N, start_gx, end_gx);
                    } else if (n > 0) {
                        if (use_few)
                            success = nbor_list_few(s0, pos, wib, nb, st->nbor_depth1, n, st->chain_id,
                                                    st->pos, st->where_is_bead, N, p->n_nearby, L, ng,
                                                    grid_window, dim);
                        else
                            success = nbor_list_cells(s0, pos, wib, nb, st->nbor_depth1, n, st->chain_id,
                                                      st->pos, st, p->n_nearby, L, grid_window, dim);
                    }
                    if (!success) shared[t][5] = -ii;
#pragma omp barrier
                    for (int u = 0; u < T; u++)
                        if (shared[u][5] < 0) shared[t][5] = shared[u][5];
#pragma omp barrier
                }
                steps_until += p->n_steps_update;
            }
            (void)inject_step;
        }
        free(rscratch);
    }
    out->dt = shared[0][0];
    out->dt_used_total = shared[0][1];
    out->steps = shared[0][2];
    out->max_forces_strength = shared[0][3];
    out->counter = shared[0][4];
    out->flag = shared[0][5];
    free(shared);
    free(bounds);
    return rc;
}

/* ------------------------------------------------------------------ */
/* Several populations in one box: updates.SRK2_force_calc over a list */
/* of populations (updates.py:146-247) with the cross-population pair  */
/* forces of the SRK loop (SRK.py:229-245, 287-294), SRK2, one thread  */
/* per population.                                                     */
/* ------------------------------------------------------------------ */

/* forces.central_pair_force with rule forces.WCA (forces.py:13-15, 57-145)
 * between population P (beads XP) and population Q (beads XQ), restated
 * over all pairs: bead b of P gets the force of every bead j of Q within
 * r_cut, in ascending j.  same != 0 (Q is P): b itself and the beads of its
 * chain within n_nearby of it (the whole chain for n_nearby < 0) are
 * excluded, as update_nbor_list excludes them (updates.py:586-669).  The
 * reference walks a Verlet list built from cells: the same pairs while the
 * list is fresh, summed in the list's order. */
static void pair_forces_all(const double *XP, int64_t nP, const int64_t *chainP, int64_t n_nearby,
                            const double *XQ, int64_t nQ, int same, const double *wp, double L, int dim,
                            double *F)
{
    const double half_L = L / 2.0, rc_sq = wp[3] * wp[3];
    double seps[3];
    for (int64_t b = 0; b < nP; b++) {
        for (int64_t j = 0; j < nQ; j++) {
            if (same) {
                if (j == b) continue;
                if (chainP[j] == chainP[b]) {
                    int64_t d = j > b ? j - b : b - j;
                    if (n_nearby < 0 || d <= n_nearby) continue;
                }
            }
            double ds = 0.0;
            for (int i = 0; i < dim; i++) {
                double sep = XQ[j * dim + i] - XP[b * dim + i];
                if (sep < -half_L)
                    sep += L;
                else if (sep >= half_L)
                    sep -= L;
                seps[i] = sep;
                ds += sep * sep;
            }
            if (0.0 < ds && ds <= rc_sq) {
                if (wp[2] != 0.0) {
                    double mag = sqrt(ds);
                    double nm = mag + wp[2];
                    if (nm < 0.0) nm = 0.0;
                    double rescale = nm / mag;
                    for (int i = 0; i < dim; i++) seps[i] *= rescale;
                    ds = nm * nm;
                }
                double coeff = ipow_neg(ds, 4) * (wp[0] - wp[1] * ipow_neg(ds, 3));
                for (int i = 0; i < dim; i++) F[b * dim + i] += seps[i] * coeff;
            }
        }
    }
}

GCRO_EXPORT void gcro_pair_forces_all(const double *XP, int64_t nP, const int64_t *chainP, int64_t n_nearby,
                                      const double *XQ, int64_t nQ, int same, const double *wp, double L, int dim,
                                      double *F)
{
    pair_forces_all(XP, nP, chainP, n_nearby, XQ, nQ, same, wp, L, dim, F);
}

/* ------------------------------------------------------------------ */
/* Motors: forces.calc_motor_push (forces.py:248-283), the motor        */
/* parameters of Chain_Collection.interactions (populations.py:276-287) */
/* and the diffusion of Motor_Population (SRK.py:389-395)                */
/* ------------------------------------------------------------------ */

/* params = [motor_max_dist_sq, b_one_motor_per_bead, imparts_force, k_on,
 * k_off].  The reference's loop as written: beads in order, each bead's
 * motor neighbours in its list's order (nbor rows [count, ids...]); an
 * attached motor stays with probability 1 - k_off (and then adds nothing),
 * else it detaches -- whichever bead it was attached to, the count of the
 * bead that drew is decremented -- and a free motor attaches with
 * probability k_on when within motor_max_dist, adding imparts_force times
 * the bead's tangent.  b_one_motor_per_bead ends the inner loop's body with
 * `continue` and so changes nothing.  Draws come from the MT19937 stream
 * `mt` in the reference's order (np.random.random, forces.py:268, 275). */
GCRO_EXPORT void gcro_motor_push_mt(const double *pos_b, int64_t nb, const int64_t *nbor, int64_t nbd1,
                                    double *forces_b, int64_t *where_active_b, const double *tangent, double L,
                                    const double *pos_m, int64_t *where_active_m, const double *params, gcro_mt *mt,
                                    int dim)
{
    const double half_L = L / 2.0;
    double seps[3];
    for (int64_t bi = 0; bi < nb; bi++) {
        const int64_t *row = nbor + bi * nbd1;
        for (int64_t k = 0; k < row[0]; k++) {
            const int64_t mi = row[1 + k];
            if (where_active_m[mi] >= 0) {
                if (mt_double(mt) > params[4]) continue;
                where_active_m[mi] = -1;
                where_active_b[bi] -= 1;
            }
            if (where_active_m[mi] < 0) {
                if (mt_double(mt) < params[3]) {
                    double ds = inbounds_diff(pos_m + mi * dim, pos_b + bi * dim, half_L, L, seps, dim);
                    if (ds <= params[0]) {
                        where_active_b[bi] += 1;
                        where_active_m[mi] = bi;
                        for (int i = 0; i < dim; i++) forces_b[bi * dim + i] += params[2] * tangent[bi * dim + i];
                    }
                }
            }
        }
    }
}

/* The same loop over every bead and every motor within sqrt(list_r2) of it
 * (the beads whose list holds the motor), in ascending motor id, with the
 * keyed draws of gcro_motor_uniforms(seed, motor, bead, step, stage). */
static void motor_push_keyed(const double *pos_b, int64_t nb, double *forces_b, int32_t *act_b,
                             const double *tangent, double L, const double *pos_m, int64_t nm, int32_t *act_m,
                             const double *params, double list_r2, uint64_t seed, int64_t step, int stage, int dim)
{
    const double half_L = L / 2.0;
    double seps[3], u[2];
    for (int64_t bi = 0; bi < nb; bi++) {
        for (int64_t mi = 0; mi < nm; mi++) {
            double ds = inbounds_diff(pos_m + mi * dim, pos_b + bi * dim, half_L, L, seps, dim);
            if (!(ds <= list_r2)) continue;
            gcro_motor_uniforms(seed, (uint32_t)mi, (uint32_t)bi, step, stage, u);
            if (act_m[mi] >= 0) {
                if (u[0] > params[4]) continue;
                act_m[mi] = -1;
                act_b[bi] -= 1;
            }
            if (act_m[mi] < 0 && u[1] < params[3] && ds <= params[0]) {
                act_b[bi] += 1;
                act_m[mi] = (int32_t)bi;
                for (int i = 0; i < dim; i++) forces_b[bi * dim + i] += params[2] * tangent[bi * dim + i];
            }
        }
    }
}

/* n_pops populations: ps[k] / sts[k] as gcro_srk2_run takes them (one
 * thread each; the lists of sts[k] are not used), fixed[k] (pop.fixed: never
 * moves, feels nothing, acts on the others), cross[(k*n + q)*4 + 0..3] the
 * WCA parameters of the force on population k from population q
 * (interpop_forces, updates.py:274-312; r_cut <= 0 or p0 = p1 = 0: none).
 * The call's time values come from g (dt, dtmax, max_dist_per_step,
 * rk_cheat, max_dt_usable, max_steps, noise_mode, step0, srk_order: 2 or 4
 * with sts[k]->forces_aux for SRK4); noise modes as
 * gcro_srk2_run (0: sts[k]->mt[0], 1: injected, 2: Philox with ps[k]->seed).
 * out->max_forces_strength is the first moving population's own value
 * (shared_arr[0, 3], the thread of the first population pair). */
/* A motor population in a group (Motor_Population pushing Chain_Collection
 * `chain_pop`): where_active of every population is reset to -1 at the start
 * of each step (SRK.py:132), the chains get the motor push of each stage as
 * the force of the other population (SRK.py:261-267), and with dont_diffuse
 * an attached motor keeps its position in the stage's update (SRK.py:389-395:
 * after a predictor its pos1 keeps the previous value). */
typedef struct {
    int32_t motor_pop, chain_pop;
    int32_t dont_diffuse;
    int32_t pad;
    double params[5]; /* [motor_max_dist_sq, b_one_motor_per_bead, imparts_force, k_on, k_off] */
    double list_r2;   /* a motor is on the list of the beads within sqrt(list_r2) */
    int32_t *act[8];  /* where_active of each population, int32 [n_beads] */
} gcro_motors;

static int group_run(int n_pops, const gcro_params *const *ps, gcro_state *const *sts, const int32_t *fixed,
                     const double *cross, const gcro_params *g, gcro_result *out, const gcro_motors *mo);

GCRO_EXPORT int gcro_group_run(int n_pops, const gcro_params *const *ps, gcro_state *const *sts,
                               const int32_t *fixed, const double *cross, const gcro_params *g, gcro_result *out)
{
    return group_run(n_pops, ps, sts, fixed, cross, g, out, NULL);
}

/* gcro_group_run with a motor population (SRK2, Philox noise and draws) */
GCRO_EXPORT int gcro_group_run_motors(int n_pops, const gcro_params *const *ps, gcro_state *const *sts,
                                      const int32_t *fixed, const double *cross, const gcro_params *g,
                                      gcro_result *out, const gcro_motors *mo)
{
    if (!mo || g->srk_order == 4 || g->noise_mode != 2) return -3;
    if (mo->motor_pop < 0 || mo->motor_pop >= n_pops || mo->chain_pop < 0 || mo->chain_pop >= n_pops ||
        mo->motor_pop == mo->chain_pop)
        return -1;
    return group_run(n_pops, ps, sts, fixed, cross, g, out, mo);
}

GCRO_EXPORT int gcro_sizeof_motors(void) { return (int)sizeof(gcro_motors); }

static int group_run(int n_pops, const gcro_params *const *ps, gcro_state *const *sts, const int32_t *fixed,
                     const double *cross, const gcro_params *g, gcro_result *out, const gcro_motors *mo)
{
    if (n_pops < 1 || n_pops > 8) return -1;
    const int dim = g->dim;
    const double L = g->L;
    double *tmp[8], *rscr[8];
    int64_t nmax = 1;
    for (int k = 0; k < n_pops; k++) nmax = ps[k]->n_beads > nmax ? ps[k]->n_beads : nmax;
    for (int k = 0; k < n_pops; k++) {
        tmp[k] = (double *)calloc((size_t)nmax * dim, sizeof(double));
        rscr[k] = (double *)malloc(sizeof(double) * (size_t)nmax * 7);
    }
    int first = -1;
    for (int k = 0; k < n_pops; k++)
        if (!fixed[k] && first < 0) first = k;
    /* SRK4 (SRK.py:186-215, 296-321): four stages, each stage's force in
     * forces_aux, their weighted sum in forces */
    const int srk4 = g->srk_order == 4;
    const int n_stages = srk4 ? 4 : 2;
    for (int k = 0; k < n_pops; k++)
        if (srk4 && !fixed[k] && !sts[k]->forces_aux) return -2;
    double dt = g->dt, elapsed = 0.0, mfs0 = 0.0;
    int64_t steps = 0;
    while ((steps < g->max_steps || g->max_steps < 0) && (elapsed < g->max_dt_usable || g->max_dt_usable < 0)) {
        if (mo)
            for (int k = 0; k < n_pops; k++)
                for (int64_t b = 0; b < ps[k]->n_beads; b++) mo->act[k][b] = -1;
        /* noise, SRK.py:134-142, and the SRK2 force wipe */
        for (int k = 0; k < n_pops; k++) {
            if (fixed[k]) continue;
            const gcro_params *p = ps[k];
            gcro_state *st = sts[k];
            const int64_t n = p->n_beads;
            double *noise = st->noise;
            if (g->noise_mode == 0) {
                if (p->D > 0)
                    for (int64_t b = 0; b < n; b++)
                        for (int i = 0; i < dim; i++) noise[b * 2 * dim + i] = draw_normal(st, 0);
                if (p->Dr > 0)
                    for (int64_t b = 0; b < n; b++)
                        for (int i = dim; i < 2 * dim; i++) noise[b * 2 * dim + i] = draw_normal(st, 0);
            } else if (g->noise_mode == 1) {
                int64_t s = steps < st->noise_inject_steps ? steps : st->noise_inject_steps - 1;
                const double *src = st->noise_inject + s * n * 2 * dim;
                for (int64_t b = 0; b < n * 2 * dim; b++) noise[b] = src[b];
            } else {
                for (int64_t b = 0; b < n; b++) {
                    double z[4];
                    double *row = noise + b * 2 * dim;
                    int64_t gs = g->step0 + steps;
                    if (p->D > 0) {
                        gcro_philox_pair(p->seed, (uint32_t)b, gs, 0u, z);
                        if (dim == 3) gcro_philox_pair(p->seed, (uint32_t)b, gs, 1u, z + 2);
                        for (int i = 0; i < dim; i++) row[i] = z[i];
                    }
                    if (p->Dr > 0) {
                        gcro_philox_pair(p->seed, (uint32_t)b, gs, 2u, z);
                        if (dim == 3) gcro_philox_pair(p->seed, (uint32_t)b, gs, 3u, z + 2);
                        for (int i = 0; i < dim; i++) row[dim + i] = z[i];
                    }
                }
            }
            for (int64_t b = 0; b < n * dim; b++) (srk4 ? st->forces_aux : st->forces)[b] = 0.0;
        }
        double dt_for_update = dt;
        for (int stage = 0; stage < n_stages; stage++) {
            const double pref = srk4 ? 1.0 : (stage == 0 ? 1.0 : 0.5);
            const double rescale = stage <= 1 ? 0.5 : 1.0;
            if (srk4 && stage > 0)
                for (int k = 0; k < n_pops; k++)
                    if (!fixed[k])
                        for (int64_t b = 0; b < ps[k]->n_beads * dim; b++) sts[k]->forces_aux[b] = 0.0;
            /* forces taken at pos (stage 0) or pos1; a fixed population's pos1 is its pos */
            double *X[8];
            for (int k = 0; k < n_pops; k++) X[k] = (stage == 0 || fixed[k]) ? sts[k]->pos : sts[k]->pos1;
            for (int k = 0; k < n_pops; k++) {
                if (fixed[k]) continue;
                const gcro_params *p = ps[k];
                gcro_state *st = sts[k];
                double *Fs = srk4 ? st->forces_aux : st->forces; /* write_to_forces */
                if (p->calc_springs)
                    spring_forces(X[k], st->tangent, st->chain_id, Fs, p->n_beads, L, p->spring, st->rest_lengths,
                                  dim);
                if (p->calc_wca)
                    pair_forces_all(X[k], p->n_beads, st->chain_id, p->n_nearby, X[k], p->n_beads, 1, p->wca, L,
                                    dim, Fs);
                if (p->self_propel) self_propel(Fs, st->tangent, p->n_beads, p->active, dim);
            }
            /* the other populations' forces, added in turns (SRK.py:287-294) */
            for (int ii = 1; ii < n_pops; ii++)
                for (int k = 0; k < n_pops; k++) {
                    if (fixed[k]) continue;
                    const int q = (k + ii) % n_pops;
                    if (mo && k == mo->chain_pop && q == mo->motor_pop) {
                        const int64_t n = ps[k]->n_beads;
                        memset(tmp[k], 0, sizeof(double) * (size_t)n * dim);
                        motor_push_keyed(X[k], n, tmp[k], mo->act[k], sts[k]->tangent, L, X[q], ps[q]->n_beads,
                                         mo->act[q], mo->params, mo->list_r2, ps[q]->seed, g->step0 + steps, stage,
                                         dim);
                        double *Fs = sts[k]->forces;
                        for (int64_t b = 0; b < n * dim; b++) Fs[b] += tmp[k][b];
                        continue;
                    }
                    const double *w = cross + ((size_t)k * n_pops + q) * 4;
                    if (!(w[3] > 0.0) || (w[0] == 0.0 && w[1] == 0.0)) continue;
                    const int64_t n = ps[k]->n_beads;
                    memset(tmp[k], 0, sizeof(double) * (size_t)n * dim);
                    pair_forces_all(X[k], n, sts[k]->chain_id, 0, X[q], ps[q]->n_beads, 0, w, L, dim, tmp[k]);
                    double *Fs = srk4 ? sts[k]->forces_aux : sts[k]->forces;
                    for (int64_t b = 0; b < n * dim; b++) Fs[b] += tmp[k][b];
                }
            if (srk4) {
                /* SRK.py:296-321: weighted sum of the stage forces */
                const double mult = (stage == 0 || stage == 3) ? 1. / 6. : 1. / 3.;
                for (int k = 0; k < n_pops; k++) {
                    if (fixed[k]) continue;
                    double *F = sts[k]->forces;
                    const double *Fa = sts[k]->forces_aux;
                    for (int64_t b = 0; b < ps[k]->n_beads * dim; b++) F[b] = stage == 0 ? Fa[b] * mult : F[b] + Fa[b] * mult;
                }
            }
            if (stage == n_stages - 1) {
                /* SRK.py:323-353 over every moving population */
                double Sg = 0.0;
                for (int k = 0; k < n_pops; k++) {
                    if (fixed[k]) continue;
                    const gcro_params *p = ps[k];
                    const double *F = sts[k]->forces;
                    double S = sqrt(2.0 * p->D);
                    if (p->n_beads > 0) {
                        double m = -1.0;
                        for (int64_t b = 0; b < p->n_beads; b++) {
                            double s2 = 0.0;
                            for (int i = 0; i < dim; i++) s2 += F[b * dim + i] * F[b * dim + i];
                            if (s2 > m) m = s2;
                        }
                        S += pref * sqrt(m) / p->radius;
                    }
                    if (k == first) mfs0 = S;
                    if (S > Sg) Sg = S;
                }
                if (Sg == 0.0)
                    dt = g->dtmax;
                else {
                    double c = g->max_dist_per_step / Sg;
                    dt = g->dtmax < c ? g->dtmax : c;
                }
                double dt_used = g->rk_cheat * dt;
                if (g->max_dt_usable > 0) {
                    double lim = g->max_dt_usable - elapsed;
                    if (lim < dt_used) dt_used = lim;
                }
                elapsed += dt_used;
                dt_for_update = dt_used;
            }
            for (int k = 0; k < n_pops; k++) {
                if (fixed[k]) continue;
                const gcro_params *p = ps[k];
                gcro_state *st = sts[k];
                const int64_t n = p->n_beads;
                double *W = srk4 ? (stage == 3 ? st->pos : st->pos1) : (stage == 0 ? st->pos1 : st->pos);
                double dt_eff = srk4 ? dt_for_update * rescale * pref : dt_for_update * pref;
                const double s2 = sqrt(2.0 * dt_for_update * p->D);
                const int rigid = p->rigid_rod != 0.0 && p->longest_chain_length > 2;
                /* SRK.py:355-362: virtual SRK4 updates use the stage force */
                const double *Fu = (srk4 && stage < 3) ? st->forces_aux : st->forces;
                if (n > 0 && rigid) {
                    project_rigid(W, X[k], Fu, st->noise, n, st->chain_id, st->rest_lengths, p->rigid_rod, L,
                                  dt_eff, p->D, p->radius, dim, rscr[k], rscr[k] + 3 * n, rscr[k] + 6 * n);
                } else {
                    dt_eff /= p->radius;
                    const int hold = mo && k == mo->motor_pop && mo->dont_diffuse;
                    for (int64_t b = 0; b < n; b++)
                        for (int i = 0; i < dim; i++) {
                            if (hold && mo->act[k][b] >= 0) continue; /* an attached motor stays */
                            double t = st->pos[b * dim + i] + dt_eff * Fu[b * dim + i];
                            if (s2 != 0.0) t += s2 * st->noise[b * 2 * dim + i];
                            W[b * dim + i] = py_mod(t, L);
                        }
                }
            }
        }
        /* rotational diffusion, SRK.py:399-423 */
        for (int k = 0; k < n_pops; k++) {
            const gcro_params *p = ps[k];
            const int b_get_orientations = p->calc_springs ? (p->spring[4] != 0.0) : 0;
            if (fixed[k] || !(p->Dr > 0) || b_get_orientations) continue;
            gcro_state *st = sts[k];
            double sq = sqrt(2.0 * dt_for_update * p->Dr) * 3.141592653589793;
            for (int64_t b = 0; b < p->n_beads; b++) {
                double *xr = st->noise + b * 2 * dim + dim;
                double *tb = st->tangent + b * dim;
                double proj = 0.0;
                for (int i = 0; i < dim; i++) proj += xr[i] * tb[i];
                for (int i = 0; i < dim; i++) xr[i] -= proj * tb[i];
                double mag = 0.0;
                for (int i = 0; i < dim; i++) {
                    double v = tb[i] + sq * xr[i];
                    mag += v * v;
                    tb[i] = v;
                }
                mag = sqrt(mag);
                for (int i = 0; i < dim; i++) tb[i] /= mag;
            }
        }
        steps++;
    }
    for (int k = 0; k < n_pops; k++) {
        free(tmp[k]);
        free(rscr[k]);
    }
    out->dt = dt;
    out->dt_used_total = elapsed;
    out->steps = (double)steps;
    out->max_forces_strength = mfs0;
    out->counter = 0.0;
    out->flag = 0.0;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Observables                                                         */
/* ------------------------------------------------------------------ */

/* output_methods.calc_avg_phi_chain (492-510) + analysis.polar_orderparameter
 * (315-328) + analysis.nematic_orderparameter (294-313).  Chains are given
 * as contiguous bead ranges [chain_start[c], chain_start[c+1]).
 * out = [P, S, director_angle]. */
GCRO_EXPORT void gcro_order_params(const double *tangent, const int64_t *chain_start, int64_t n_chains,
                                   int dim, double *out)
{
    double ex_sum = 0.0, ey_sum = 0.0, q11 = 0.0, q12 = 0.0;
    for (int64_t c = 0; c < n_chains; c++) {
        double sx = 0.0, sy = 0.0;
        for (int64_t b = chain_start[c]; b < chain_start[c + 1]; b++) {
            sx += tangent[b * dim];
            sy += tangent[b * dim + 1];
        }
        double phi = atan2(sy, sx);
        double ex = cos(phi), ey = sin(phi);
        ex_sum += ex;
        ey_sum += ey;
        q11 += 2.0 * ex * ex - 1.0;
        q12 += 2.0 * ex * ey;
    }
    double P = sqrt(ex_sum * ex_sum + ey_sum * ey_sum) / (double)n_chains;
    double Sfull = sqrt(q11 * q11 + q12 * q12);
    double ang = atan((Sfull - q11) / q12);
    out[0] = P;
    out[1] = Sfull / (double)n_chains;
    out[2] = ang;
}

GCRO_EXPORT int gcro_sizeof_params(void) { return (int)sizeof(gcro_params); }
GCRO_EXPORT int gcro_sizeof_state(void) { return (int)sizeof(gcro_state); }
GCRO_EXPORT int gcro_sizeof_mt(void) { return (int)sizeof(gcro_mt); }
