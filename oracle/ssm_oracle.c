/*
 * ssm_oracle.c -- TEST ORACLE: a sequential CPU restatement of the reference
 * simulators (ssm-simulators, src/cssm/*.pyx, n_threads=1 path).
 *
 * Test infrastructure only.  Tests, the smoke check and the CPU-baseline leg of
 * the benchmark link this file; the product never does.
 *
 * Arithmetic follows the C that Cython generates for the reference, operation
 * by operation: float32 where the source uses C floats, double where Cython
 * emits double literals (e.g. `-1.0 * b`, `z * 2.0`, `u * 0.5`).  Compile with
 * -O2 -ffp-contract=off (no fast-math) so every operation rounds as written.
 *
 * Noise comes from one of two sources:
 *  - stream mode: the reference's batch layout -- increments are read from a
 *    buffer of num_draws values that is refilled through a callback when
 *    exhausted (src/cssm/ddm_models.pyx:729-739); the Python driver fills it
 *    from numpy.random.default_rng(seed), reproducing the reference exactly;
 *  - row mode (noise injection): trajectory w reads row w of a caller matrix,
 *    which is what the GPU kernels consume in their noise-injection mode.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef void (*oracle_refill_fn)(float *buf, int64_t n, int64_t trial);

typedef struct {
    /* row mode */
    const float *rows;
    int64_t row_len;
    const float *urows;
    /* stream mode */
    float *gbuf;
    int64_t gn, m;
    oracle_refill_fn refill_g;
    float *ubuf;
    int64_t un, mu;
    oracle_refill_fn refill_u;
    /* diagnostics */
    int64_t overrun;
} oracle_noise;

static inline float next_g(oracle_noise *nz, int64_t w, int64_t i, int64_t trial) {
    if (nz->rows) {
        if (i >= nz->row_len) {
            nz->overrun += 1;
            return 0.0f;
        }
        return nz->rows[w * nz->row_len + i];
    }
    float g = nz->gbuf[nz->m];
    nz->m += 1;
    if (nz->m == nz->gn) {
        nz->refill_g(nz->gbuf, nz->gn, trial);
        nz->m = 0;
    }
    return g;
}

static inline float next_u(oracle_noise *nz, int64_t w, int64_t trial) {
    if (nz->rows) return nz->urows[w];
    float u = nz->ubuf[nz->mu];
    nz->mu += 1;
    if (nz->mu == nz->un) {
        nz->refill_u(nz->ubuf, nz->un, trial);
        nz->mu = 0;
    }
    return u;
}

/* compute_smooth_unif (src/cssm/_utils.pyx:668-695): double arithmetic. */
static inline float smooth_jitter(int smooth, float tp, float dl_tmp, float dt, float u) {
    if (!smooth) return 0.0f;
    if (tp == 0.0) return (float)(((double)u * 0.5) * (double)dt);
    if (tp < dl_tmp) return (float)((0.5 - (double)u) * (double)dt);
    return 0.0f;
}

/* compute_deadline_tmp (src/cssm/_utils.pyx:712-718). */
static inline float deadline_tmp(float max_t, float deadline, float t) {
    float x = deadline - t;
    return (x < max_t) ? x : max_t;
}

static inline int sign_f(float y) { return (y > 0) - (y < 0); }

/*
 * One trial k of ddm_flexbound / levy_flexbound (ddm_models.pyx:696-744,
 * levy_models.pyx:160-222).  `scale` is sqrt(dt)*s (DDM) or s*dt^(1/alpha)
 * (Levy); `bound` is the trial's boundary table of nb entries.  Outputs are
 * written at index n * n_trials + k.
 */
int64_t oracle_flex_trial(int64_t k, int64_t n_samples, int64_t n_trials, float v, float z,
                          float t, float deadline, float scale, const float *bound, int64_t nb,
                          float max_t, float dt, int smooth, oracle_noise *nz, float *rts,
                          int32_t *choices, int32_t *steps, float *traj, int64_t traj_len) {
    const float dl = deadline_tmp(max_t, deadline, t);
    int64_t total_steps = 0;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        float y = (float)((-1.0 * (double)bound[0]) + (((double)z * 2.0) * (double)bound[0]));
        float tp = 0.0f;
        int64_t ix = 0;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec && traj_len > 0) traj[0] = y;
        for (;;) {
            const float b = bound[ix < nb ? ix : nb - 1];
            if (!((y >= (-1.0 * (double)b)) && (y <= b) && (tp <= dl))) break;
            const float g = next_g(nz, w, ix, k);
            /* the reference build (-ffast-math) evaluates y += v*dt + scale*g
               as (y + v*dt) + scale*g; verified on its recorded trajectories */
            y = (y + (v * dt)) + (scale * g);
            tp = tp + dt;
            ix += 1;
            if (rec && ix < traj_len) traj[ix] = y;
        }
        const float u = next_u(nz, w, k);
        const float sm = smooth_jitter(smooth, tp, dl, dt, u);
        float rt = (tp + t) + sm;
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        rts[w] = rt;
        choices[w] = sign_f(y);
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/* One trial of the legacy DDM on [0, a] (ddm_models.pyx:446-481). */
int64_t oracle_ddm_trial(int64_t k, int64_t n_samples, int64_t n_trials, float v, float a,
                         float z, float t, float deadline, float s, float sqrt_dt, float max_t,
                         float dt, int smooth, oracle_noise *nz, float *rts, int32_t *choices,
                         int32_t *steps, float *traj, int64_t traj_len) {
    const float dl = deadline_tmp(max_t, deadline, t);
    const float sqrt_st = sqrt_dt * s;
    int64_t total_steps = 0;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        float y = z * a;
        float tp = 0.0f;
        int64_t ix = 0;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec && traj_len > 0) traj[0] = y;
        while (y <= a && y >= 0 && tp <= dl) {
            const float g = next_g(nz, w, ix, k);
            y = (y + (v * dt)) + (sqrt_st * g);
            tp = tp + dt;
            ix += 1;
            if (rec && ix < traj_len) traj[ix] = y;
        }
        const float u = next_u(nz, w, k);
        const float sm = smooth_jitter(smooth, tp, dl, dt, u);
        float rt = (tp + t) + sm;
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        rts[w] = rt;
        choices[w] = sign_f(y);
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/*
 * One trial of ddm_sdv (variant 0; ddm_models.pyx:2612-2668) or full_ddm
 * (variant 1; ddm_models.pyx:2233-2316): the flexible-bound DDM with a drift
 * drawn per sample, v + sv * N(0,1), and for full_ddm a start point displaced
 * by U(-sz, sz) and a non-decision time displaced by U(-st, st).
 *
 * Stream order per sample (full_ddm): the drift normal is read, the t and y
 * uniforms are consumed, then the drift normal is consumed; ddm_sdv consumes
 * its drift normal at once.  Row mode: row w = [drift normal, walk normals...];
 * uniform row w (stride ustride) = [u_t, u_y, u_smooth] (full_ddm) or
 * [u_smooth] (ddm_sdv).
 */
static inline float peek_g(oracle_noise *nz, int64_t w) {
    if (nz->rows) return nz->rows[w * nz->row_len];
    return nz->gbuf[nz->m];
}
static inline void advance_g(oracle_noise *nz, int64_t trial) {
    if (nz->rows) return;
    nz->m += 1;
    if (nz->m == nz->gn) {
        nz->refill_g(nz->gbuf, nz->gn, trial);
        nz->m = 0;
    }
}
static inline float next_u_at(oracle_noise *nz, int64_t w, int64_t ustride, int64_t j, int64_t trial) {
    if (nz->rows) return nz->urows[w * ustride + j];
    return next_u(nz, w, trial);
}

int64_t oracle_var_trial(int64_t k, int64_t n_samples, int64_t n_trials, int variant, float v,
                         float z, float t, float sz, float sv, float st, float deadline,
                         float sqrt_st, const float *bound, int64_t nb, float max_t, float dt,
                         int smooth, oracle_noise *nz, float *rts, int32_t *choices,
                         int32_t *steps, float *traj, int64_t traj_len) {
    const float dl = deadline_tmp(max_t, deadline, t);
    const int64_t ustride = variant ? 3 : 1;
    int64_t total_steps = 0;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        float y = (float)((-1.0 * (double)bound[0]) + (((double)z * 2.0) * (double)bound[0]));
        const float drift = (v + (sv * peek_g(nz, w))) * dt;
        float t_tmp = t;
        if (variant) {
            /* t + 2 (u - 0.5) st and y + 2 (u - 0.5) sz, in double as the generated C */
            const float ut = next_u_at(nz, w, ustride, 0, k);
            t_tmp = (float)((double)t + ((2.0 * ((double)ut - 0.5)) * (double)st));
            const float uy = next_u_at(nz, w, ustride, 1, k);
            y = (float)((double)y + ((2.0 * ((double)uy - 0.5)) * (double)sz));
        }
        advance_g(nz, k);
        float tp = 0.0f;
        int64_t ix = 0;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec && traj_len > 0) traj[0] = y;
        for (;;) {
            const float b = bound[ix < nb ? ix : nb - 1];
            if (!((y >= (-1.0 * (double)b)) && (y <= b) && (tp <= dl))) break;
            const float g = next_g(nz, w, ix + 1, k);
            y = (y + drift) + (sqrt_st * g);
            tp = tp + dt;
            ix += 1;
            if (rec && ix < traj_len) traj[ix] = y;
        }
        const float u = next_u_at(nz, w, ustride, ustride - 1, k);
        const float sm = smooth_jitter(smooth, tp, dl, dt, u);
        float rt = (tp + t_tmp) + sm;
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        rts[w] = rt;
        choices[w] = sign_f(y);
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/*
 * One trial of ornstein_uhlenbeck (src/cssm/ornstein_models.pyx:157-199):
 * y += (v - g y) dt + sqrt(dt) s N(0,1) between the boundaries +-b(t).
 */
int64_t oracle_ou_trial(int64_t k, int64_t n_samples, int64_t n_trials, float v, float z, float g,
                        float t, float deadline, float sqrt_st, const float *bound, int64_t nb,
                        float max_t, float dt, int smooth, oracle_noise *nz, float *rts,
                        int32_t *choices, int32_t *steps, float *traj, int64_t traj_len) {
    const float dl = deadline_tmp(max_t, deadline, t);
    int64_t total_steps = 0;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        /* (-1) * b0 + z * 2 * b0: all float in the generated C (int literals) */
        float y = (-bound[0]) + ((z * 2.0f) * bound[0]);
        float tp = 0.0f;
        int64_t ix = 0;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec && traj_len > 0) traj[0] = y;
        for (;;) {
            const float b = bound[ix < nb ? ix : nb - 1];
            if (!((y >= (-1.0 * (double)b)) && (y <= b) && (tp <= dl))) break;
            const float gm = next_g(nz, w, ix, k);
            y = (y + ((v - (g * y)) * dt)) + (sqrt_st * gm);
            tp = tp + dt;
            ix += 1;
            if (rec && ix < traj_len) traj[ix] = y;
        }
        const float u = next_u(nz, w, k);
        const float sm = smooth_jitter(smooth, tp, dl, dt, u);
        float rt = (tp + t) + sm;
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        rts[w] = rt;
        choices[w] = sign_f(y);
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/*
 * One trial of ddm_flex (src/cssm/ddm_models.pyx:996-1043): the drift of step
 * ix is the trial's drift table at ix (the drift function on the time grid),
 * y += (v(t_ix) * dt) + sqrt_st * g.
 */
int64_t oracle_dflex_trial(int64_t k, int64_t n_samples, int64_t n_trials, float z, float t,
                           float deadline, float sqrt_st, const float *bound, int64_t nb,
                           const float *drift, int64_t nd, float max_t, float dt, int smooth,
                           oracle_noise *nz, float *rts, int32_t *choices, int32_t *steps, float *traj,
                           int64_t traj_len) {
    const float dl = deadline_tmp(max_t, deadline, t);
    int64_t total_steps = 0;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        /* (-1) * b0 + z * 2 * b0 with integer literals: float arithmetic */
        float y = (-bound[0]) + ((z * 2.0f) * bound[0]);
        float tp = 0.0f;
        int64_t ix = 0;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec && traj_len > 0) traj[0] = y;
        for (;;) {
            const float b = bound[ix < nb ? ix : nb - 1];
            if (!((y >= (-1.0 * (double)b)) && (y <= b) && (tp <= dl))) break;
            const float gm = next_g(nz, w, ix, k);
            y = (y + (drift[ix < nd ? ix : nd - 1] * dt)) + (sqrt_st * gm);
            tp = tp + dt;
            ix += 1;
            if (rec && ix < traj_len) traj[ix] = y;
        }
        const float u = next_u(nz, w, k);
        const float sm = smooth_jitter(smooth, tp, dl, dt, u);
        float rt = (tp + t) + sm;
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        rts[w] = rt;
        choices[w] = sign_f(y);
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/*
 * One trial of racing_diffusion_model (src/cssm/race_models.pyx:1205-1266):
 * np accumulators start at U(0, A) (the reference draws these with C rand(),
 * rand() / RAND_MAX in float), each step updates them in index order,
 * x_j += v_j dt + sqrt_st g, and the first one at or above b ends the walk
 * before the time is advanced.  No lower boundary.  Row mode: increments
 * step-major (step * np + j); uniform row w = [starts..., u_smooth].
 */
#include <stdlib.h>
int64_t oracle_rdm_trial(int64_t k, int64_t n_samples, int64_t n_trials, int np_, const float *v,
                         float b, float A, float t, float deadline, float sqrt_st, float max_t,
                         float dt, int smooth, oracle_noise *nz, float *rts, int32_t *choices,
                         int32_t *steps, float *traj, int64_t traj_len) {
    float x[64];
    const float dl = deadline_tmp(max_t, deadline, t);
    int64_t total_steps = 0;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        for (int j = 0; j < np_; ++j) {
            float u;
            if (nz->rows) u = nz->urows[w * (np_ + 1) + j];
            else u = ((float)rand()) / RAND_MAX;
            x[j] = u * A;
        }
        float tp = 0.0f;
        int64_t ix = 0;
        int winner = -1;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec)
            for (int j = 0; j < np_ && j < traj_len; ++j) traj[j] = x[j];
        while (winner < 0 && tp <= dl) {
            for (int j = 0; j < np_; ++j) {
                const float g = next_g(nz, w, ix * np_ + j, k);
                x[j] = (x[j] + (v[j] * dt)) + (sqrt_st * g);
                if (x[j] >= b) {
                    winner = j;
                    break;
                }
            }
            if (winner >= 0) break;
            tp = tp + dt;
            ix += 1;
            if (rec && (ix + 1) * np_ <= traj_len)
                for (int j = 0; j < np_; ++j) traj[ix * np_ + j] = x[j];
        }
        const float u = nz->rows ? nz->urows[w * (np_ + 1) + np_] : next_u(nz, w, k);
        const float sm = smooth_jitter(smooth, tp, dl, dt, u);
        float rt = (tp + t) + sm;
        int ch = winner;
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        if (rt == -999.0f || winner < 0) {
            rt = -999.0f;
            ch = -1;
        }
        rts[w] = rt;
        choices[w] = ch;
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/*
 * One trial of race_model (race_models.pyx:417-464) or lca
 * (race_models.pyx:825-879), selected by `lca`.  v, z, sqrt_st hold the
 * trial's np particle values; increments are consumed particle-major within a
 * step (draw index step*np + j in row mode).
 */
int64_t oracle_race_trial(int64_t k, int64_t n_samples, int64_t n_trials, int np_, int lca,
                          const float *v, const float *z, const float *sqrt_st, float g_leak,
                          float b_inh, float t, float deadline, const float *bound, int64_t nb,
                          float max_t, float dt, int smooth, oracle_noise *nz, float *rts,
                          int32_t *choices, int32_t *steps, float *traj, int64_t traj_len) {
    float p[64], red[64];
    const float dl = deadline_tmp(max_t, deadline, t);
    /* lca's time accumulator is an undeclared local in the reference, which
       Cython infers as C double (race_models.pyx:838,862); race_model's is float */
    int64_t total_steps = 0;
    if (np_ > 64) return -1;
    for (int64_t n = 0; n < n_samples; ++n) {
        const int64_t w = n * n_trials + k;
        for (int j = 0; j < np_; ++j) p[j] = z[j] * bound[0];
        float tp = 0.0f;
        double tpd = 0.0;
        int64_t ix = 0, di = 0;
        const int rec = (traj != 0 && n == 0 && k == 0);
        if (rec && traj_len > 0)
            for (int j = 0; j < np_; ++j) traj[j] = p[j];
        for (;;) {
            const float b = bound[ix < nb ? ix : nb - 1];
            int finished = 0;
            for (int j = 0; j < np_; ++j)
                if (p[j] > b) { finished = 1; break; }
            if (finished || !(lca ? (tpd <= (double)dl) : (tp <= dl))) break;
            if (lca) {
                float sum = 0.0f;
                for (int j = 0; j < np_; ++j) sum = sum + p[j];
                for (int j = 0; j < np_; ++j) {
                    red[j] = (float)((-1.0 * (double)p[j]) + (double)sum);
                    const float g = next_g(nz, w, di++, k);
                    /* reference build association: (p + A*dt) + sqrt_st*g */
                    p[j] = (p[j] + (((v[j] - (g_leak * p[j])) - (b_inh * red[j])) * dt)) + (sqrt_st[j] * g);
                    p[j] = (float)fmax(0.0, (double)p[j]);
                }
            } else {
                for (int j = 0; j < np_; ++j) {
                    const float g = next_g(nz, w, di++, k);
                    p[j] = (p[j] + (v[j] * dt)) + (sqrt_st[j] * g);
                    p[j] = (float)fmax(0.0, (double)p[j]);
                }
            }
            if (lca) tpd = tpd + (double)dt; else tp = tp + dt;
            ix += 1;
            if (rec && (ix + 1) * np_ <= traj_len)
                for (int j = 0; j < np_; ++j) traj[ix * np_ + j] = p[j];
        }
        const float u = next_u(nz, w, k);
        /* compute_smooth_unif receives the time rounded to a C float */
        const float sm = smooth_jitter(smooth, lca ? (float)tpd : tp, dl, dt, u);
        /* choice = np.argmax(particles): first index of the maximum */
        int best = 0;
        for (int j = 1; j < np_; ++j)
            if (p[j] > p[best]) best = j;
        float rt = lca ? (float)((tpd + (double)t) + (double)sm) : ((tp + t) + sm);
        if (rt >= deadline || deadline <= 0) rt = -999.0f;
        rts[w] = rt;
        choices[w] = best;
        if (steps) steps[w] = (int32_t)ix;
        total_steps += ix;
    }
    return total_steps;
}

/*
 * lba_vanilla closed form (src/cssm/lba_models.pyx:101-115) in float32 on
 * caller draws: zs[n][k][j] ~ U(0, A), vs[n][k][j] = |N(v, sd)|.
 */
void oracle_lba_f32(int64_t n_samples, int64_t n_trials, int nact, const float *a,
                    const float *t, const float *deadline, const float *zs, const float *vs,
                    float *rts, int32_t *choices) {
    for (int64_t n = 0; n < n_samples; ++n)
        for (int64_t k = 0; k < n_trials; ++k) {
            const int64_t w = n * n_trials + k;
            int best = 0;
            float bx = 0.0f;
            for (int j = 0; j < nact; ++j) {
                const float x = (a[k] - zs[w * nact + j]) / vs[w * nact + j];
                if (j == 0 || x < bx) { bx = x; best = j; }
            }
            float rt = bx + t[k];
            if (rt >= deadline[k]) rt = -999.0f;
            rts[w] = rt;
            choices[w] = best;
        }
}

int oracle_abi_version(void) { return 1; }
