/*
 * ssm_b200.h -- C ABI of the sm_100a sequential-sampling-model simulators.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), launches asynchronously on that stream and returns an
 * int status (SSM_OK on success).  Nothing here allocates device memory: the
 * caller owns outputs and provides the scratch workspace whose size the
 * matching *_workspace_bytes() query reports.  Outputs follow the reference
 * package's layout: rts float32 and choices int32, indexed by
 * (sample n, trial k) as  n * n_trials + k  ([n_samples, n_trials, 1] in the
 * reference), or -- for the ragged batched form -- sample_offsets[k] + n.
 *
 * Each entry point cites the reference interface it replaces (paths relative
 * to the ssm-simulators source tree).
 */
#ifndef SSM_B200_H
#define SSM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SSM_OK 0
#define SSM_ERR_ARG 1          /* invalid argument (null pointer, bad size, bad enum) */
#define SSM_ERR_CUDA 2         /* a CUDA runtime call failed; see ssm_last_error() */
#define SSM_ERR_WORKSPACE 3    /* workspace missing or smaller than *_workspace_bytes() */
#define SSM_ERR_NOISE_RANGE 4  /* a trajectory needed more injected increments than its row holds */
#define SSM_ERR_DEVICE 5       /* the device reported an error flag (read by ssm_check_status) */

/* ---- boundary kinds for the single-accumulator simulators -------------- */
/* The reference evaluates boundary_fun(t_s, **boundary_params) on the host
 * into a float32 table (src/cssm/_utils.pyx:655-666).  Here the common
 * families are evaluated in registers; any other function uses TABLE. */
#define SSM_BOUND_TABLE 0    /* b(ix) = table[k * table_stride + min(ix, table_len-1)] */
#define SSM_BOUND_CONSTANT 1 /* b(t) = a                                               */
#define SSM_BOUND_LINEAR 2   /* b(t) = a + t * p1   (angle: p1 = -sin(theta)/cos(theta)) */
#define SSM_BOUND_WEIBULL 3  /* b(t) = a * exp(-(t / p2)^p1)  (p1 = alpha, p2 = beta)   */

/* ---- noise sources ------------------------------------------------------ */
/* Device RNG: counter-based Philox4x32-10 keyed by (seed, trial k, sample n),
 * so a trajectory's stream does not depend on the launch configuration.
 * Noise injection: the caller passes pre-drawn standard increments, one row
 * of noise_row_len float32 per trajectory (row index = output index), plus
 * one uniform per trajectory for the rt jitter; results are then bit-exact
 * with a sequential CPU restatement consuming the same rows. */

/* Per-call launch options shared by the simulators. */
typedef struct ssm_launch {
    int block_threads;     /* 0 = library default (autotuned value if set) */
    int blocks_per_sm;     /* 0 = as many as fit                            */
    int chunk;             /* trajectories a warp claims per queue access; 0 = default */
    int refill_min;        /* ended walks a warp collects before restarting lanes (1-32); 0 = default */
    /* Index that trial 0 of this call has in the random streams (0 = none).
     * A batch simulated as several calls over consecutive trial windows --
     * each with its per-trial pointers advanced to the window, first_trial =
     * the window's first trial, and the window's slice of the batch's ragged
     * sample_offsets (whose values stay global output indices) -- gives the
     * same outputs as one call over the whole batch. */
    int64_t first_trial;
    /* Processing order of the trials (every Euler simulator; ragged layout
     * only; NULL = index order): trial_order[j] is the trial simulated
     * j-th and order_offsets[0..n_trials] the prefix sums of the sample
     * counts in that order (order_offsets[0] = 0).  Outputs and random
     * streams do not depend on the order; starting the longest walks first
     * shortens the launch's tail.  An entry that does not match
     * sample_offsets stores SSM_ERR_ARG and its position in the device error
     * word (ssm_check_status then returns SSM_ERR_DEVICE) and its
     * trajectories are skipped. */
    const int32_t *trial_order;
    const int64_t *order_offsets;
    /* Lanes per trajectory of the single-accumulator simulators (device RNG,
     * constant / linear / Weibull boundary): 1, 2, 4 or 8; 0 = automatic,
     * which is 1 for the ragged layout and otherwise chosen from the number
     * of trajectories against the grid's lanes (ssm_auto_lanes_per_walk).
     * With W > 1 the W lanes of a group draw a walk's increments in parallel
     * and step it together: results are bit-identical to W = 1, and a launch
     * with fewer trajectories than lanes ends sooner; chunk is 32 / W. */
    int lanes_per_walk;
} ssm_launch;

/* Version / diagnostics -------------------------------------------------- */
int ssm_version(void);
/* Last error message of the calling thread (static storage, never NULL). */
const char *ssm_last_error(void);
/* Copy the device error word written by the last launch that used `workspace`
 * back to the host (synchronises `stream`); returns SSM_OK or the stored code. */
int ssm_check_status(const void *workspace, void *stream);

/* ---- single-accumulator Euler-Maruyama DDM family ----------------------- */

/* Bytes of scratch the DDM-family entry points need for n_trials trials. */
size_t ssm_ddm_workspace_bytes(int64_t n_trials);
/* Lanes per walk (ssm_launch.lanes_per_walk) the library picks for a
 * single-accumulator launch of n_walks trajectories on the current device
 * when the option is 0 and the layout is not ragged; callers of the ragged
 * layout, which know their total, pass it explicitly.  No reference
 * counterpart: a launch-shape choice of this library. */
int ssm_auto_lanes_per_walk(int64_t n_walks);

/*
 * ssm_ddm_flexbound -- replaces cssm.ddm_flexbound
 * (src/cssm/ddm_models.pyx:589-878, sequential loop :696-744).
 * Per trial k: start y = -b(0) + 2 z b(0); while -b(ix) <= y <= b(ix) and
 * t <= min(max_t, deadline - t_nd): y += v dt + sqrt(dt) s g.  rt = t + t_nd +
 * jitter, choice = sign(y), rt = -999 when rt >= deadline or deadline <= 0.
 *
 * v, a, z, t, deadline, s : float32[n_trials]
 * bound_p1, bound_p2      : float32[n_trials] or NULL (see SSM_BOUND_*)
 * bound_table             : float32[n_trials * table_stride] (TABLE only)
 * sample_offsets          : NULL for n_samples per trial in the reference
 *                           layout, else int64[n_trials+1] ragged prefix sums
 *                           (output index sample_offsets[k] + n; the call
 *                           simulates outputs sample_offsets[0] ..
 *                           sample_offsets[n_trials] - 1)
 * max_t_per_trial         : NULL (use max_t) or float32[n_trials]
 * noise_rows / noise_row_len / noise_unif : NULL for the device RNG
 * traj                    : NULL or float32[traj_len]; receives trial 0 /
 *                           sample 0's path (-999 padded) as in the reference
 * steps                   : NULL or int32 per output; Euler steps taken
 */
int ssm_ddm_flexbound(const float *v, const float *a, const float *z, const float *t,
                      const float *deadline, const float *s, int64_t n_trials, int64_t n_samples,
                      const int64_t *sample_offsets, float max_t, const float *max_t_per_trial,
                      float delta_t, int bound_kind, const float *bound_p1, const float *bound_p2,
                      const float *bound_table, int64_t table_stride, int64_t table_len,
                      uint64_t seed, int smooth_unif, const float *noise_rows,
                      int64_t noise_row_len, const float *noise_unif, float *rts,
                      int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                      const ssm_launch *launch, void *workspace, size_t workspace_bytes,
                      void *stream);

/*
 * ssm_ddm -- replaces cssm.ddm (src/cssm/ddm_models.pyx:349-582): the legacy
 * DDM on [0, a] with start z a and exit when y > a or y < 0.  Layout and noise
 * conventions as ssm_ddm_flexbound.
 */
int ssm_ddm(const float *v, const float *a, const float *z, const float *t, const float *deadline,
            const float *s, int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets,
            float max_t, float delta_t,
            uint64_t seed, int smooth_unif, const float *noise_rows, int64_t noise_row_len,
            const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
            int64_t traj_len, const ssm_launch *launch, void *workspace, size_t workspace_bytes,
            void *stream);

/*
 * ssm_levy_flexbound -- replaces cssm.levy_flexbound
 * (src/cssm/levy_models.pyx:47-348): y += v dt + s dt^(1/alpha) X, X symmetric
 * alpha-stable drawn in-kernel by Chambers-Mallows-Stuck (reference sampler:
 * src/cssm/_utils.pyx:369-472).  Same boundary/offset/noise conventions as
 * ssm_ddm_flexbound; injected rows hold alpha-stable draws.
 */
int ssm_levy_flexbound(const float *v, const float *a, const float *z, const float *alpha,
                       const float *t, const float *deadline, const float *s, int64_t n_trials,
                       int64_t n_samples, const int64_t *sample_offsets, float max_t,
                       float delta_t, int bound_kind, const float *bound_p1, const float *bound_p2,
                       const float *bound_table, int64_t table_stride, int64_t table_len,
                       uint64_t seed, int smooth_unif, const float *noise_rows,
                       int64_t noise_row_len, const float *noise_unif, float *rts,
                       int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                       const ssm_launch *launch, void *workspace, size_t workspace_bytes,
                       void *stream);

/*
 * ssm_ddm_sdv -- replaces cssm.ddm_sdv (src/cssm/ddm_models.pyx:2500-2797):
 * ddm_flexbound with the drift drawn per trajectory, v + sv * N(0,1).
 * Noise injection: row w = [drift normal, walk normals...] (noise_row_len >=
 * 1 + steps), noise_unif[w] = the jitter uniform.
 */
int ssm_ddm_sdv(const float *v, const float *a, const float *z, const float *t, const float *sv,
                const float *deadline, const float *s, int64_t n_trials, int64_t n_samples,
                const int64_t *sample_offsets, float max_t, float delta_t, int bound_kind,
                const float *bound_p1, const float *bound_p2, const float *bound_table,
                int64_t table_stride, int64_t table_len, uint64_t seed, int smooth_unif,
                const float *noise_rows, int64_t noise_row_len, const float *noise_unif, float *rts,
                int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                const ssm_launch *launch, void *workspace, size_t workspace_bytes, void *stream);

/*
 * ssm_full_ddm -- replaces cssm.full_ddm (src/cssm/ddm_models.pyx:2177-2497):
 * as ssm_ddm_sdv, plus a start point displaced by U(-sz, sz) and a
 * non-decision time displaced by U(-st, st) per trajectory (the deadline
 * horizon still uses t).  Noise injection: rows as ssm_ddm_sdv; three
 * uniforms per trajectory, noise_unif[3w .. 3w+2] = [u_t, u_y, u_jitter].
 */
int ssm_full_ddm(const float *v, const float *a, const float *z, const float *t, const float *sz,
                 const float *sv, const float *st, const float *deadline, const float *s,
                 int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets, float max_t,
                 float delta_t, int bound_kind, const float *bound_p1, const float *bound_p2,
                 const float *bound_table, int64_t table_stride, int64_t table_len, uint64_t seed,
                 int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                 const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
                 int64_t traj_len, const ssm_launch *launch, void *workspace,
                 size_t workspace_bytes, void *stream);

/*
 * ssm_ornstein_uhlenbeck -- replaces cssm.ornstein_uhlenbeck
 * (src/cssm/ornstein_models.pyx:47-330): y += (v - g y) dt + sqrt(dt) s N(0,1)
 * between +-b(t).  `a` is the boundary height (the reference passes it in
 * boundary_params).  Layout and noise conventions as ssm_ddm_flexbound.
 */
int ssm_ornstein_uhlenbeck(const float *v, const float *a, const float *z, const float *g,
                           const float *t, const float *deadline, const float *s, int64_t n_trials,
                           int64_t n_samples, const int64_t *sample_offsets, float max_t,
                           float delta_t, int bound_kind, const float *bound_p1,
                           const float *bound_p2, const float *bound_table, int64_t table_stride,
                           int64_t table_len, uint64_t seed, int smooth_unif,
                           const float *noise_rows, int64_t noise_row_len, const float *noise_unif,
                           float *rts, int32_t *choices, int32_t *steps, float *traj,
                           int64_t traj_len, const ssm_launch *launch, void *workspace,
                           size_t workspace_bytes, void *stream);

/*
 * ssm_ddm_flex -- replaces cssm.ddm_flex (src/cssm/ddm_models.pyx:884-1193):
 * the flexible-bound DDM with a time-varying drift, y += v(t_ix) dt +
 * sqrt(dt) s N(0,1).  drift_table holds each trial's drift function evaluated
 * on the time grid t_ix = ix * dt (float32 [n_trials * drift_stride],
 * drift_len entries per trial; later steps use the last entry); `v` is
 * accepted for the reference's signature and unused, the drift function
 * carries it.  Layout and noise conventions as ssm_ddm_flexbound.
 */
int ssm_ddm_flex(const float *v, const float *a, const float *z, const float *t, const float *deadline,
                 const float *s, int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets,
                 float max_t, float delta_t, int bound_kind, const float *bound_p1,
                 const float *bound_p2, const float *bound_table, int64_t table_stride,
                 int64_t table_len, const float *drift_table, int64_t drift_stride, int64_t drift_len,
                 uint64_t seed, int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                 const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
                 int64_t traj_len, const ssm_launch *launch, void *workspace,
                 size_t workspace_bytes, void *stream);

/*
 * ssm_drift_table -- the drift table ssm_ddm_flex reads, evaluated on the
 * device for the registered drift functions
 * (ssms/basic_simulators/drift_functions.py; registry in
 * ssms/config/_modelconfig/base.py).  Replaces the reference's per-trial
 * host evaluation drift_fun(t=t_s, **params_k)
 * (src/cssm/ddm_models.pyx:1063-1066) for the device-RNG path: one thread per
 * (trial, time) entry with the reference's float32 / float64 operation order;
 * values agree with numpy's to a few float32 ulps (the math library
 * differs).  params: float32 [n_params][n_trials] in the registry's parameter
 * order for `kind` (SSM_DRIFT_*); t_s: float32 [t_len], increasing; table:
 * float32 [n_trials * stride], entries t_len .. stride-1 of each row zeroed.
 */
#define SSM_DRIFT_CONSTANT 0              /* v */
#define SSM_DRIFT_GAMMA 1                 /* v, shape, scale, c */
#define SSM_DRIFT_CONFLICT_DS 2           /* v, tinit, dinit, tslope, dslope, tfixedp, tcoh, dcoh */
#define SSM_DRIFT_CONFLICT_DSSTIMFLEX 3   /* ... conflict_ds + tonset, donset (onsets relative to the first) */
#define SSM_DRIFT_CONFLICT_STIMFLEX 4     /* v, vt, vd, tcoh, dcoh, tonset, donset */
#define SSM_DRIFT_CONFLICT_STIMFLEXREL1 5 /* as STIMFLEX, onsets relative to the first */
#define SSM_DRIFT_ATTEND 6                /* v, ptarget, pouter, pinner, r, sda */
#define SSM_DRIFT_ATTEND_SIMPLE 7         /* v, ptarget, pouter, r, sda */
int ssm_drift_table(int kind, const float *params, int n_params, int64_t n_trials, const float *t_s,
                    int64_t t_len, float *table, int64_t stride, void *stream);

/* ---- multi-accumulator race / LCA --------------------------------------- */

/* Bytes of scratch ssm_race_model / ssm_lca need. */
size_t ssm_race_workspace_bytes(int64_t n_trials, int n_particles);

/*
 * ssm_race_model -- replaces cssm.race_model (src/cssm/race_models.pyx:141-506,
 * sequential loop :417-464).  n_particles accumulators start at z_j b(0); while
 * no accumulator exceeds b(t) and t <= min(max_t, deadline - t_nd), each
 * does x_j = max(0, x_j + v_j dt + sqrt(dt) s_j g_j).  choice = argmax_j x_j.
 * v, z, s: float32[n_trials * n_particles] (row-major); t, deadline: [n_trials].
 * Boundary: a (+ bound_p1 / bound_p2) or a table, as for ssm_ddm_flexbound.
 * Injected rows hold n_particles increments per step (index step*np + j).
 */
int ssm_race_model(const float *v, const float *z, const float *t, const float *s,
                   const float *deadline, int64_t n_trials, int64_t n_samples, int n_particles,
                   const int64_t *sample_offsets, float max_t, float delta_t, int bound_kind,
                   const float *a, const float *bound_p1, const float *bound_p2,
                   const float *bound_table, int64_t table_stride, int64_t table_len,
                   uint64_t seed, int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                   const float *noise_unif, float *rts, int32_t *choices, int32_t *steps,
                   float *traj, int64_t traj_len, const ssm_launch *launch, void *workspace,
                   size_t workspace_bytes, void *stream);

/*
 * ssm_lca -- replaces cssm.lca (src/cssm/race_models.pyx:509-920, sequential
 * loop :825-879): as the race with leak g and lateral inhibition b,
 * x_j += ((v_j - g x_j) - b (sum - x_j)) dt + sqrt(dt) s_j g_j, clipped at 0; the
 * time accumulator is double precision as in the reference.  g, b: [n_trials].
 */
int ssm_lca(const float *v, const float *z, const float *g, const float *b, const float *t,
            const float *s, const float *deadline, int64_t n_trials, int64_t n_samples,
            int n_particles, const int64_t *sample_offsets, float max_t, float delta_t,
            int bound_kind, const float *a, const float *bound_p1, const float *bound_p2,
            const float *bound_table, int64_t table_stride, int64_t table_len, uint64_t seed,
            int smooth_unif, const float *noise_rows, int64_t noise_row_len,
            const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
            int64_t traj_len, const ssm_launch *launch, void *workspace, size_t workspace_bytes,
            void *stream);

/*
 * ssm_racing_diffusion -- replaces cssm.racing_diffusion_model
 * (src/cssm/race_models.pyx:925-1300): n_particles Wiener accumulators
 * starting at U(0, A) race to one threshold b without a lower barrier; the
 * first one (in index order) at or above b wins, and the step that reaches it
 * does not advance the time.  v: float32 [n_trials, n_particles]; b, A, t, s:
 * one value per trial.  Choices 0..n_particles-1, -1 with rt -999 when no
 * accumulator wins before the deadline.  Noise injection: row w holds the
 * increments step-major (step * n_particles + j); noise_unif holds
 * n_particles + 1 values per trajectory, the start uniforms then the jitter
 * uniform.  Workspace: ssm_race_workspace_bytes.
 */
int ssm_racing_diffusion(const float *v, const float *b, const float *A, const float *t, const float *s,
                         const float *deadline, int64_t n_trials, int64_t n_samples, int n_particles,
                         const int64_t *sample_offsets, float max_t, float delta_t, uint64_t seed,
                         int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                         const float *noise_unif, float *rts, int32_t *choices, int32_t *steps,
                         float *traj, int64_t traj_len, const ssm_launch *launch, void *workspace,
                         size_t workspace_bytes, void *stream);

/*
 * ssm_lba_vanilla -- replaces cssm.lba_vanilla (src/cssm/lba_models.pyx:36-139):
 * per sample x_j = (a - U(0, z)) / |N(v_j, sd_j)|, choice = argmin_j x_j,
 * rt = min_j x_j + t, rt = -999 when rt >= deadline.  v, sd: float32[n_trials *
 * nact]; a, z, t, deadline: [n_trials].  noise_u / noise_g (both or neither):
 * injected U(0,1) and N(0,1) draws, float32[total * nact].  No workspace.
 */
int ssm_lba_vanilla(const float *v, const float *a, const float *z, const float *deadline,
                    const float *sd, const float *t, int64_t n_trials, int64_t n_samples, int nact,
                    const int64_t *sample_offsets, uint64_t seed, const float *noise_u,
                    const float *noise_g, float *rts, int32_t *choices, void *stream);

/* ---- log-rt Gaussian KDE (batched over parameter sets) ------------------ */
/*
 * ssm_kde_fit -- replaces LogKDE.__init__ / _attach_data_from_simulator /
 * compute_bandwidths (ssms/support_utils/kde_class.py:48-186, 438-504) and
 * bandwidth_silverman (:508-553) for n_sets simulated data sets at once.
 * Set s owns rts/choices [sample_offsets[s], sample_offsets[s+1]).  Group
 * g = s * n_choices + c collects log(rt - displace[s]) of the set's
 * non-omitted samples with choice choice_values[c] into
 * points[point_offsets[g] .. point_offsets[g+1]) (sample order), and gets
 * count_all (omissions included), n_valid, proportion = count_all / n,
 * bandwidth (Silverman on the group's log-rts, -1 when empty) and
 * log_norm = log p - log n - log h - log(2 pi)/2.  points must hold the
 * sets' total sample count.  displace (float64 per set) may be NULL; when
 * given, displaced_logs (float64, total samples) receives the values the
 * reference's bandwidth is computed from, log(exp(log_f32 rt) - displace).
 */
int ssm_kde_fit(const float *rts, const int32_t *choices, int64_t n_sets,
                const int64_t *sample_offsets, const int32_t *choice_values, int n_choices,
                const double *displace, double *displaced_logs, int64_t *count_all,
                int64_t *n_valid, int64_t *point_offsets, float *points, double *bandwidth,
                double *log_norm, double *proportion, void *stream);

/*
 * ssm_kde_eval -- replaces LogKDE.kde_eval (kde_class.py:188-329): for each
 * query (rt, group), queries sorted by group with query_offsets[G+1] and
 * n_queries = query_offsets[G], loglik = log_norm + log sum_j exp(-(q - x_j)^2
 * / 2h^2) - q with q = log(max(rt - displace, eps)); lb where that is <= lb or
 * rt - displace <= 0; -log(n_set * max_t) for groups without data.  float64
 * output.  The work is spread evenly over a persistent grid whatever the
 * groups' sizes; workspace (256-byte aligned, contents need not be cleared)
 * must hold ssm_kde_eval_workspace_bytes(n_sets, n_choices, n_queries) bytes,
 * computed with the same device current.  Results are deterministic.
 */
size_t ssm_kde_eval_workspace_bytes(int64_t n_sets, int n_choices, int64_t n_queries);
int ssm_kde_eval(const float *points, const int64_t *point_offsets, const double *bandwidth,
                 const double *log_norm, int64_t n_sets, int n_choices,
                 const int64_t *sample_offsets, const double *displace,
                 const int64_t *query_offsets, const double *query_rt, int64_t n_queries, double lb,
                 double eps, double max_t, void *workspace, size_t workspace_bytes,
                 double *out_loglik, void *stream);

/*
 * ssm_kde_sample -- replaces LogKDE.kde_sample's per-choice draws
 * (kde_class.py:331-434; KernelDensity.sample for a Gaussian kernel): group g
 * fills out_rt[out_offsets[g] ..]: the first n_kde[g] slots with
 * exp(x_J + h N(0,1)) + displace (J uniform over the group's points; U(0,
 * max_t) + displace when the group is empty), the remaining slots with
 * U(unif_lo, unif_hi) rts (the mixture's uniform component).
 */
int ssm_kde_sample(const float *points, const int64_t *point_offsets, const double *bandwidth,
                   int64_t n_sets, int n_choices, const double *displace,
                   const int64_t *out_offsets, const int64_t *n_kde, uint64_t seed, double max_t,
                   double unif_lo, double unif_hi, double *out_rt, void *stream);

/*
 * ssm_kde_records -- the row layout of ResampleMixtureStrategy.generate
 * (ssms/dataset_generators/strategies/resample_mixture_strategy.py:64-214):
 * per set, rows [theta..., rt, choice, loglik] (float32) for its evaluated
 * queries plus n_down rows with rt ~ U(-1, 0.0001) and loglik =
 * negative_rt_loglik, shuffled within the set.  rows_per_set <= 12288.
 */
int ssm_kde_records(const float *theta, int n_params, int64_t n_sets, int n_choices,
                    const int32_t *choice_values, const int64_t *query_offsets,
                    const double *query_rt, const double *query_loglik, int64_t n_down,
                    int64_t rows_per_set, float negative_rt_loglik, uint64_t seed, float *out,
                    void *stream);

/*
 * ssm_set_summary -- the auxiliary labels of SimulationPipeline
 * (ssms/dataset_generators/pipelines/simulation_pipeline.py:262-351) per set:
 * choice counts [n_sets * n_choices], no-go counts ((choice != max choice) or
 * rt == -999), omission counts (choices equal to -999, as the pipeline counts
 * them) and per-choice rt histograms with np.histogram's rules over
 * np.linspace(0, max_t, nbins + 1), omissions excluded, laid out
 * [n_sets, nbins, n_choices].
 */
int ssm_set_summary(const float *rts, const int32_t *choices, int64_t n_sets,
                    const int64_t *sample_offsets, const int32_t *choice_values, int n_choices,
                    double max_t, int64_t *choice_counts, int64_t *nogo_counts,
                    int64_t *omission_counts, int nbins_a, float *hist_a, int nbins_b,
                    float *hist_b, void *stream);

/*
 * ssm_simulator_summary -- the derived outputs of simulator()
 * (ssms/basic_simulators/simulator.py:806-863) and its pooled rt histograms
 * (bin_simulator_output, simulator.py:435-497) for an output in the reference
 * layout (index n * n_trials + k): per trial, choice counts [n_trials,
 * n_choices], choice counts among non-omitted samples, omission counts (rt ==
 * -999) and no-go counts (choice != the largest choice value, or omitted);
 * pooled over all trials, per-choice histograms [nbins, n_choices] of the
 * non-omitted rts with numpy.histogram's rule on the float64 bin edges
 * (nbins + 1 of them; the last may be +inf).  Counters are int64 and cleared
 * by the call.
 */
int ssm_simulator_summary(const float *rts, const int32_t *choices, int64_t n_samples, int64_t n_trials,
                          const int32_t *choice_values, int n_choices, const double *edges_a, int nbins_a,
                          const double *edges_b, int nbins_b, int64_t *choice_counts, int64_t *kept_counts,
                          int64_t *omission_counts, int64_t *nogo_counts, int64_t *hist_a, int64_t *hist_b,
                          void *stream);

/*
 * ssm_ddm_flexbound_static -- no counterpart in the reference.  The same
 * simulation as ssm_ddm_flexbound for callers that cannot allocate device
 * memory (for example code running inside an allocator-free host plugin, or a
 * caller whose memory pool is owned by someone else): it takes no workspace.
 * Its scratch (work counter, error word and one 64-byte row per trial) lives in
 * a file-scope __device__ array of SSM_STATIC_WS_BYTES bytes that every GPU
 * loading this library holds until the process exits; n_trials above
 * SSM_STATIC_MAX_TRIALS is rejected with SSM_ERR_ARG.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current, so make that first call before any stream capture.  The
 * address is cached per device with the id of the CUDA context it belongs to;
 * after a cudaDeviceReset (a new context) the next call looks it up again,
 * and that call, too, belongs before any stream capture.  Every
 * call shares the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller.  Device-side
 * error flags of this variant are not reported; use the workspace form when
 * they are needed.  The caller still owns every input and output buffer.
 */
#define SSM_STATIC_MAX_TRIALS 16384
#define SSM_STATIC_WS_BYTES (256 + 64 * SSM_STATIC_MAX_TRIALS)
int ssm_ddm_flexbound_static(const float *v, const float *a, const float *z, const float *t,
                             const float *deadline, const float *s, int64_t n_trials,
                             int64_t n_samples, const int64_t *sample_offsets, float max_t,
                             const float *max_t_per_trial, float delta_t, int bound_kind,
                             const float *bound_p1, const float *bound_p2,
                             const float *bound_table, int64_t table_stride, int64_t table_len,
                             uint64_t seed, int smooth_unif, const float *noise_rows,
                             int64_t noise_row_len, const float *noise_unif, float *rts,
                             int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                             const ssm_launch *launch, void *stream);

/*
 * ssm_ddm_nf_loglik -- no counterpart in the reference.  float64
 * Navarro-Fuss log-density of (rt, choice) under the constant-bound DDM in
 * the reference's parameterisation (bounds +-a, start -a + 2 z a, choice +1 at
 * the upper bound, non-decision t, noise s; src/cssm/ddm_models.pyx ddm /
 * ddm_flexbound), and with out_grad != NULL its gradient [n, 4] w.r.t.
 * (v, a, z, t).  Parameters are arrays of n entries (per_query_params = 1) or
 * single values (0); s may be NULL (unit noise).  rt <= t gives -inf (NaN
 * gradient).  eps is the series truncation error (1e-14 typical).
 */
int ssm_ddm_nf_loglik(const double *rt, const int32_t *choice, const double *v, const double *a,
                      const double *z, const double *t, const double *s, int64_t n,
                      int per_query_params, double eps, double *out_loglik, double *out_grad,
                      void *stream);

/*
 * Likelihood surrogate -- no counterpart in the reference, which only writes
 * the (theta, rt, choice, loglik) training records
 * (ssms/dataset_generators/lan_mlp.py:66-133, the records of
 * ResampleMixtureStrategy) for a network trained elsewhere.  A 7 -> 100 ->
 * 100 -> 120 -> 1 tanh MLP: layers 1-3 run on the tensor cores with bf16
 * weights and activations and fp32 accumulation, the 120 -> 1 output layer in
 * fp32.  Inputs are [theta(5), rt, choice] rows, normalised as
 * (x - norm_c[j]) * norm_s[j] before the first layer.
 *
 * Parameters live in one fp32 vector of SSM_MLP_NPARAMS floats in nn.Linear
 * order (W1[100,7], b1, W2[100,100], b2, W3[120,100], b3, w4[120], b4).  The
 * kernels read a packed image of SSM_MLP_IMAGE_BYTES bytes (16-byte aligned)
 * made by ssm_mlp_pack and kept current by ssm_mlp_adam.  `status` (device int,
 * may be NULL) receives SSM_MLP_ERR_TIMEOUT if a bounded wait expired.
 */
#define SSM_MLP_NPARAMS 23141
#define SSM_MLP_PARTIAL_STRIDE 23168 /* floats per per-CTA gradient partial */
#define SSM_MLP_IMAGE_BYTES 59280
#define SSM_MLP_ERR_TIMEOUT 7
int ssm_mlp_pack(const float *params, void *image, void *stream);

/* out[i] = net(x[i]); with dx != NULL also dx[i, 0:7] = d out[i] / d x[i]. */
int ssm_mlp_forward(const void *image, const float *x, int64_t n, int x_stride,
                    const float *norm_c, const float *norm_s, float *out, float *dx,
                    int dx_stride, int max_ctas, int *status, void *stream);

/*
 * One training gradient: records [n, rec_stride] = (x[0:7], target); loss
 * Huber(delta 1) (loss_kind 0) or squared error (1) times inv_batch, summed.
 * Each of n_ctas CTAs writes its gradient over its rows to
 * partials[cta * SSM_MLP_PARTIAL_STRIDE + p] and its loss sum (before
 * inv_batch) to loss_partials[cta]; out (may be NULL) receives predictions.
 */
int ssm_mlp_train_grad(const void *image, const float *records, int64_t n, int rec_stride,
                       const float *norm_c, const float *norm_s, int loss_kind, float inv_batch,
                       float *out, float *partials, float *loss_partials, int n_ctas,
                       int *status, void *stream);

/* Adam (Kingma & Ba) on the summed partials; bias_corr_k = 1 - beta_k^step. */
int ssm_mlp_adam(float *params, float *m, float *v, const float *partials, int n_partials,
                 float lr, float beta1, float beta2, float eps, float bias_corr1,
                 float bias_corr2, void *image, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SSM_B200_H */
