// Single-accumulator Euler-Maruyama simulators for sm_100a: the flexible-bound
// DDM (cssm.ddm_flexbound), the legacy [0, a] DDM (cssm.ddm) and the Levy
// flight DDM (cssm.levy_flexbound).
//
// Design (one thread per trajectory, persistent grid):
//  * A per-trial prologue (k_prep) turns the reference's per-trial arrays into
//    a 64-byte TrialRow with every derived float computed once, in the same
//    IEEE operation order the reference uses (src/cssm/ddm_models.pyx:700-744).
//  * The main kernel runs one grid of resident CTAs.  Each warp claims
//    trajectories from a global work counter in chunks; once refill_min of
//    its lanes have ended their walks (ballot), it writes their results and
//    hands them the next trajectories of its chunk (popc rank) in one
//    divergent pass, so that pass is paid once per several trajectories and
//    an ended lane idles for a few blocks at most.
//  * Steps run in blocks of 36 (24 for ddm_flex with a Weibull or table
//    bound, 8 for Levy): six independent Philox4x32-10 calls yield 24 words =
//    18 Box-Muller pairs = the block's increments, already scaled to drift +
//    s sqrt(dt) N(0,1), each call drawn in the step loop just before the six
//    steps that use it; the steps themselves are predicated (no per-step
//    branch), and a warp whose walks cannot reach their time limit within the
//    block skips the time test.
//  * A launch with about as many trajectories as the grid has lanes lasts as
//    long as its longest walk.  There W = 2, 4 or 8 lanes share a walk
//    (ssm_launch.lanes_per_walk, wide_block): each draws a third of the
//    block's increments and all step it, bit-identical to one lane per walk.
//  * Boundaries are evaluated in registers (constant / linear collapse /
//    Weibull) or read from a caller-evaluated table for arbitrary shapes.
//  * Noise injection replaces the generator by caller rows and switches every
//    float operation to explicit round-to-nearest intrinsics, giving results
//    bit-identical to the sequential CPU restatement.
#include <cuda.h>  // CUcontext / CUresult types of the driver entry points below

#include <mutex>

#include "common.cuh"





namespace ssm {

// M_SDV: ddm_sdv (drift v + sv N(0,1) per trajectory); M_FULL: full_ddm (and
// start point + U(-sz, sz), non-decision time + U(-st, st)); M_OU:
// ornstein_uhlenbeck (drift v - g y); M_DFLEX: ddm_flex (drift v(t) from a
// per-trial table the host evaluates from the drift function).
enum Model { M_FLEX = 0, M_LEGACY = 1, M_LEVY = 2, M_SDV = 3, M_FULL = 4, M_OU = 5, M_DFLEX = 6 };

struct alignas(16) TrialRow {
    float drift;     // v * dt ; SDV/FULL: v
    float scale;     // sqrt(dt) * s ;  Levy: s * dt^(1/alpha)
    float y0;        // start point
    float dl_tmp;    // min(max_t, deadline - t): the walk runs while t <= dl_tmp
    float t;         // non-decision time
    float deadline;  // rt >= deadline (or deadline <= 0) -> omission
    float a;         // boundary height (legacy DDM: upper bound)
    float p1;        // LINEAR: slope ; WEIBULL: shape alpha
    float p2;        // WEIBULL: scale beta
    float dtp1;      // dt * p1 (linear boundary per step, fast path)
    float inv_beta;  // 1 / beta
    float alpha;     // Levy: stability index ; SDV/FULL: sv ; OU: v
    float inv_alpha; // Levy: 1 / alpha ; FULL: sz ; OU: g
    float expo;      // Levy: (1 - alpha) / alpha ; FULL: st ; OU: 1 - g dt
    float capf;      // hard limit on Euler steps: a walk reaching it raises SSM_ERR_DEVICE
    float c2;        // -2 ln(2) * scale^2: folds the noise scale into Box-Muller's radius
};
static_assert(sizeof(TrialRow) == 64, "TrialRow is one 64-byte line");

struct SingleParams {
    PhiloxKeys key;
    const TrialRow *rows;
    const int64_t *offsets;  // ragged prefix sums (n_trials + 1) or nullptr
    const int32_t *order;    // ragged only: trial simulated j-th (nullptr = index order)
    const int64_t *qoff;     // prefix sums of the sample counts in that order
    int64_t n_trials;
    int64_t total;           // number of trajectories; -1 = offsets[n_trials] - offsets[0]
    uint32_t k_base;         // random-stream index of trial 0 (trial windows of a larger batch)
    int ustride;             // injected uniforms per trajectory (3 for full_ddm: u_t, u_y, u_smooth)
    float dt;
    int smooth;
    int chunk;
    int refill_min;          // ended walks a warp collects before it restarts lanes
    const float *table;
    int64_t tstride, tlen;
    const float *dtable;     // DFLEX: drift v(t_ix) per trial, row stride dstride, dlen entries
    int64_t dstride, dlen;
    int dvec;                // rows 16-byte aligned: a block's drifts are float4 loads
    const float *noise;      // injected increments: row w holds nlen floats
    int64_t nlen;
    const float *nunif;      // injected jitter uniforms, one per trajectory
    float *rts;
    int32_t *choices;
    int32_t *steps;
    WorkspaceHeader *hdr;
    float *traj;             // trajectory recorder (record kernel only)
    int64_t traj_len;
};

struct PrepArgs {
    const float *v, *a, *z, *t, *deadline, *s, *alpha, *p1, *p2, *maxt_k, *table;
    const float *sv, *sz, *st, *g;  // variability (SDV/FULL) and leak (OU) parameters
    int64_t n_trials, tstride;
    float dt, sqrt_dt, max_t;
    int model, bound;
    TrialRow *rows;
};

// ------------------------------------------------------------------ prologue
__global__ void k_prep(const PrepArgs A) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.n_trials) return;
    TrialRow r;
    const float dt = A.dt;
    r.drift = __fmul_rn(A.v[k], dt);
    r.t = A.t[k];
    r.deadline = A.deadline[k];
    const float maxt = A.maxt_k ? A.maxt_k[k] : A.max_t;
    const float dl = __fsub_rn(r.deadline, r.t);
    r.dl_tmp = (dl < maxt) ? dl : maxt;  // src/cssm/_utils.pyx:712-718
    r.a = A.a ? A.a[k] : 0.f;
    r.p1 = A.p1 ? A.p1[k] : 0.f;
    r.p2 = A.p2 ? A.p2[k] : 1.f;
    r.dtp1 = dt * r.p1;
    r.inv_beta = 1.0f / r.p2;
    r.alpha = A.alpha ? A.alpha[k] : 2.f;
    r.inv_alpha = (float)(1.0 / (double)r.alpha);
    r.expo = (float)((1.0 - (double)r.alpha) / (double)r.alpha);
    if (A.model == M_SDV || A.model == M_FULL) {
        r.drift = A.v[k];  // the drift increment (v + sv g) dt is drawn per trajectory
        r.alpha = A.sv[k];
        r.inv_alpha = (A.model == M_FULL) ? A.sz[k] : 0.f;
        r.expo = (A.model == M_FULL) ? A.st[k] : 0.f;
    } else if (A.model == M_OU) {
        r.alpha = A.v[k];
        r.inv_alpha = A.g[k];
        r.expo = 1.0f - A.g[k] * dt;
    }
    // The walk stops once the float32 time passes dl_tmp, i.e. after about
    // dl_tmp/dt steps; twice that plus slack bounds every legal walk.  A stalled
    // accumulator (dt below half an ulp of t) or an infinite horizon hits the cap.
    const double nsteps = (double)r.dl_tmp / (double)dt;
    if (!(nsteps > 0.0)) r.capf = 64.f;                   // NaN or <= 0: at most one step
    else if (nsteps <= 8388608.0) r.capf = (float)(int)(2.0 * nsteps + 64.0);
    else r.capf = 0.f;                                    // unsupported horizon: flagged
    if (A.model == M_LEVY) {
        // delta_t_alpha = s * pow(delta_t, 1.0 / alpha) in double (levy_models.pyx:166)
        r.scale = __double2float_rn((double)A.s[k] * pow((double)dt, 1.0 / (double)r.alpha));
    } else {
        r.scale = __fmul_rn(A.sqrt_dt, A.s[k]);  // ddm_models.pyx:705
    }
    r.c2 = -1.3862944f * r.scale * r.scale;
    if (A.model == M_LEGACY) {
        r.y0 = __fmul_rn(A.z[k], r.a);  // ddm_models.pyx:451
    } else if (A.model == M_OU || A.model == M_DFLEX) {
        // (-1) * b0 + z * 2 * b0 with integer literals: float arithmetic
        // (ornstein_models.pyx:167, ddm_models.pyx:1014)
        const float b0 = (A.bound == SSM_BOUND_TABLE) ? A.table[k * A.tstride] : r.a;
        r.y0 = __fadd_rn(-b0, __fmul_rn(__fmul_rn(A.z[k], 2.0f), b0));
    } else {
        const float b0 = (A.bound == SSM_BOUND_TABLE) ? A.table[k * A.tstride] : r.a;
        // -b0 + z*2*b0, evaluated in double as the generated C does (ddm_models.pyx:709)
        const double bd = (double)b0;
        r.y0 = __double2float_rn(__dadd_rn(-bd, __dmul_rn(__dmul_rn((double)A.z[k], 2.0), bd)));
    }
    reinterpret_cast<TrialRow *>(A.rows)[k] = r;
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ int64_t ragged_find(const int64_t *off, int64_t K, int64_t w,
                                               int64_t hint) {
    int64_t k = hint;
    if (k < 0 || k >= K || __ldg(off + k) > w) k = 0;
    int64_t step = 1;
    while (k + step < K && __ldg(off + k + step) <= w) {
        k += step;
        step <<= 1;
    }
    int64_t hi = (k + step < K) ? k + step : K;
    while (hi - k > 1) {
        const int64_t mid = (k + hi) >> 1;
        if (__ldg(off + mid) <= w) k = mid; else hi = mid;
    }
    return k;
}

template <int BOUND, bool EXACT>
__device__ __forceinline__ float bound_at(const TrialRow &r, float ixf, int ix,
                                          const SingleParams &p, int64_t k) {
    if (BOUND == SSM_BOUND_CONSTANT) {
        return r.a;
    } else if (BOUND == SSM_BOUND_LINEAR) {
        // table value a + f32(ix*dt) * p1 (boundary_functions.py:57-72 on t_s)
        if (EXACT) return __fadd_rn(r.a, __fmul_rn(__fmul_rn(ixf, p.dt), r.p1));
        return fmaf(ixf, r.dtp1, r.a);
    } else if (BOUND == SSM_BOUND_WEIBULL) {
        // a * exp(-(t/beta)^alpha) (boundary_functions.py:103-122)
        const float x = ixf * p.dt * r.inv_beta;
        const float pw = (x > 0.f) ? exp2f(r.p1 * __log2f(x)) : 0.f;
        return r.a * __expf(-pw);
    } else {
        const int64_t i = (ix < p.tlen) ? ix : p.tlen - 1;
        return __ldg(p.table + k * p.tstride + i);
    }
}

// sin x and cos x on [0, pi/2] from their Taylor series through x^11 and x^12
// (truncation errors below 6e-8 and 7e-9 there): short branch-free code for
// the stable sampler, whose angles are always reduced to that interval.
__device__ __forceinline__ float sin_q(float x) {
    const float t = x * x;
    float p = fmaf(t, -2.5052108e-08f, 2.7557319e-06f);  // -1/11!, 1/9!
    p = fmaf(t, p, -1.9841270e-04f);                     // -1/7!
    p = fmaf(t, p, 8.3333333e-03f);                      // 1/5!
    p = fmaf(t, p, -1.6666667e-01f);                     // -1/3!
    p = fmaf(t, p, 1.0f);
    return x * p;
}
__device__ __forceinline__ float cos_q(float x) {
    const float t = x * x;
    float p = fmaf(t, 2.0876757e-09f, -2.7557319e-07f);  // 1/12!, -1/10!
    p = fmaf(t, p, 2.4801587e-05f);                      // 1/8!
    p = fmaf(t, p, -1.3888889e-03f);                     // -1/6!
    p = fmaf(t, p, 4.1666667e-02f);                      // 1/4!
    p = fmaf(t, p, -0.5f);
    return fmaf(t, p, 1.0f);
}

// Symmetric alpha-stable variate by Chambers-Mallows-Stuck (Chambers, Mallows
// & Stuck, JASA 71, 1976) with the reference's guards (_utils.pyx:426-472):
// U ~ U(-pi/2 + 1e-7, pi/2 - 1e-7), W ~ Exp(1) floored at 1e-10, output
// clipped to +-1e10 and NaN -> 0.
//   X = sin(alpha U) / cos(U)^(1/alpha) * (cos((1 - alpha) U) / W)^((1 - alpha) / alpha)
// (tan U for alpha = 1).  U = pi (u - 1/2) with u on a 2^-23 grid; the sampler
// works with |U| and its complement V = pi/2 - |U| = pi min(u, 1 - u), which
// carries one rounding only, so cos U = sin V keeps its relative precision as
// |U| -> pi/2, where the heavy tail comes from.  Both powers are taken as one
// power of two.
__device__ __forceinline__ float cms_stable(uint32_t bu, uint32_t bw, const TrialRow &r) {
    const float u01 = bits_to_1_2(bu) - 1.0f;
    const float m = fmaxf(0.5f - fabsf(u01 - 0.5f), 3.1830988e-08f);  // V >= 1e-7 (the U clamp)
    const float V = 3.14159265f * m;
    const float aU = 1.57079633f - V;  // |U|
    const float W = fmaxf(-0.69314718f * lg2_ftz(uniform_open(bw)), 1e-10f);
    float X;
    if (r.alpha == 1.0f) {
        X = cos_q(V) / sin_q(V);  // |tan U|
    } else {
        const float cu = sin_q(V);                                             // cos U > 0
        // cos((1 - alpha) U) = cos(c |U|), c = |1 - alpha| <= 1, evaluated as
        // sin(pi/2 - c |U|) = sin(pi/2 (1 - c) + c V): two non-negative terms,
        // so the argument does not cancel, and one polynomial serves every c |U|
        const float c = fabsf(1.0f - r.alpha);
        const float cua = fmaxf(sin_q(fmaf(c, V, 1.57079633f * (1.0f - c))), 1e-10f);
        // alpha |U| in [0, pi); past pi/2 use pi - alpha |U| = pi (1 - alpha/2) + alpha V,
        // which does not cancel as alpha -> 2
        float A = r.alpha * aU;
        if (A > 1.57079633f) A = fmaf(r.alpha, V, 3.14159265f * fmaf(-0.5f, r.alpha, 1.0f));
        const float e = fmaf(r.expo, lg2_ftz(cua) - lg2_ftz(W), -r.inv_alpha * lg2_ftz(cu));
        float p2;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(p2) : "f"(e));
        X = sin_q(A) * p2;  // |sin(alpha U)| ...
    }
    X = (u01 < 0.5f) ? -X : X;  // ... times sign(U): every factor but sin(alpha U) is even in U
    if (X != X) X = 0.f;
    return fminf(fmaxf(X, -1e10f), 1e10f);
}

// Euler steps per block.  The Gaussian models draw six increments per
// Philox4x32-10 call (three Box-Muller pairs, see bm6_increment), so a
// 36-step block makes six independent Philox calls whose latencies overlap.
// Measured on the 4096-set angle batch on one B200 (ms per launch): six per
// call with 24-step blocks 27.8, 36 steps 26.8, 48 steps 27.0 (all 80
// registers, 3 CTAs per SM; 4 CTAs per SM at 64 registers 27.3 for 24 and 36
// steps); four per call with 32-step blocks 31.2.  With the re-tuned launch
// (128 threads, claims of 256): 30 steps 26.95, 36 steps 26.54, 42 steps
// 26.39, but on 1024 sets 42 steps is the slower (8.02 against 7.92 ms).
// ddm_flex holds a block's table drifts in registers as well: with the
// increments drawn a block at a time, 24 steps (four Philox calls, six float4
// drift loads) took 14.46 ms on the 1 024 conflict_ds sets against 15.73 for
// 12 steps and 16.51 for 16-step blocks of four increments per call (36 steps
// spilled).  With the draws fused into the steps (step_block FUSE) 36 steps
// fit for the constant and linear bounds (11.42 -> 11.00 ms against 24); the
// Weibull and table bounds keep 24 (at 36 the Weibull bound spills 294 bytes).
// The Levy model keeps 8-step blocks (its stable draws already give each
// block enough independent work; 16-step blocks measured 8 % slower there).
// Call h of block b uses counter (BLK/6) b + h, so a stream does not depend
// on the block length.
template <int MODEL, int BOUND = SSM_BOUND_CONSTANT> struct Blk {
    static constexpr int value =
        (MODEL == M_LEVY) ? 8
                          : ((MODEL == M_DFLEX && BOUND != SSM_BOUND_CONSTANT && BOUND != SSM_BOUND_LINEAR) ? 24 : 36);
};
// Lanes per walk W (see wide_block): 1 is the throughput mode above; W = 2,
// 4, 8 give each trajectory an aligned group of W lanes and blocks of 18 W
// steps, three Philox calls per lane.
template <int MODEL, int W, int BOUND = SSM_BOUND_CONSTANT> struct BlkW {
    static constexpr int value = (W == 1) ? Blk<MODEL, BOUND>::value : 18 * W;
};
// Device-RNG Gaussian models draw their increments inside the step loop
// (step_block FUSE).  Outputs are bit-identical to drawing the block first;
// measured on one B200 (ms per launch): 4 096-set angle batch 26.43 -> 26.33
// (80 -> 64 registers), 1 024 conflict_ds sets 12.29 -> 11.42 (its 52-62 bytes
// of spills gone), Ornstein 20.70 -> 20.41.
template <int MODEL, bool NOISE> struct FuseOk {
    static constexpr bool value = !NOISE && MODEL != M_LEVY;
};
template <int MODEL, bool NOISE, int BOUND> struct WideOk {
    static constexpr bool value =
        !NOISE && MODEL != M_LEVY && MODEL != M_DFLEX && BOUND != SSM_BOUND_TABLE;
};
// Resident 256-thread CTAs per SM the compiler must fit (register cap
// 65536 / (256 n)): 3 (80 registers) for blocks longer than 8 steps, 4 otherwise
// (and 4 for the lanes-per-walk mode, whose lanes hold 18 increments).
template <int MODEL, int W = 1> struct MinCtas {
    static constexpr int value = (W == 1 && Blk<MODEL>::value > 8) ? 3 : 4;
};

struct Lane {
    int64_t w;
    uint32_t k, n, blk;
    int ix;           // steps taken (maintained where an integer index is needed)
    float y, tp, ixf; // position, float32 time accumulator, steps taken as float (see step_block)
    float tpb;        // time accumulator at the start of the current block
    float dinc;       // SDV/FULL: this trajectory's drift increment (v + sv g) dt
};

// models whose drift is drawn once per trajectory
template <int MODEL> struct DrawnDrift { static constexpr bool value = (MODEL == M_SDV || MODEL == M_FULL); };

// Increments 6h .. 6h+5 of the lane's current block from the device RNG
// (Gaussian models): Philox call (BLK/6) blk + h of the trajectory's stream.
template <int MODEL, int BOUND>
__device__ __forceinline__ void draw_call(const SingleParams &p, const Lane &L, const TrialRow &r, int h,
                                          float *g6) {
    constexpr int BLK = Blk<MODEL, BOUND>::value;
    // ddm_flex: drift 0 here, v(t_ix) dt from the table in the step
    const float drift = (MODEL == M_DFLEX) ? 0.f : (DrawnDrift<MODEL>::value ? L.dinc : r.drift);
    const uint4 b = philox10(make_uint4((uint32_t)(BLK / 6) * L.blk + (uint32_t)h, L.n, L.k + p.k_base, 0u),
                             p.key);
    bm6_increment(b, r.c2, drift, g6);
}

// The block's increments.  Noise injection returns the raw caller draws (the
// step applies drift and scale with explicit rounding); the device RNG returns
// finished increments drift + scale * X.
template <int MODEL, int BOUND, bool NOISE>
__device__ __forceinline__ void draw_block(const SingleParams &p, const Lane &L, const TrialRow &r,
                                           float g[Blk<MODEL, BOUND>::value]) {
    constexpr int BLK = Blk<MODEL, BOUND>::value;
    if (NOISE) {
        // SDV/FULL rows start with the trajectory's drift normal
        constexpr int OFF = DrawnDrift<MODEL>::value ? 1 : 0;
        const float *row = p.noise + L.w * p.nlen + OFF;
#pragma unroll
        for (int q = 0; q < BLK; ++q) g[q] = (L.ix + OFF + q < p.nlen) ? __ldg(row + L.ix + q) : 0.f;
    } else if (MODEL == M_LEVY) {
#pragma unroll
        for (int h = 0; h < BLK / 2; h += 2) {
            const uint4 b = philox10(make_uint4(L.blk, L.n, L.k + p.k_base, 2u + (uint32_t)h), p.key);
            g[2 * h + 0] = fmaf(r.scale, cms_stable(b.x, b.y, r), r.drift);
            g[2 * h + 1] = fmaf(r.scale, cms_stable(b.z, b.w, r), r.drift);
            const uint4 c = philox10(make_uint4(L.blk, L.n, L.k + p.k_base, 3u + (uint32_t)h), p.key);
            g[2 * h + 2] = fmaf(r.scale, cms_stable(c.x, c.y, r), r.drift);
            g[2 * h + 3] = fmaf(r.scale, cms_stable(c.z, c.w, r), r.drift);
        }
    } else {
        static_assert(MODEL == M_LEVY || BLK % 6 == 0, "six increments per Philox call");
#pragma unroll
        for (int h = 0; h < BLK / 6; ++h) draw_call<MODEL, BOUND>(p, L, r, h, g + 6 * h);
    }
}

// Advance one lane by up to BLK Euler steps.  Every step first tests the
// reference's `while` condition (ddm_models.pyx:719; legacy DDM :451); once it
// fails the remaining steps of the block are predicated off.  Returns whether
// the walk is still running.  With FUSE (device RNG, Gaussian models) the
// increments are drawn inside the step loop, six per Philox call (g unused):
// the same values as draw_block, with each call's draws in the same straight-
// line code as the steps, so their independent work fills the latency of the
// dependent step chain and only six increments are live at a time.
template <int MODEL, int BOUND, bool NOISE, bool RECORD, bool TCHK = true, bool FUSE = false>
__device__ __forceinline__ bool step_block(const SingleParams &p, Lane &L, const TrialRow &r,
                                           const float *g) {
    constexpr int BLK = Blk<MODEL, BOUND>::value;
    static_assert(!FUSE || (!NOISE && MODEL != M_LEVY), "fused draws: device RNG, Gaussian models");
    float g6[6];
    if (L.ixf >= r.capf) {
        raise_error(p.hdr, SSM_ERR_DEVICE, (int)L.w);
        return false;
    }
    constexpr bool INT_IX = NOISE || RECORD || BOUND == SSM_BOUND_TABLE;
    // Without an integer index (device RNG, in-register bounds) step q of the
    // block sits at step ixf0 + q: the step count advances once per block,
    // the linear bound is a + ixf0 slope dt plus q slope dt, and finalize()
    // recovers the steps of the last block from the time accumulator.
    const float ixf0 = L.ixf;
    const float b0 = (!INT_IX && BOUND == SSM_BOUND_LINEAR) ? fmaf(ixf0, r.dtp1, r.a) : 0.f;
    if (!INT_IX) L.tpb = L.tp;
    const float *drow = (MODEL == M_DFLEX) ? p.dtable + (int64_t)L.k * p.dstride : nullptr;
    // device RNG: the block's drifts v(t_ix .. t_ix+BLK-1) are read before
    // the steps, off the dependency chain (a live walk starts every block at
    // a multiple of BLK steps); past the table's end the last entry repeats
    float dvq[BLK];
    if (MODEL == M_DFLEX && !NOISE) {
        const int ix0 = INT_IX ? L.ix : (int)ixf0;  // the block's first step
        if (p.dvec && (ix0 & 3) == 0 && ix0 + BLK <= p.dlen) {
            const float4 *d4 = reinterpret_cast<const float4 *>(drow + ix0);
#pragma unroll
            for (int h = 0; h < BLK / 4; ++h) {
                const float4 a = __ldg(d4 + h);
                dvq[4 * h] = a.x; dvq[4 * h + 1] = a.y; dvq[4 * h + 2] = a.z; dvq[4 * h + 3] = a.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < BLK; ++q) dvq[q] = __ldg(drow + ((ix0 + q < p.dlen) ? ix0 + q : p.dlen - 1));
        }
    }
    bool live = true;
#pragma unroll
    for (int q = 0; q < BLK; ++q) {
        if (FUSE && q % 6 == 0) draw_call<MODEL, BOUND>(p, L, r, q / 6, g6);
        const float gq = FUSE ? g6[q % 6] : g[q];
        bool inside;
        // the time test; a block whose every step is known to pass it skips it (TCHK false)
        const bool in_time = !TCHK || (L.tp <= r.dl_tmp);
        if (MODEL == M_LEGACY) {
            inside = live && (L.y <= r.a) && (L.y >= 0.f) && in_time;
        } else {
            float b;
            if (INT_IX) b = bound_at<BOUND, NOISE>(r, L.ixf, L.ix, p, L.k);
            else if (BOUND == SSM_BOUND_LINEAR) b = (q == 0) ? b0 : fmaf((float)q, r.dtp1, b0);
            else b = bound_at<BOUND, NOISE>(r, ixf0 + (float)q, 0, p, L.k);
            inside = live && (fabsf(L.y) <= b) && in_time;
        }
        if (NOISE && inside && L.ix + (DrawnDrift<MODEL>::value ? 1 : 0) >= p.nlen) {
            raise_error(p.hdr, SSM_ERR_NOISE_RANGE, (int)L.w);
            inside = false;
        }
        if (inside) {
            if (NOISE) {
                if (MODEL == M_OU) {
                    // (y + (v - g y) dt) + scale*g (ornstein_models.pyx:177)
                    const float lk = __fmul_rn(__fsub_rn(r.alpha, __fmul_rn(r.inv_alpha, L.y)), p.dt);
                    L.y = __fadd_rn(__fadd_rn(L.y, lk), __fmul_rn(r.scale, gq));
                } else if (MODEL == M_DFLEX) {
                    // (y + v(t_ix) dt) + scale*g (ddm_models.pyx:1025)
                    const float dv = __ldg(drow + ((L.ix < p.dlen) ? L.ix : p.dlen - 1));
                    L.y = __fadd_rn(__fadd_rn(L.y, __fmul_rn(dv, p.dt)), __fmul_rn(r.scale, gq));
                } else {
                    // (y + v*dt) + scale*g: the association the reference build uses
                    const float dr = DrawnDrift<MODEL>::value ? L.dinc : r.drift;
                    L.y = __fadd_rn(__fadd_rn(L.y, dr), __fmul_rn(r.scale, gq));
                }
                L.tp = __fadd_rn(L.tp, p.dt);
            } else {
                if (MODEL == M_OU) L.y = fmaf(L.y, r.expo, gq);  // y (1 - g dt) + v dt + noise
                else if (MODEL == M_DFLEX)                          // y + v(t_ix) dt + noise
                    L.y += fmaf(dvq[q], p.dt, gq);
                else L.y += gq;
                L.tp += p.dt;
            }
            if (INT_IX) {
                L.ixf += 1.0f;
                L.ix += 1;
            }
            if (RECORD && L.ix < p.traj_len) p.traj[L.ix] = L.y;
        }
        live = inside;
    }
    if (!INT_IX) L.ixf = ixf0 + (float)BLK;
    return live;
}

// True when all BLK time tests of the lane's next block are known to pass
// (device RNG, in-register bounds only).  Step q of the block tests the float
// accumulator after q more additions of dt, at most t + (BLK-1) dt plus the
// additions' rounding; below 65536 dt an ulp of t is at most dt/64, so that
// rounding stays under dt/4, and t + (BLK+1) dt <= dl_tmp, evaluated in float,
// leaves more than that margin.
template <int MODEL, int BOUND, bool NOISE, int BLK = Blk<MODEL, BOUND>::value>
__device__ __forceinline__ bool block_in_time(const SingleParams &p, const Lane &L, const TrialRow &r) {
    constexpr bool INT_IX = NOISE || BOUND == SSM_BOUND_TABLE;
    if (INT_IX) return false;
    // longer blocks (lanes-per-walk mode, 36-144 steps) keep a margin of
    // 2 dt per 64 steps: past 65536 dt an addition rounds by up to dt/64
    constexpr float SPAN = (float)(BLK + 1 + 2 * (BLK / 64));
    return (L.tp < p.dt * 65536.f) && (fmaf(SPAN, p.dt, L.tp) <= r.dl_tmp);
}

// Steps taken by a walk that has ended.  Without an integer index L.ixf
// counts whole blocks; the steps of the last block are those that took the
// time accumulator from L.tpb to L.tp (the same float additions replayed).
template <int MODEL, int BOUND, bool NOISE, int BLK = Blk<MODEL, BOUND>::value>
__device__ __forceinline__ int steps_taken(const SingleParams &p, const Lane &L) {
    constexpr bool INT_IX = NOISE || BOUND == SSM_BOUND_TABLE;
    if (INT_IX) return (int)L.ixf;
    float tt = L.tpb;
    int c = 0;
    while (c < BLK && tt != L.tp) {
        tt += p.dt;
        ++c;
    }
    return (int)L.ixf - BLK + c;
}

template <int MODEL, int BOUND, bool NOISE, int BLK = Blk<MODEL, BOUND>::value>
__device__ __forceinline__ void finalize(const SingleParams &p, const Lane &L, bool writer = true) {
    // fields needed only here are re-read instead of being held across the walk
    const TrialRow *row = p.rows + L.k;
    const float t = __ldg(&row->t), deadline = __ldg(&row->deadline), dl = __ldg(&row->dl_tmp);
    float u;
    if (NOISE) u = __ldg(p.nunif + L.w * p.ustride + (p.ustride - 1));
    else u = uniform_co(philox10(make_uint4(0u, L.n, L.k + p.k_base, 1u), p.key).x);
    float tt = t;
    if (MODEL == M_FULL) {
        // t + 2 (u - 0.5) st in double (ddm_models.pyx:2253); the same uniform as at the start
        float ut;
        if (NOISE) ut = __ldg(p.nunif + L.w * p.ustride);
        else ut = uniform_co(philox10(make_uint4(0u, L.n, L.k + p.k_base, 3u), p.key).z);
        tt = __double2float_rn((double)t + (2.0 * ((double)ut - 0.5)) * (double)__ldg(&row->expo));
    }
    // compute_smooth_unif (_utils.pyx:668-695): double arithmetic, float result
    float sm = 0.f;
    if (p.smooth) {
        if (L.tp == 0.f) sm = __double2float_rn(((double)u * 0.5) * (double)p.dt);
        else if (L.tp < dl) sm = __double2float_rn((0.5 - (double)u) * (double)p.dt);
    }
    float rt = __fadd_rn(__fadd_rn(L.tp, tt), sm);
    if (rt >= deadline || deadline <= 0.f) rt = -999.f;  // enforce_deadline
    const int choice = (L.y > 0.f) - (L.y < 0.f);         // sign(y)
    if (!writer) return;
    p.rts[L.w] = rt;
    p.choices[L.w] = choice;
    if (p.steps) p.steps[L.w] = steps_taken<MODEL, BOUND, NOISE, BLK>(p, L);
}

// Start lane L on the trajectory with queue index w; false (and the error
// word set) if a caller-given processing order does not cover that index.
template <int MODEL, bool NOISE>
__device__ __forceinline__ bool lane_init(const SingleParams &p, Lane &L, TrialRow &r, int64_t w,
                                          int64_t &hint) {
    int64_t k, n;
    if (p.offsets == nullptr) {
        k = w % p.n_trials;
        n = w / p.n_trials;
    } else if (p.order != nullptr) {
        // queue index -> position j in the processing order -> trial k; the
        // output index stays offsets[k] + n, so results do not depend on the order
        const int64_t j = ragged_find(p.qoff, p.n_trials, w, hint);
        hint = j;
        k = __ldg(p.order + j);
        n = w - __ldg(p.qoff + j);
        if (k < 0 || k >= p.n_trials || n < 0 || n >= __ldg(p.offsets + k + 1) - __ldg(p.offsets + k)) {
            raise_error(p.hdr, SSM_ERR_ARG, (int)j);
            return false;
        }
        w = __ldg(p.offsets + k) + n;
    } else {
        w += __ldg(p.offsets);  // global output index (trial windows start past 0)
        k = ragged_find(p.offsets, p.n_trials, w, hint);
        n = w - __ldg(p.offsets + k);
        hint = k;
    }
    const float4 *src = reinterpret_cast<const float4 *>(p.rows + k);
    float4 *dst = reinterpret_cast<float4 *>(&r);
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[i] = __ldg(src + i);
    L.w = w;
    L.k = (uint32_t)k;
    L.n = (uint32_t)n;
    L.blk = 0;
    L.ix = 0;
    L.ixf = 0.f;
    L.tp = 0.f;
    L.y = r.y0;
    if (DrawnDrift<MODEL>::value) {
        // per-trajectory drift normal and (full_ddm) start-point uniform
        // (ddm_models.pyx:2249-2266): injected, or drawn from the trajectory's stream
        float g0, uy = 0.5f;
        if (NOISE) {
            g0 = __ldg(p.noise + L.w * p.nlen);
            if (MODEL == M_FULL) uy = __ldg(p.nunif + L.w * p.ustride + 1);
        } else {
            const uint4 b = philox10(make_uint4(0u, L.n, L.k + p.k_base, 3u), p.key);
            g0 = box_muller(b.x, b.y).x;
            uy = uniform_co(b.w);
        }
        L.dinc = __fmul_rn(__fadd_rn(r.drift, __fmul_rn(r.alpha, g0)), p.dt);
        if (MODEL == M_FULL)
            L.y = __double2float_rn((double)L.y + (2.0 * ((double)uy - 0.5)) * (double)r.inv_alpha);
    }
    return true;
}

// One block of the lanes-per-walk mode (W = 2, 4, 8; device RNG, in-register
// boundaries).  The W lanes of an aligned group carry one trajectory and
// hold identical state.  A block is 18 W steps: lane s of the group makes
// Philox calls 3 W b + 3 s + m (m = 0, 1, 2) of block b -- the counters the
// one-lane mode uses for the same steps -- and every lane of the group then
// runs the block's steps in order, each increment broadcast by a shuffle from
// the lane that drew it.  The warp issues about 8 instructions per step of
// 32 / W walks instead of about 21 per step of 32: throughput traded for the
// latency of one walk, which is what bounds a launch with fewer
// trajectories than resident lanes.  18 W is a multiple of 36, so the linear
// boundary comes from the same 36-step bases as in the one-lane mode and the
// results are bit-identical to it.  Every lane of the warp takes part (the
// shuffles need the whole warp); a lane without a running walk (`active`
// false, possibly still holding an ended walk's state for finalize) changes
// nothing.
template <int MODEL, int BOUND, bool TCHK, int W>
__device__ __forceinline__ bool wide_block(const SingleParams &p, Lane &L, const TrialRow &r, bool active,
                                           int src0, int sub) {
    static_assert(W == 2 || W == 4 || W == 8, "lanes per walk");
    constexpr int BLK = 18 * W;
    constexpr unsigned FULL = 0xffffffffu;
    const bool capped = active && L.ixf >= r.capf;
    if (capped) raise_error(p.hdr, SSM_ERR_DEVICE, (int)L.w);
    bool live = active && !capped;
    const float drift = DrawnDrift<MODEL>::value ? L.dinc : r.drift;
    float g[18];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const uint4 b = philox10(
            make_uint4((uint32_t)(3 * W) * L.blk + (uint32_t)(3 * sub + m), L.n, L.k + p.k_base, 0u), p.key);
        bm6_increment(b, r.c2, drift, g + 6 * m);
    }
    const float ixf0 = L.ixf;
    float b36[W / 2];  // linear boundary at the block's 36-step bases
#pragma unroll
    for (int u = 0; u < W / 2; ++u)
        b36[u] = (BOUND == SSM_BOUND_LINEAR) ? fmaf(ixf0 + (float)(36 * u), r.dtp1, r.a) : 0.f;
    if (live) L.tpb = L.tp;
#pragma unroll
    for (int s = 0; s < W; ++s) {
#pragma unroll
        for (int j = 0; j < 18; ++j) {
            const float gq = __shfl_sync(FULL, g[j], src0 + s);
            const int q = 18 * s + j;
            const bool in_time = !TCHK || (L.tp <= r.dl_tmp);
            bool inside;
            if (MODEL == M_LEGACY) {
                inside = live && (L.y <= r.a) && (L.y >= 0.f) && in_time;
            } else {
                float bq;
                if (BOUND == SSM_BOUND_LINEAR)
                    bq = (q % 36 == 0) ? b36[q / 36] : fmaf((float)(q % 36), r.dtp1, b36[q / 36]);
                else
                    bq = bound_at<BOUND, false>(r, ixf0 + (float)q, 0, p, L.k);
                inside = live && (fabsf(L.y) <= bq) && in_time;
            }
            if (inside) {
                if (MODEL == M_OU) L.y = fmaf(L.y, r.expo, gq);
                else L.y += gq;
                L.tp += p.dt;
            }
            live = inside;
        }
    }
    if (active && !capped) L.ixf = ixf0 + (float)BLK;
    return live;
}

// ------------------------------------------------------------------ main kernel
// W lanes per walk (1 = one lane per trajectory; 2, 4, 8 = wide_block).  The
// queue logic counts walks: a group's lanes share `active`, so a ballot of
// free lanes holds W bits per free walk.
template <int MODEL, int BOUND, bool NOISE, int W>
__global__ void __launch_bounds__(256, (MinCtas<MODEL, W>::value))
    k_single(const __grid_constant__ SingleParams p) {
    static_assert(W == 1 || WideOk<MODEL, NOISE, BOUND>::value, "lanes per walk > 1: device RNG, in-register bound");
    constexpr int BLK = BlkW<MODEL, W, BOUND>::value;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int sub = lane & (W - 1);              // place in the group
    const int src0 = lane - sub;                 // the group's first lane
    const unsigned lt_mask = (1u << src0) - 1u;  // lanes of the groups before this one
    const int64_t total = (p.total >= 0) ? p.total : __ldg(p.offsets + p.n_trials) - __ldg(p.offsets);
    const int64_t chunk = warp_chunk(p.chunk, total, 32 / W);

    Lane L;
    TrialRow r = {};
    L.w = 0; L.k = L.n = L.blk = 0; L.ix = 0; L.y = L.tp = L.ixf = L.dinc = L.tpb = 0.f;
    bool active = false;
    bool pending = false;  // walk ended, result not yet written
    bool exhausted = false;
    int64_t q_next = 0, q_end = 0, hint = 0;

    for (;;) {
        // Lanes whose walk ended wait (predicated off) until refill_min of
        // them have: finishing and restarting lanes runs divergently, with the
        // rest of the warp idle, so it is done for several lanes in one pass.
        // Once the queue is empty, pending results are written at once.
        const unsigned need = __ballot_sync(FULL, !active);
        const int free_walks = __popc(need) / W;
        const bool pass = exhausted ? (__ballot_sync(FULL, pending) != 0u) : (free_walks >= p.refill_min);
        if (pass && pending) {
            finalize<MODEL, BOUND, NOISE, BLK>(p, L, sub == 0);
            pending = false;
        }
        if (pass && !exhausted) {
            const int cnt = free_walks;
            const int64_t avail = q_end - q_next;
            int64_t base = 0;
            if (avail < cnt) {
                unsigned long long b = 0ull;
                if (lane == 0) b = atomicAdd(&p.hdr->counter, (unsigned long long)chunk);
                base = (int64_t)__shfl_sync(FULL, b, 0);
                if (base >= total) exhausted = true;
            }
            if (!active) {
                const int rank = __popc(need & lt_mask) / W;
                const int64_t w = (rank < avail) ? q_next + rank : base + (rank - avail);
                if (w < total) active = lane_init<MODEL, NOISE>(p, L, r, w, hint);
            }
            if (avail >= cnt) {
                q_next += cnt;
            } else {
                q_next = base + (cnt - avail);
                q_end = base + chunk;
            }
        }
        if (__ballot_sync(FULL, active) == 0u) break;
        // warp-uniform: skip the per-step time test when no active lane can reach its limit in this block
        const bool skip_time = __all_sync(FULL, !active || block_in_time<MODEL, BOUND, NOISE, BLK>(p, L, r));
        bool live = false;
        if constexpr (W == 1) {
            if (active) {
                if constexpr (FuseOk<MODEL, NOISE>::value) {
                    live = skip_time ? step_block<MODEL, BOUND, NOISE, false, false, true>(p, L, r, nullptr)
                                     : step_block<MODEL, BOUND, NOISE, false, true, true>(p, L, r, nullptr);
                } else {
                    float g[Blk<MODEL, BOUND>::value];
                    draw_block<MODEL, BOUND, NOISE>(p, L, r, g);
                    live = skip_time ? step_block<MODEL, BOUND, NOISE, false, false>(p, L, r, g)
                                     : step_block<MODEL, BOUND, NOISE, false, true>(p, L, r, g);
                }
            }
        } else {
            live = skip_time ? wide_block<MODEL, BOUND, false, W>(p, L, r, active, src0, sub)
                             : wide_block<MODEL, BOUND, true, W>(p, L, r, active, src0, sub);
        }
        if (active) {
            L.blk += 1;
            if (!live) {
                active = false;
                pending = true;
            }
        }
    }
}

// Re-simulates trial 0 / sample 0 with the same stream and writes its path
// (metadata['trajectory'], -999 padded: ddm_models.pyx:714-728).
template <int MODEL, int BOUND, bool NOISE>
__global__ void k_record(const __grid_constant__ SingleParams p) {
    for (int64_t i = threadIdx.x; i < p.traj_len; i += blockDim.x) p.traj[i] = -999.f;
    __syncthreads();
    if (threadIdx.x != 0) return;
    Lane L;
    TrialRow r;
    int64_t hint = 0;
    lane_init<MODEL, NOISE>(p, L, r, 0, hint);
    if (p.traj_len > 0) p.traj[0] = L.y;
    for (;;) {
        float g[Blk<MODEL, BOUND>::value];
        draw_block<MODEL, BOUND, NOISE>(p, L, r, g);
        const bool live = step_block<MODEL, BOUND, NOISE, true>(p, L, r, g);
        L.blk += 1;
        if (!live) break;
    }
}

// ------------------------------------------------------------------ host side
// Lanes per walk chosen when the caller leaves it at 0: the wide modes pay
// where a launch holds about as many trajectories as the grid has lanes
// (the walks' latency sets the time) and cost throughput beyond.
int auto_lanes_per_walk(int64_t n_walks) {
    if (n_walks <= 0) return 1;
    const double per_lane = (double)n_walks / ((double)sm_count() * 768.0);  // 24 resident warps per SM
    if (per_lane <= 0.25) return 8;
    if (per_lane <= 1.5) return 4;
    if (per_lane <= 4.0) return 2;
    return 1;
}

struct Launcher {
    template <int MODEL, int BOUND, bool NOISE, int W>
    static int launch(const SingleParams &p, int threads, const ssm_launch *opt, cudaStream_t st) {
        auto kern = k_single<MODEL, BOUND, NOISE, W>;
        int per_sm = 0;
        SSM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
        if (opt && opt->blocks_per_sm > 0 && opt->blocks_per_sm < per_sm) per_sm = opt->blocks_per_sm;
        if (per_sm < 1) per_sm = 1;
        kern<<<sm_count() * per_sm, threads, 0, st>>>(p);
        SSM_CUDA(cudaGetLastError());
        return SSM_OK;
    }

    template <int MODEL, int BOUND, bool NOISE>
    static int run(const SingleParams &p, const ssm_launch *opt, cudaStream_t st) {
        int threads = (opt && opt->block_threads > 0) ? opt->block_threads : 256;
        if (threads > 256 || threads % 32) {
            set_error("block_threads must be a multiple of 32 and at most 256");
            return SSM_ERR_ARG;
        }
        constexpr bool WIDE = WideOk<MODEL, NOISE, BOUND>::value;
        const int W = (opt && opt->lanes_per_walk > 0) ? opt->lanes_per_walk
                                                        : (WIDE && p.total >= 0 ? auto_lanes_per_walk(p.total) : 1);
        if (W != 1 && W != 2 && W != 4 && W != 8) {
            set_error("lanes_per_walk must be 0 (automatic), 1, 2, 4 or 8");
            return SSM_ERR_ARG;
        }
        if (W > 1 && !WIDE) {
            set_error("lanes_per_walk > 1 needs the device RNG and a constant, linear or Weibull boundary");
            return SSM_ERR_ARG;
        }
        int rc = SSM_OK;
        if (W == 1) {
            rc = launch<MODEL, BOUND, NOISE, 1>(p, threads, opt, st);
        } else if constexpr (WIDE) {
            // a warp holds 32 / W walks: it claims that many at a time and
            // restarts a group as soon as its walk ends (unless told otherwise)
            SingleParams q = p;
            const int slots = 32 / W;
            q.chunk = slots;
            q.refill_min = (opt && opt->refill_min > 0) ? min(opt->refill_min, slots) : 1;
            rc = (W == 2)   ? launch<MODEL, BOUND, NOISE, 2>(q, threads, opt, st)
                 : (W == 4) ? launch<MODEL, BOUND, NOISE, 4>(q, threads, opt, st)
                            : launch<MODEL, BOUND, NOISE, 8>(q, threads, opt, st);
        }
        if (rc != SSM_OK) return rc;
        if (p.traj && p.traj_len > 0) {
            SingleParams pr = p;  // trial 0 / sample 0, whatever the processing order
            pr.order = nullptr;
            pr.qoff = nullptr;
            k_record<MODEL, BOUND, NOISE><<<1, 128, 0, st>>>(pr);
            SSM_CUDA(cudaGetLastError());
        }
        return SSM_OK;
    }

    template <int MODEL>
    static int dispatch(int bound, bool noise, const SingleParams &p, const ssm_launch *opt,
                        cudaStream_t st) {
        if (MODEL == M_LEGACY) {
            return noise ? run<MODEL, SSM_BOUND_CONSTANT, true>(p, opt, st)
                         : run<MODEL, SSM_BOUND_CONSTANT, false>(p, opt, st);
        }
        switch (bound) {
            case SSM_BOUND_TABLE:
                return noise ? run<MODEL, SSM_BOUND_TABLE, true>(p, opt, st)
                             : run<MODEL, SSM_BOUND_TABLE, false>(p, opt, st);
            case SSM_BOUND_CONSTANT:
                return noise ? run<MODEL, SSM_BOUND_CONSTANT, true>(p, opt, st)
                             : run<MODEL, SSM_BOUND_CONSTANT, false>(p, opt, st);
            case SSM_BOUND_LINEAR:
                return noise ? run<MODEL, SSM_BOUND_LINEAR, true>(p, opt, st)
                             : run<MODEL, SSM_BOUND_LINEAR, false>(p, opt, st);
            case SSM_BOUND_WEIBULL:
                return noise ? run<MODEL, SSM_BOUND_WEIBULL, true>(p, opt, st)
                             : run<MODEL, SSM_BOUND_WEIBULL, false>(p, opt, st);
            default:
                set_error("unknown boundary kind %d", bound);
                return SSM_ERR_ARG;
        }
    }
};

static size_t single_ws_bytes(int64_t n_trials) {
    size_t b = sizeof(WorkspaceHeader) + (size_t)(n_trials > 0 ? n_trials : 0) * sizeof(TrialRow);
    return (b + 255) & ~(size_t)255;
}

struct SingleCall {
    int model;
    const float *v, *a, *z, *alpha, *t, *deadline, *s;
    const float *sv, *sz, *st, *g;
    const float *dtable;
    int64_t dstride, dlen;
    int64_t n_trials, n_samples;
    const int64_t *offsets;
    float max_t;
    const float *maxt_k;
    float dt;
    int bound;
    const float *p1, *p2, *table;
    int64_t tstride, tlen;
    uint64_t seed;
    int smooth;
    const float *noise;
    int64_t nlen;
    const float *nunif;
    float *rts;
    int32_t *choices, *steps;
    float *traj;
    int64_t traj_len;
    const ssm_launch *launch;
    void *ws;
    size_t ws_bytes;
    void *stream;
};

static int run_single(const SingleCall &c) {
    SSM_REQUIRE(c.n_trials >= 0 && c.n_samples >= 0, "n_trials and n_samples must be >= 0");
    SSM_REQUIRE(c.dt > 0.f && isfinite(c.dt), "delta_t must be finite and > 0");
    SSM_REQUIRE(c.maxt_k || (isfinite(c.max_t) && (double)c.max_t / (double)c.dt <= 8388608.0),
                "max_t must be finite with max_t / delta_t <= 2^23");
    SSM_REQUIRE(c.v && c.z && c.t && c.deadline && c.s && c.a, "v, a, z, t, deadline, s are required");
    SSM_REQUIRE((c.rts && c.choices) || (!c.offsets && c.n_trials * c.n_samples == 0),
                "rts and choices outputs are required");
    SSM_REQUIRE(c.model != M_LEVY || c.alpha, "alpha is required for the Levy model");
    SSM_REQUIRE((c.model != M_SDV && c.model != M_FULL) || c.sv, "sv is required");
    SSM_REQUIRE(c.model != M_FULL || (c.sz && c.st), "sz and st are required");
    SSM_REQUIRE(c.model != M_OU || c.g, "g is required for the Ornstein-Uhlenbeck model");
    SSM_REQUIRE(c.model != M_DFLEX || (c.dtable && c.dlen >= 1 && c.dstride >= c.dlen),
                "ddm_flex needs drift_table with drift_stride >= drift_len >= 1");
    if (c.model != M_LEGACY) {
        SSM_REQUIRE(c.bound >= SSM_BOUND_TABLE && c.bound <= SSM_BOUND_WEIBULL, "unknown boundary kind %d", c.bound);
        SSM_REQUIRE(c.bound != SSM_BOUND_LINEAR || c.p1, "linear boundary needs bound_p1");
        SSM_REQUIRE(c.bound != SSM_BOUND_WEIBULL || (c.p1 && c.p2), "weibull boundary needs bound_p1 and bound_p2");
        SSM_REQUIRE(c.bound != SSM_BOUND_TABLE || (c.table && c.tlen >= 1 && c.tstride >= c.tlen),
                    "table boundary needs bound_table with table_stride >= table_len >= 1");
    }
    SSM_REQUIRE(!c.noise || (c.nlen > 0 && c.nunif), "noise_rows needs noise_row_len > 0 and noise_unif");
    SSM_REQUIRE(!c.traj || c.traj_len >= 1, "traj needs traj_len >= 1");
    SSM_REQUIRE(!c.launch || (!c.launch->trial_order == !c.launch->order_offsets),
                "trial_order and order_offsets go together");
    SSM_REQUIRE(!c.launch || !c.launch->trial_order || c.offsets,
                "a trial order needs the ragged layout (sample_offsets)");
    const size_t need = single_ws_bytes(c.n_trials);
    if (!c.ws || c.ws_bytes < need || ((uintptr_t)c.ws & 255u)) {
        set_error("workspace must be 256-byte aligned and hold %zu bytes", need);
        return SSM_ERR_WORKSPACE;
    }
    cudaStream_t st = (cudaStream_t)c.stream;
    WorkspaceHeader *hdr = (WorkspaceHeader *)c.ws;
    TrialRow *rows = (TrialRow *)((char *)c.ws + sizeof(WorkspaceHeader));
    SSM_CUDA(cudaMemsetAsync(hdr, 0, sizeof(WorkspaceHeader), st));
    if (c.n_trials == 0) return SSM_OK;

    PrepArgs A;
    A.v = c.v; A.a = c.a; A.z = c.z; A.t = c.t; A.deadline = c.deadline; A.s = c.s;
    A.alpha = c.alpha; A.p1 = c.p1; A.p2 = c.p2; A.maxt_k = c.maxt_k; A.table = c.table;
    A.sv = c.sv; A.sz = c.sz; A.st = c.st; A.g = c.g;
    A.n_trials = c.n_trials; A.tstride = c.tstride; A.dt = c.dt;
    A.sqrt_dt = (float)sqrt((double)c.dt);  // setup_simulation: sqrt(delta_t) -> float
    A.max_t = c.max_t; A.model = c.model; A.bound = c.bound; A.rows = rows;
    k_prep<<<(unsigned)((c.n_trials + 127) / 128), 128, 0, st>>>(A);
    SSM_CUDA(cudaGetLastError());

    SingleParams p;
    p.key = philox_keys(c.seed);
    p.rows = rows;
    p.offsets = c.offsets;
    p.order = c.offsets && c.launch ? c.launch->trial_order : nullptr;
    p.qoff = p.order ? c.launch->order_offsets : nullptr;
    p.n_trials = c.n_trials;
    p.total = c.offsets ? -1 : c.n_trials * c.n_samples;
    p.k_base = (uint32_t)((c.launch && c.launch->first_trial > 0) ? c.launch->first_trial : 0);
    p.ustride = (c.model == M_FULL) ? 3 : 1;
    p.dtable = c.dtable; p.dstride = c.dstride; p.dlen = c.dlen;
    p.dvec = (c.dtable && ((uintptr_t)c.dtable & 15u) == 0 && (c.dstride & 3) == 0) ? 1 : 0;
    p.dt = c.dt;
    p.smooth = c.smooth ? 1 : 0;
    p.chunk = (c.launch && c.launch->chunk >= 32) ? c.launch->chunk : 64;
    p.refill_min = (c.launch && c.launch->refill_min > 0) ? min(c.launch->refill_min, 32) : SSM_REFILL_MIN;
    p.table = c.table; p.tstride = c.tstride; p.tlen = c.tlen;
    p.noise = c.noise; p.nlen = c.nlen; p.nunif = c.nunif;
    p.rts = c.rts; p.choices = c.choices; p.steps = c.steps;
    p.hdr = hdr;
    p.traj = c.traj; p.traj_len = c.traj_len;
    if (p.total == 0) {
        if (c.traj) {  // nothing simulated: trajectory metadata is all padding
            p.traj_len = c.traj_len;
        }
        return SSM_OK;
    }
    const bool noise = c.noise != nullptr;
    switch (c.model) {
        case M_FLEX: return Launcher::dispatch<M_FLEX>(c.bound, noise, p, c.launch, st);
        case M_LEGACY: return Launcher::dispatch<M_LEGACY>(c.bound, noise, p, c.launch, st);
        case M_SDV: return Launcher::dispatch<M_SDV>(c.bound, noise, p, c.launch, st);
        case M_FULL: return Launcher::dispatch<M_FULL>(c.bound, noise, p, c.launch, st);
        case M_OU: return Launcher::dispatch<M_OU>(c.bound, noise, p, c.launch, st);
        case M_DFLEX: return Launcher::dispatch<M_DFLEX>(c.bound, noise, p, c.launch, st);
        default: return Launcher::dispatch<M_LEVY>(c.bound, noise, p, c.launch, st);
    }
}

}  // namespace ssm

extern "C" {

size_t ssm_ddm_workspace_bytes(int64_t n_trials) { return ssm::single_ws_bytes(n_trials); }
int ssm_auto_lanes_per_walk(int64_t n_walks) { return ssm::auto_lanes_per_walk(n_walks); }

int ssm_ddm_flexbound(const float *v, const float *a, const float *z, const float *t,
                      const float *deadline, const float *s, int64_t n_trials, int64_t n_samples,
                      const int64_t *sample_offsets, float max_t, const float *max_t_per_trial,
                      float delta_t, int bound_kind, const float *bound_p1, const float *bound_p2,
                      const float *bound_table, int64_t table_stride, int64_t table_len,
                      uint64_t seed, int smooth_unif, const float *noise_rows,
                      int64_t noise_row_len, const float *noise_unif, float *rts,
                      int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                      const ssm_launch *launch, void *workspace, size_t workspace_bytes,
                      void *stream) {
    ssm::SingleCall c{ssm::M_FLEX, v, a, z, nullptr, t, deadline, s, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0,
                      n_trials, n_samples,
                      sample_offsets, max_t, max_t_per_trial, delta_t, bound_kind, bound_p1,
                      bound_p2, bound_table, table_stride, table_len, seed, smooth_unif,
                      noise_rows, noise_row_len, noise_unif, rts, choices, steps, traj,
                      traj_len, launch, workspace, workspace_bytes, stream};
    return ssm::run_single(c);
}

int ssm_ddm(const float *v, const float *a, const float *z, const float *t, const float *deadline,
            const float *s, int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets,
            float max_t, float delta_t,
            uint64_t seed, int smooth_unif, const float *noise_rows, int64_t noise_row_len,
            const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
            int64_t traj_len, const ssm_launch *launch, void *workspace, size_t workspace_bytes,
            void *stream) {
    ssm::SingleCall c{ssm::M_LEGACY, v, a, z, nullptr, t, deadline, s, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0,
                      n_trials, n_samples,
                      sample_offsets, max_t, nullptr, delta_t, SSM_BOUND_CONSTANT, nullptr, nullptr,
                      nullptr, 0, 0, seed, smooth_unif, noise_rows, noise_row_len, noise_unif,
                      rts, choices, steps, traj, traj_len, launch, workspace, workspace_bytes,
                      stream};
    return ssm::run_single(c);
}

int ssm_levy_flexbound(const float *v, const float *a, const float *z, const float *alpha,
                       const float *t, const float *deadline, const float *s, int64_t n_trials,
                       int64_t n_samples, const int64_t *sample_offsets, float max_t,
                       float delta_t, int bound_kind, const float *bound_p1, const float *bound_p2,
                       const float *bound_table, int64_t table_stride, int64_t table_len,
                       uint64_t seed, int smooth_unif, const float *noise_rows,
                       int64_t noise_row_len, const float *noise_unif, float *rts,
                       int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                       const ssm_launch *launch, void *workspace, size_t workspace_bytes,
                       void *stream) {
    ssm::SingleCall c{ssm::M_LEVY, v, a, z, alpha, t, deadline, s, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0,
                      n_trials, n_samples,
                      sample_offsets, max_t, nullptr, delta_t, bound_kind, bound_p1, bound_p2,
                      bound_table, table_stride, table_len, seed, smooth_unif, noise_rows,
                      noise_row_len, noise_unif, rts, choices, steps, traj, traj_len, launch,
                      workspace, workspace_bytes, stream};
    return ssm::run_single(c);
}

int ssm_ddm_sdv(const float *v, const float *a, const float *z, const float *t, const float *sv,
                const float *deadline, const float *s, int64_t n_trials, int64_t n_samples,
                const int64_t *sample_offsets, float max_t, float delta_t, int bound_kind,
                const float *bound_p1, const float *bound_p2, const float *bound_table,
                int64_t table_stride, int64_t table_len, uint64_t seed, int smooth_unif,
                const float *noise_rows, int64_t noise_row_len, const float *noise_unif, float *rts,
                int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                const ssm_launch *launch, void *workspace, size_t workspace_bytes, void *stream) {
    ssm::SingleCall c{ssm::M_SDV, v, a, z, nullptr, t, deadline, s, sv, nullptr, nullptr, nullptr, nullptr, 0, 0,
                      n_trials, n_samples, sample_offsets, max_t, nullptr, delta_t, bound_kind,
                      bound_p1, bound_p2, bound_table, table_stride, table_len, seed, smooth_unif,
                      noise_rows, noise_row_len, noise_unif, rts, choices, steps, traj, traj_len,
                      launch, workspace, workspace_bytes, stream};
    return ssm::run_single(c);
}

int ssm_full_ddm(const float *v, const float *a, const float *z, const float *t, const float *sz,
                 const float *sv, const float *st, const float *deadline, const float *s,
                 int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets, float max_t,
                 float delta_t, int bound_kind, const float *bound_p1, const float *bound_p2,
                 const float *bound_table, int64_t table_stride, int64_t table_len, uint64_t seed,
                 int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                 const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
                 int64_t traj_len, const ssm_launch *launch, void *workspace,
                 size_t workspace_bytes, void *stream) {
    ssm::SingleCall c{ssm::M_FULL, v, a, z, nullptr, t, deadline, s, sv, sz, st, nullptr, nullptr, 0, 0,
                      n_trials, n_samples, sample_offsets, max_t, nullptr, delta_t, bound_kind,
                      bound_p1, bound_p2, bound_table, table_stride, table_len, seed, smooth_unif,
                      noise_rows, noise_row_len, noise_unif, rts, choices, steps, traj, traj_len,
                      launch, workspace, workspace_bytes, stream};
    return ssm::run_single(c);
}

int ssm_ornstein_uhlenbeck(const float *v, const float *a, const float *z, const float *g,
                           const float *t, const float *deadline, const float *s, int64_t n_trials,
                           int64_t n_samples, const int64_t *sample_offsets, float max_t,
                           float delta_t, int bound_kind, const float *bound_p1,
                           const float *bound_p2, const float *bound_table, int64_t table_stride,
                           int64_t table_len, uint64_t seed, int smooth_unif,
                           const float *noise_rows, int64_t noise_row_len, const float *noise_unif,
                           float *rts, int32_t *choices, int32_t *steps, float *traj,
                           int64_t traj_len, const ssm_launch *launch, void *workspace,
                           size_t workspace_bytes, void *stream) {
    ssm::SingleCall c{ssm::M_OU, v, a, z, nullptr, t, deadline, s, nullptr, nullptr, nullptr, g, nullptr, 0, 0,
                      n_trials, n_samples, sample_offsets, max_t, nullptr, delta_t, bound_kind,
                      bound_p1, bound_p2, bound_table, table_stride, table_len, seed, smooth_unif,
                      noise_rows, noise_row_len, noise_unif, rts, choices, steps, traj, traj_len,
                      launch, workspace, workspace_bytes, stream};
    return ssm::run_single(c);
}

int ssm_ddm_flex(const float *v, const float *a, const float *z, const float *t, const float *deadline,
                 const float *s, int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets,
                 float max_t, float delta_t, int bound_kind, const float *bound_p1,
                 const float *bound_p2, const float *bound_table, int64_t table_stride,
                 int64_t table_len, const float *drift_table, int64_t drift_stride, int64_t drift_len,
                 uint64_t seed, int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                 const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
                 int64_t traj_len, const ssm_launch *launch, void *workspace,
                 size_t workspace_bytes, void *stream) {
    ssm::SingleCall c{ssm::M_DFLEX, v, a, z, nullptr, t, deadline, s, nullptr, nullptr, nullptr, nullptr,
                      drift_table, drift_stride, drift_len, n_trials, n_samples, sample_offsets, max_t,
                      nullptr, delta_t, bound_kind, bound_p1, bound_p2, bound_table, table_stride,
                      table_len, seed, smooth_unif, noise_rows, noise_row_len, noise_unif, rts, choices,
                      steps, traj, traj_len, launch, workspace, workspace_bytes, stream};
    return ssm::run_single(c);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant.  Its scratch is this file-scope device array; host
// code must not hand the symbol itself to a kernel (in host code it names a
// host-side stand-in), so the device address is looked up with the device
// current and cached per device together with the unique id of the CUDA
// context it was looked up in.  A call under another context of that device
// (after cudaDeviceReset, or a primary-context reset) looks the address up
// again instead of reusing one from a context that no longer exists.
namespace ssm {
static __device__ __align__(256) unsigned char g_static_ws[SSM_STATIC_WS_BYTES];
static std::mutex g_static_mu;
struct StaticSlot {
    unsigned long long ctx_id;  // 0: not looked up yet
    void *ptr;
};
static StaticSlot g_static_slot[64] = {};

using PfnCtxGetCurrent = CUresult (*)(CUcontext *);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current CUDA context (cuCtxGetId, CUDA
// 12.0+, reached through the runtime's driver entry points); 0 when no context
// is current or the driver does not offer the query.  Called under g_static_mu.
static unsigned long long current_context_id() {
    static bool resolved = false;
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    if (!resolved) {
        resolved = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
        f = nullptr;
        q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PfnCtxGetId>(f);
    }
    if (get_current == nullptr || get_id == nullptr) return 0;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    unsigned long long id = 0;
    return get_id(ctx, &id) == CUDA_SUCCESS ? id : 0;
}

static int static_workspace(void **out) {
    int dev = 0;
    SSM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("device ordinal %d out of range for the static workspace", dev);
        return SSM_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    StaticSlot &slot = g_static_slot[dev];
    const unsigned long long id = current_context_id();
    if (slot.ctx_id == 0 || id != slot.ctx_id) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_ws);  // makes the device's context current
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_ws)");
        slot.ptr = p;
        slot.ctx_id = current_context_id();
    }
    *out = slot.ptr;
    return SSM_OK;
}
}  // namespace ssm

extern "C" int ssm_ddm_flexbound_static(
    const float *v, const float *a, const float *z, const float *t, const float *deadline,
    const float *s, int64_t n_trials, int64_t n_samples, const int64_t *sample_offsets,
    float max_t, const float *max_t_per_trial, float delta_t, int bound_kind,
    const float *bound_p1, const float *bound_p2, const float *bound_table, int64_t table_stride,
    int64_t table_len, uint64_t seed, int smooth_unif, const float *noise_rows,
    int64_t noise_row_len, const float *noise_unif, float *rts, int32_t *choices, int32_t *steps,
    float *traj, int64_t traj_len, const ssm_launch *launch, void *stream) {
    if (n_trials > SSM_STATIC_MAX_TRIALS) {
        ssm::set_error("ssm_ddm_flexbound_static supports at most %d trials (got %lld); "
                       "use ssm_ddm_flexbound with a caller workspace",
                       SSM_STATIC_MAX_TRIALS, (long long)n_trials);
        return SSM_ERR_ARG;
    }
    void *ws = nullptr;
    const int st = ssm::static_workspace(&ws);
    if (st != SSM_OK) return st;
    return ssm_ddm_flexbound(v, a, z, t, deadline, s, n_trials, n_samples, sample_offsets, max_t,
                             max_t_per_trial, delta_t, bound_kind, bound_p1, bound_p2,
                             bound_table, table_stride, table_len, seed, smooth_unif, noise_rows,
                             noise_row_len, noise_unif, rts, choices, steps, traj, traj_len,
                             launch, ws, SSM_STATIC_WS_BYTES, stream);
}
