// Multi-accumulator Euler-Maruyama simulators for sm_100a: the race model
// (cssm.race_model, src/cssm/race_models.pyx:356-506) and the leaky competing
// accumulator (cssm.lca, race_models.pyx:757-920).
//
// Same execution model as the single-accumulator kernel: one thread per
// trajectory, persistent grid, warps refill finished lanes from a global work
// counter.  The NP accumulators of a trajectory live in registers.  Each step
// tests the reference's loop condition (no accumulator above b(t) and
// t <= min(max_t, deadline - t_nd)), then updates every accumulator with its
// own N(0,1) increment and clips it at 0.  Choices are argmax (first maximum).
// Philox4x32-10 supplies four increments per call; noise injection reads
// caller rows (draw index step * NP + j) and evaluates every float operation
// with explicit rounding in the reference's order.
#include "common.cuh"

namespace ssm {

constexpr int RACE_MAX_NP = 16;

// Simulator families sharing this kernel: the race model, the LCA and the
// racing diffusion model (racing_diffusion_model, race_models.pyx:1150-1266:
// starts U(0, A), no lower barrier, the first accumulator at or above b wins
// and the step that reaches it does not advance the time).
enum RaceFamily { FAM_RACE = 0, FAM_LCA = 1, FAM_RDM = 2 };

// Per-trial header (64 B) followed by v[np], sq[np] (= sqrt(dt)*s), z[np]
// padded to a multiple of 4 floats.
struct alignas(16) RaceHead {
    float t, deadline, dl_tmp, a;
    float p1, dtp1, inv_beta, capf;
    float g, b, y0scale, pad0;   // y0scale = b(0): start p_j = z_j * b(0)
    float pad[4];
};
static_assert(sizeof(RaceHead) == 64, "RaceHead is one 64-byte line");

__host__ __device__ inline int64_t race_row_floats(int np) {
    return 16 + ((3 * (int64_t)np + 3) / 4) * 4;
}

struct RaceParams {
    PhiloxKeys key;
    const float *rows;
    int64_t row_floats;
    const int64_t *offsets;
    const int32_t *order;     // ragged only: trial simulated j-th (nullptr = index order)
    const int64_t *qoff;      // prefix sums of the sample counts in that order
    int64_t n_trials, total;  // total -1: offsets[n_trials] - offsets[0]
    uint32_t k_base;          // random-stream index of trial 0 (trial windows of a larger batch)
    int np;
    float dt;
    int smooth, chunk;
    int refill_min;           // ended walks a warp collects before it restarts lanes
    const float *table;
    int64_t tstride, tlen;
    const float *noise;
    int64_t nlen;
    const float *nunif;
    float *rts;
    int32_t *choices, *steps;
    WorkspaceHeader *hdr;
    float *traj;
    int64_t traj_len;
};

struct RacePrep {
    const float *v, *z, *t, *s, *deadline, *a, *p1, *p2, *g, *b, *table;
    int per_trial_zs;  // rdm: z (the start range A) and s hold one value per trial
    int64_t n_trials, tstride, row_floats;
    int np, bound;
    float dt, sqrt_dt, max_t;
    float *rows;
};

__global__ void k_race_prep(const RacePrep A) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.n_trials) return;
    float *row = A.rows + k * A.row_floats;
    RaceHead h;
    const float dt = A.dt;
    h.t = A.t[k];
    h.deadline = A.deadline[k];
    const float dl = __fsub_rn(h.deadline, h.t);
    h.dl_tmp = (dl < A.max_t) ? dl : A.max_t;  // compute_deadline_tmp (_utils.pyx:712-718)
    h.a = A.a ? A.a[k] : 0.f;
    h.p1 = A.p1 ? A.p1[k] : 0.f;
    h.dtp1 = dt * h.p1;
    h.inv_beta = 1.0f / (A.p2 ? A.p2[k] : 1.f);
    const double nsteps = (double)h.dl_tmp / (double)dt;
    if (!(nsteps > 0.0)) h.capf = 64.f;
    else if (nsteps <= 8388608.0) h.capf = (float)(int)(2.0 * nsteps + 64.0);
    else h.capf = 0.f;
    h.g = A.g ? A.g[k] : 0.f;
    h.b = A.b ? A.b[k] : 0.f;
    h.y0scale = (A.bound == SSM_BOUND_TABLE) ? A.table[k * A.tstride] : h.a;
    h.pad0 = 0.f;
    for (int i = 0; i < 4; ++i) h.pad[i] = 0.f;
    *reinterpret_cast<RaceHead *>(row) = h;
    float *v = row + 16, *sq = v + A.np, *z = sq + A.np;
    for (int j = 0; j < A.np; ++j) {
        v[j] = A.v[k * A.np + j];
        const int64_t i = A.per_trial_zs ? k : k * A.np + j;
        sq[j] = __fmul_rn(A.sqrt_dt, A.s[i]);  // delta_t_sqrt * s (race_models.pyx:385)
        z[j] = A.z[i];
    }
}

template <int BOUND, bool EXACT>
__device__ __forceinline__ float race_bound(const RaceHead &h, float ixf, int ix,
                                            const RaceParams &p, int64_t k) {
    if (BOUND == SSM_BOUND_CONSTANT) {
        return h.a;
    } else if (BOUND == SSM_BOUND_LINEAR) {
        if (EXACT) return __fadd_rn(h.a, __fmul_rn(__fmul_rn(ixf, p.dt), h.p1));
        return fmaf(ixf, h.dtp1, h.a);
    } else if (BOUND == SSM_BOUND_WEIBULL) {
        const float x = ixf * p.dt * h.inv_beta;
        const float pw = (x > 0.f) ? exp2f(h.p1 * __log2f(x)) : 0.f;
        return h.a * __expf(-pw);
    } else {
        const int64_t i = (ix < p.tlen) ? ix : p.tlen - 1;
        return __ldg(p.table + k * p.tstride + i);
    }
}

__device__ __forceinline__ float2 std_normal_pair(uint32_t a, uint32_t b) {
    return box_muller(a, b);
}

// Models with at most 4 accumulators draw a window of WIN steps' normals at
// once, six per Philox4x32-10 call (bm6_increment), WIN * NP a multiple of six:
// 2 accumulators 12 steps, 3 accumulators 8, 4 accumulators 6 -- four
// independent calls per window, whose latencies overlap.  Measured on the
// 1024-set workloads (ms per launch): LCA 50.3 -> 44.8 and race 19.2 -> 17.0
// against one call (four normals) per step drawn eight steps ahead, which
// itself had taken LCA from 66.0 (2 ahead 65.5, 4 ahead 56.3, 8 ahead 52.1).
template <int NP> struct RaceWin { static constexpr int value = NP == 2 ? 12 : (NP == 3 ? 8 : 6); };

template <int NP>
struct RaceLane {
    int64_t w;
    uint32_t k, n;
    float ixf, tp;  // steps taken (as float); race: float32 time accumulator
    double tpd;     // lca: double time accumulator (Cython infers double, race_models.pyx:838)
    int win;        // rdm: index of the winning accumulator (-1 while racing)
    float x[NP];
};

// The next window's increments, drawn ahead six per Philox call (calls ctr ..
// ctr + CALLS - 1) and stored accumulator-major: pre[j * WIN + s] is
// accumulator j's increment v_j dt + sq_j N(0,1) at step s of the window.
// WIN is even, so every Box-Muller pair belongs to one accumulator and that
// accumulator's scale and drift fold into the pair (radius constant
// c2 = -2 ln(2) sq_j^2, drift v_j dt): a step adds one increment instead of
// scaling a standard normal and adding the drift.
template <int NP>
__device__ __forceinline__ void draw_window(const RaceParams &p, const RaceLane<NP> &L, const float *vr,
                                            const float *sr, uint32_t ctr, float *pre) {
    constexpr int WIN = RaceWin<NP>::value;
    constexpr int CALLS = WIN * NP / 6;
    static_assert(WIN % 2 == 0 && (WIN * NP) % 6 == 0, "pairs within one accumulator, whole calls");
    float c2a[NP], dta[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        c2a[j] = -1.3862944f * sr[j] * sr[j];
        dta[j] = vr[j] * p.dt;
    }
#pragma unroll
    for (int c = 0; c < CALLS; ++c) {
        const uint4 r = philox10(make_uint4(ctr + (uint32_t)c, L.n, L.k + p.k_base, 0u), p.key);
        const float c2[3] = {c2a[(6 * c) / WIN], c2a[(6 * c + 2) / WIN], c2a[(6 * c + 4) / WIN]};
        const float d[3] = {dta[(6 * c) / WIN], dta[(6 * c + 2) / WIN], dta[(6 * c + 4) / WIN]};
        bm6_increment_pairs(r, c2, d, pre + 6 * c);
    }
}

// True when none of the lane's next `win` steps can reach the step cap or the
// time limit: the float32 accumulator after (win - 1) more additions of dt is
// at most t + (win - 1) dt plus their roundings (under dt/4 below 65536 dt),
// so t + (win + 1) dt <= dl_tmp leaves margin; LCA's float64 accumulator
// rounds far less.
template <int NP, int FAM>
__device__ __forceinline__ bool window_clear(const RaceParams &p, const RaceLane<NP> &L, const RaceHead &h,
                                             int win) {
    if (L.ixf + (float)win > h.capf) return false;
    const float span = (float)(win + 1);
    if (FAM == FAM_LCA) return L.tpd + (double)span * (double)p.dt <= (double)h.dl_tmp;
    return (L.tp < p.dt * 65536.f) && (fmaf(span, p.dt, L.tp) <= h.dl_tmp);
}

// One Euler step of every accumulator.  Returns false when the loop condition
// failed before the step (the walk is over).  With PRE the step's increments
// v_j dt + sq_j N(0,1) come from pre[j * PSTRIDE] (draw_window); ctr still
// counts the steps.
// CHECKED false skips the step-cap check and the time test, for a window the
// caller has shown both to pass for (window_clear).
template <int NP, int FAM, int BOUND, bool NOISE, bool RECORD, bool PRE = false, bool CHECKED = true,
          int PSTRIDE = 1>
__device__ __forceinline__ bool race_step(const RaceParams &p, RaceLane<NP> &L, const RaceHead &h,
                                          const float *v, const float *sq, int np, uint32_t &ctr,
                                          const float *pre = nullptr) {
    if (CHECKED && L.ixf >= h.capf) {
        raise_error(p.hdr, SSM_ERR_DEVICE, (int)L.w);
        return false;
    }
    const float bnd = race_bound<BOUND, NOISE>(h, L.ixf, (int)L.ixf, p, L.k);
    bool finished = false;
    if (FAM != FAM_RDM) {  // race / LCA test the bound before the step; RDM after each update
#pragma unroll
        for (int j = 0; j < NP; ++j)
            if (j < np) finished |= (L.x[j] > bnd);
    }
    constexpr bool LCA = (FAM == FAM_LCA);
    const bool in_time = !CHECKED || (LCA ? (L.tpd <= (double)h.dl_tmp) : (L.tp <= h.dl_tmp));
    if (finished || !in_time) return false;
    float gsn[NP];
    if (NOISE) {
        const int64_t base = (int64_t)L.ixf * np;
        if (base + np > p.nlen) {
            raise_error(p.hdr, SSM_ERR_NOISE_RANGE, (int)L.w);
            return false;
        }
        const float *row = p.noise + L.w * p.nlen + base;
#pragma unroll
        for (int j = 0; j < NP; ++j) gsn[j] = (j < np) ? __ldg(row + j) : 0.f;
    } else if (PRE) {
#pragma unroll
        for (int j = 0; j < NP; ++j) gsn[j] = pre[j * PSTRIDE];
        ctr += 1;
    } else {
#pragma unroll
        for (int j0 = 0; j0 < NP; j0 += 4) {
            if (j0 < np) {
                const uint4 r = philox10(make_uint4(ctr, L.n, L.k + p.k_base, 0u), p.key);
                ctr += 1;
                const float2 a = std_normal_pair(r.x, r.y);
                const float2 b = std_normal_pair(r.z, r.w);
                if (j0 + 0 < NP) gsn[j0 + 0] = a.x;
                if (j0 + 1 < NP) gsn[j0 + 1] = a.y;
                if (j0 + 2 < NP) gsn[j0 + 2] = b.x;
                if (j0 + 3 < NP) gsn[j0 + 3] = b.y;
            }
        }
    }
    if (LCA) {
        float sum = 0.f;
#pragma unroll
        for (int j = 0; j < NP; ++j)
            if (j < np) sum = NOISE ? __fadd_rn(sum, L.x[j]) : sum + L.x[j];
        // with PRE the increments carry v dt + sq N: x (1 - g dt + b dt) - b dt sum + increment
        const float c1 = fmaf(h.b - h.g, p.dt, 1.f), c2 = -h.b * p.dt;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            if (j < np) {
                float xj = L.x[j];
                if (PRE && !NOISE) {
                    xj = fmaf(xj, c1, fmaf(sum, c2, gsn[j]));
                } else if (NOISE) {
                    // race_models.pyx:849-857 with the reference build's association
                    const float red = __double2float_rn(__dadd_rn(-(double)xj, (double)sum));
                    const float A = __fsub_rn(__fsub_rn(v[j], __fmul_rn(h.g, xj)), __fmul_rn(h.b, red));
                    xj = __fadd_rn(__fadd_rn(xj, __fmul_rn(A, p.dt)), __fmul_rn(sq[j], gsn[j]));
                } else {
                    const float red = sum - xj;
                    const float A = v[j] - h.g * xj - h.b * red;
                    xj = fmaf(sq[j], gsn[j], fmaf(A, p.dt, xj));
                }
                L.x[j] = fmaxf(0.f, xj);
            }
        }
        L.tpd = NOISE ? __dadd_rn(L.tpd, (double)p.dt) : L.tpd + (double)p.dt;
    } else if (FAM == FAM_RDM) {
        // no lower barrier; the first accumulator (in index order) at or above b
        // wins and its step does not advance the time (race_models.pyx:1227-1244)
        bool hit = false;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            if (j < np) {
                float xj;
                if (NOISE) xj = __fadd_rn(__fadd_rn(L.x[j], __fmul_rn(v[j], p.dt)), __fmul_rn(sq[j], gsn[j]));
                else if (PRE) xj = L.x[j] + gsn[j];
                else xj = fmaf(sq[j], gsn[j], L.x[j] + v[j] * p.dt);
                L.x[j] = xj;
                hit |= (xj >= bnd);
            }
        }
        if (hit) {  // once per walk: the winner is the first accumulator at or above b
            int win = 0;
#pragma unroll
            for (int j = NP - 1; j >= 0; --j)
                if (j < np && L.x[j] >= bnd) win = j;
            L.win = win;
            return false;
        }
        L.tp = NOISE ? __fadd_rn(L.tp, p.dt) : L.tp + p.dt;
    } else {
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            if (j < np) {
                float xj;
                if (NOISE) xj = __fadd_rn(__fadd_rn(L.x[j], __fmul_rn(v[j], p.dt)), __fmul_rn(sq[j], gsn[j]));
                else if (PRE) xj = L.x[j] + gsn[j];
                else xj = fmaf(sq[j], gsn[j], L.x[j] + v[j] * p.dt);
                L.x[j] = fmaxf(0.f, xj);
            }
        }
        L.tp = NOISE ? __fadd_rn(L.tp, p.dt) : L.tp + p.dt;
    }
    L.ixf += 1.0f;  // steps taken, exact in float32 below 2^24
    if (RECORD) {
        const int64_t ix = (int64_t)L.ixf;
        if ((ix + 1) * np <= p.traj_len)
            for (int j = 0; j < np && j < NP; ++j) p.traj[ix * np + j] = L.x[j];
    }
    return true;
}

template <int NP, int FAM, bool NOISE>
__device__ __forceinline__ void race_finalize(const RaceParams &p, const RaceLane<NP> &L,
                                              const RaceHead &h, int np) {
    float u;
    if (NOISE) u = __ldg(p.nunif + ((FAM == FAM_RDM) ? L.w * (np + 1) + np : L.w));
    else u = uniform_co(philox10(make_uint4(0xFFFFFFFFu, L.n, L.k + p.k_base, 1u), p.key).x);
    // compute_smooth_unif receives the time as a C float (_utils.pyx:668-695)
    constexpr bool LCA = (FAM == FAM_LCA);
    const float tpf = LCA ? __double2float_rn(L.tpd) : L.tp;
    float sm = 0.f;
    if (p.smooth) {
        if (tpf == 0.f) sm = __double2float_rn(((double)u * 0.5) * (double)p.dt);
        else if (tpf < h.dl_tmp) sm = __double2float_rn((0.5 - (double)u) * (double)p.dt);
    }
    float rt;
    if (LCA) rt = __double2float_rn(__dadd_rn(__dadd_rn(L.tpd, (double)h.t), (double)sm));
    else rt = __fadd_rn(__fadd_rn(L.tp, h.t), sm);
    if (rt >= h.deadline || h.deadline <= 0.f) rt = -999.f;  // enforce_deadline
    if (FAM == FAM_RDM) {  // no decision or an omission: rt -999, choice -1
        const bool omit = (rt == -999.f) || (L.win < 0);
        p.rts[L.w] = omit ? -999.f : rt;
        p.choices[L.w] = omit ? -1 : L.win;
        if (p.steps) p.steps[L.w] = (int)L.ixf;
        return;
    }
    int best = 0;
    float bv = L.x[0];
#pragma unroll
    for (int j = 1; j < NP; ++j)
        if (j < np && L.x[j] > bv) {
            bv = L.x[j];
            best = j;
        }
    p.rts[L.w] = rt;
    p.choices[L.w] = best;
    if (p.steps) p.steps[L.w] = (int)L.ixf;
}

__device__ __forceinline__ int64_t race_find(const int64_t *off, int64_t K, int64_t w, int64_t hint) {
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

template <int NP, int FAM, bool NOISE>
__device__ __forceinline__ bool race_init(const RaceParams &p, RaceLane<NP> &L, RaceHead &h,
                                          int64_t w, int64_t &hint, int np) {
    int64_t k, n;
    if (p.offsets == nullptr) {
        k = w % p.n_trials;
        n = w / p.n_trials;
    } else if (p.order != nullptr) {
        // queue index -> position j in the processing order -> trial k (outputs
        // stay at offsets[k] + n); an entry that does not fit is reported
        const int64_t j = race_find(p.qoff, p.n_trials, w, hint);
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
        k = race_find(p.offsets, p.n_trials, w, hint);
        n = w - __ldg(p.offsets + k);
        hint = k;
    }
    const float *row = p.rows + k * p.row_floats;
    const float4 *src = reinterpret_cast<const float4 *>(row);
    float4 *dst = reinterpret_cast<float4 *>(&h);
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[i] = __ldg(src + i);
    const float *z = row + 16 + 2 * np;
    L.w = w;
    L.k = (uint32_t)k;
    L.n = (uint32_t)n;
    L.win = -1;
    if (FAM == FAM_RDM) {
        // starts U(0, A): z holds A; injected uniforms, or the trajectory's own stream
#pragma unroll
        for (int j0 = 0; j0 < NP; j0 += 4) {
            uint4 r = make_uint4(0u, 0u, 0u, 0u);
            if (!NOISE && j0 < np) r = philox10(make_uint4(0xFFFFFFFEu, L.n, L.k + p.k_base, 2u + (uint32_t)j0), p.key);
            const uint32_t wd[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = j0 + q;
                if (j < NP) {
                    const float u = NOISE ? ((j < np) ? __ldg(p.nunif + L.w * (np + 1) + j) : 0.f) : uniform_co(wd[q]);
                    L.x[j] = (j < np) ? __fmul_rn(u, __ldg(z + j)) : 0.f;
                }
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < NP; ++j) L.x[j] = (j < np) ? __fmul_rn(__ldg(z + j), h.y0scale) : 0.f;
    }
    L.ixf = 0.f;
    L.tp = 0.f;
    L.tpd = 0.0;
    return true;
}

template <int NP, int FAM, int BOUND, bool NOISE>
__global__ void __launch_bounds__(256) k_race(const __grid_constant__ RaceParams p) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t total = (p.total >= 0) ? p.total : __ldg(p.offsets + p.n_trials) - __ldg(p.offsets);
    const int64_t chunk = warp_chunk(p.chunk, total);
    const int np = (NP == RACE_MAX_NP) ? p.np : NP;
    RaceLane<NP> L;
    RaceHead h;
    L.w = 0; L.k = L.n = 0; L.ixf = L.tp = 0.f; L.tpd = 0.0; L.win = -1;
#pragma unroll
    for (int j = 0; j < NP; ++j) L.x[j] = 0.f;
    uint32_t ctr = 0;
    bool active = false, pending = false, exhausted = false;
    int64_t q_next = 0, q_end = 0, hint = 0;
    for (;;) {
        // ended walks are written and their lanes restarted refill_min at a
        // time (one divergent pass for several lanes); all at once when the
        // queue is empty
        const unsigned need = __ballot_sync(FULL, !active);
        const bool pass = exhausted ? (__ballot_sync(FULL, pending) != 0u) : (__popc(need) >= p.refill_min);
        if (pass && pending) {
            race_finalize<NP, FAM, NOISE>(p, L, h, np);
            pending = false;
        }
        if (pass && !exhausted) {
            const int cnt = __popc(need);
            const int64_t avail = q_end - q_next;
            int64_t base = 0;
            if (avail < cnt) {
                unsigned long long bb = 0ull;
                if (lane == 0) bb = atomicAdd(&p.hdr->counter, (unsigned long long)chunk);
                base = (int64_t)__shfl_sync(FULL, bb, 0);
                if (base >= total) exhausted = true;
            }
            if (!active) {
                const int rank = __popc(need & lt_mask);
                const int64_t w = (rank < avail) ? q_next + rank : base + (rank - avail);
                if (w < total && race_init<NP, FAM, NOISE>(p, L, h, w, hint, np)) {
                    ctr = 0;
                    active = true;
                }
            }
            if (avail >= cnt) {
                q_next += cnt;
            } else {
                q_next = base + (cnt - avail);
                q_end = base + chunk;
            }
        }
        if (__ballot_sync(FULL, active) == 0u) break;
        // warp-uniform: skip the per-step cap and time tests when no active
        // lane can reach either within its next window
        const bool clear = (!NOISE && NP <= 4) &&
                           __all_sync(FULL, !active || window_clear<NP, FAM>(p, L, h, RaceWin<NP>::value));
        if (active) {
            const float *row = p.rows + (int64_t)L.k * p.row_floats;
            const float *v = row + 16;
            const float *sq = v + np;
            float vr[NP], sr[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                vr[j] = (j < np) ? __ldg(v + j) : 0.f;
                sr[j] = (j < np) ? __ldg(sq + j) : 0.f;
            }
            bool live = true;
            if (!NOISE && NP <= 4) {
                // the next WIN steps' increments first (draw_window), then the
                // steps; ctr advances per window
                constexpr int WIN = RaceWin<NP>::value;
                float nrm[WIN * NP];
                draw_window<NP>(p, L, vr, sr, ctr, nrm);
                ctr += WIN * NP / 6;
                uint32_t unused = 0;
                if (clear) {
#pragma unroll
                    for (int s = 0; s < WIN; ++s)
                        if (live)
                            live = race_step<NP, FAM, BOUND, NOISE, false, true, false, WIN>(p, L, h, vr, sr, np,
                                                                                             unused, nrm + s);
                } else {
#pragma unroll
                    for (int s = 0; s < WIN; ++s)
                        if (live)
                            live = race_step<NP, FAM, BOUND, NOISE, false, true, true, WIN>(p, L, h, vr, sr, np,
                                                                                            unused, nrm + s);
                }
            } else {
#pragma unroll 1
                for (int s = 0; s < 4 && live; ++s)
                    live = race_step<NP, FAM, BOUND, NOISE, false>(p, L, h, vr, sr, np, ctr);
            }
            if (!live) {
                active = false;
                pending = true;
            }
        }
    }
}

template <int NP, int FAM, int BOUND, bool NOISE>
__global__ void k_race_record(const __grid_constant__ RaceParams p) {
    const int np = (NP == RACE_MAX_NP) ? p.np : NP;
    for (int64_t i = threadIdx.x; i < p.traj_len; i += blockDim.x) p.traj[i] = -999.f;
    __syncthreads();
    if (threadIdx.x != 0) return;
    RaceLane<NP> L;
    RaceHead h;
    int64_t hint = 0;
    race_init<NP, FAM, NOISE>(p, L, h, 0, hint, np);
    for (int j = 0; j < np && j < NP && j < p.traj_len; ++j) p.traj[j] = L.x[j];
    const float *row = p.rows + (int64_t)L.k * p.row_floats;
    float vr[NP], sr[NP];
    for (int j = 0; j < NP; ++j) {
        vr[j] = (j < np) ? row[16 + j] : 0.f;
        sr[j] = (j < np) ? row[16 + np + j] : 0.f;
    }
    uint32_t ctr = 0;
    if (!NOISE && NP <= 4) {
        // the main kernel's windows: the same normals in the same order
        constexpr int WIN = RaceWin<NP>::value;
        bool live = true;
        while (live) {
            float nrm[WIN * NP];
            draw_window<NP>(p, L, vr, sr, ctr, nrm);
            ctr += WIN * NP / 6;
            uint32_t unused = 0;
            for (int s = 0; s < WIN && live; ++s)
                live = race_step<NP, FAM, BOUND, NOISE, true, true, true, WIN>(p, L, h, vr, sr, np, unused, nrm + s);
        }
    } else {
        while (race_step<NP, FAM, BOUND, NOISE, true>(p, L, h, vr, sr, np, ctr)) {
        }
    }
}

template <int NP, int FAM, int BOUND, bool NOISE>
static int race_launch(const RaceParams &p, const ssm_launch *opt, cudaStream_t st) {
    auto kern = k_race<NP, FAM, BOUND, NOISE>;
    int threads = (opt && opt->block_threads > 0) ? opt->block_threads : 256;
    if (threads > 256 || threads % 32) {
        set_error("block_threads must be a multiple of 32 and at most 256");
        return SSM_ERR_ARG;
    }
    int per_sm = 0;
    SSM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
    if (opt && opt->blocks_per_sm > 0 && opt->blocks_per_sm < per_sm) per_sm = opt->blocks_per_sm;
    if (per_sm < 1) per_sm = 1;
    kern<<<sm_count() * per_sm, threads, 0, st>>>(p);
    SSM_CUDA(cudaGetLastError());
    if (p.traj && p.traj_len > 0) {
        RaceParams pr = p;  // trial 0 / sample 0, whatever the processing order
        pr.order = nullptr;
        pr.qoff = nullptr;
        k_race_record<NP, FAM, BOUND, NOISE><<<1, 128, 0, st>>>(pr);
        SSM_CUDA(cudaGetLastError());
    }
    return SSM_OK;
}

template <int NP, int FAM>
static int race_dispatch_bound(int bound, bool noise, const RaceParams &p, const ssm_launch *opt,
                               cudaStream_t st) {
    if (noise) {  // exact mode: any boundary shape arrives as a host table or in closed form
        switch (bound) {
            case SSM_BOUND_TABLE: return race_launch<NP, FAM, SSM_BOUND_TABLE, true>(p, opt, st);
            case SSM_BOUND_CONSTANT: return race_launch<NP, FAM, SSM_BOUND_CONSTANT, true>(p, opt, st);
            case SSM_BOUND_LINEAR: return race_launch<NP, FAM, SSM_BOUND_LINEAR, true>(p, opt, st);
            default: break;
        }
        set_error("noise injection supports table, constant and linear boundaries");
        return SSM_ERR_ARG;
    }
    switch (bound) {
        case SSM_BOUND_TABLE: return race_launch<NP, FAM, SSM_BOUND_TABLE, false>(p, opt, st);
        case SSM_BOUND_CONSTANT: return race_launch<NP, FAM, SSM_BOUND_CONSTANT, false>(p, opt, st);
        case SSM_BOUND_LINEAR: return race_launch<NP, FAM, SSM_BOUND_LINEAR, false>(p, opt, st);
        case SSM_BOUND_WEIBULL: return race_launch<NP, FAM, SSM_BOUND_WEIBULL, false>(p, opt, st);
        default: break;
    }
    set_error("unknown boundary kind %d", bound);
    return SSM_ERR_ARG;
}

template <int FAM>
static int race_dispatch(int np, int bound, bool noise, const RaceParams &p, const ssm_launch *opt,
                         cudaStream_t st) {
    switch (np) {
        case 2: return race_dispatch_bound<2, FAM>(bound, noise, p, opt, st);
        case 3: return race_dispatch_bound<3, FAM>(bound, noise, p, opt, st);
        case 4: return race_dispatch_bound<4, FAM>(bound, noise, p, opt, st);
        default: return race_dispatch_bound<RACE_MAX_NP, FAM>(bound, noise, p, opt, st);
    }
}

static size_t race_ws_bytes(int64_t n_trials, int np) {
    if (n_trials < 0) n_trials = 0;
    size_t b = sizeof(WorkspaceHeader) + (size_t)n_trials * race_row_floats(np) * sizeof(float);
    return (b + 255) & ~(size_t)255;
}

static int run_race(int fam, const float *v, const float *z, const float *t, const float *s,
                    const float *deadline, const float *g, const float *b, int64_t n_trials,
                    int64_t n_samples, int np, const int64_t *offsets, float max_t, float dt,
                    int bound, const float *a, const float *p1, const float *p2,
                    const float *table, int64_t tstride, int64_t tlen, uint64_t seed, int smooth,
                    const float *noise, int64_t nlen, const float *nunif, float *rts,
                    int32_t *choices, int32_t *steps, float *traj, int64_t traj_len,
                    const ssm_launch *launch, void *ws, size_t ws_bytes, void *stream) {
    SSM_REQUIRE(n_trials >= 0 && n_samples >= 0, "n_trials and n_samples must be >= 0");
    SSM_REQUIRE(np >= 1 && np <= RACE_MAX_NP, "n_particles must be in [1, %d]", RACE_MAX_NP);
    SSM_REQUIRE(dt > 0.f && isfinite(dt), "delta_t must be finite and > 0");
    SSM_REQUIRE(isfinite(max_t) && (double)max_t / (double)dt <= 8388608.0,
                "max_t must be finite with max_t / delta_t <= 2^23");
    SSM_REQUIRE(n_trials == 0 || (v && z && t && s && deadline), "v, z, t, s, deadline are required");
    SSM_REQUIRE(fam != FAM_LCA || n_trials == 0 || (g && b), "lca needs g and b");
    SSM_REQUIRE(!launch || (!launch->trial_order == !launch->order_offsets),
                "trial_order and order_offsets go together");
    SSM_REQUIRE(!launch || !launch->trial_order || offsets, "a trial order needs the ragged layout (sample_offsets)");
    SSM_REQUIRE((rts && choices) || (!offsets && n_trials * n_samples == 0), "rts and choices outputs are required");
    SSM_REQUIRE(bound >= SSM_BOUND_TABLE && bound <= SSM_BOUND_WEIBULL, "unknown boundary kind %d", bound);
    SSM_REQUIRE(bound == SSM_BOUND_TABLE || n_trials == 0 || a, "boundary height a is required");
    SSM_REQUIRE(bound != SSM_BOUND_LINEAR || n_trials == 0 || p1, "linear boundary needs bound_p1");
    SSM_REQUIRE(bound != SSM_BOUND_WEIBULL || n_trials == 0 || (p1 && p2), "weibull boundary needs bound_p1 and bound_p2");
    SSM_REQUIRE(bound != SSM_BOUND_TABLE || (table && tlen >= 1 && tstride >= tlen),
                "table boundary needs bound_table with table_stride >= table_len >= 1");
    SSM_REQUIRE(!noise || (nlen > 0 && nunif), "noise_rows needs noise_row_len > 0 and noise_unif");
    const size_t need = race_ws_bytes(n_trials, np);
    if (!ws || ws_bytes < need || ((uintptr_t)ws & 255u)) {
        set_error("workspace must be 256-byte aligned and hold %zu bytes", need);
        return SSM_ERR_WORKSPACE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    WorkspaceHeader *hdr = (WorkspaceHeader *)ws;
    float *rows = (float *)((char *)ws + sizeof(WorkspaceHeader));
    SSM_CUDA(cudaMemsetAsync(hdr, 0, sizeof(WorkspaceHeader), st));
    const int64_t total = offsets ? -1 : n_trials * n_samples;
    if (n_trials == 0 || total == 0) return SSM_OK;
    RacePrep A;
    A.v = v; A.z = z; A.t = t; A.s = s; A.deadline = deadline; A.a = a; A.p1 = p1; A.p2 = p2;
    A.g = g; A.b = b; A.table = table; A.n_trials = n_trials; A.tstride = tstride;
    A.row_floats = race_row_floats(np); A.np = np; A.bound = bound; A.dt = dt;
    A.sqrt_dt = (float)sqrt((double)dt); A.max_t = max_t; A.rows = rows;
    A.per_trial_zs = (fam == FAM_RDM) ? 1 : 0;
    k_race_prep<<<(unsigned)((n_trials + 127) / 128), 128, 0, st>>>(A);
    SSM_CUDA(cudaGetLastError());
    RaceParams p;
    p.key = philox_keys(seed);
    p.rows = rows; p.row_floats = race_row_floats(np); p.offsets = offsets;
    p.order = (offsets && launch) ? launch->trial_order : nullptr;
    p.qoff = p.order ? launch->order_offsets : nullptr;
    p.n_trials = n_trials; p.total = total; p.np = np; p.dt = dt; p.smooth = smooth ? 1 : 0;
    p.k_base = (uint32_t)((launch && launch->first_trial > 0) ? launch->first_trial : 0);
    p.chunk = (launch && launch->chunk >= 32) ? launch->chunk : 64;
    p.refill_min = (launch && launch->refill_min > 0) ? min(launch->refill_min, 32) : SSM_REFILL_MIN_RACE;
    p.table = table; p.tstride = tstride; p.tlen = tlen;
    p.noise = noise; p.nlen = nlen; p.nunif = nunif;
    p.rts = rts; p.choices = choices; p.steps = steps; p.hdr = hdr;
    p.traj = traj; p.traj_len = traj_len;
    switch (fam) {
        case FAM_LCA: return race_dispatch<FAM_LCA>(np, bound, noise != nullptr, p, launch, st);
        case FAM_RDM: return race_dispatch<FAM_RDM>(np, bound, noise != nullptr, p, launch, st);
        default: return race_dispatch<FAM_RACE>(np, bound, noise != nullptr, p, launch, st);
    }
}

}  // namespace ssm

extern "C" {

size_t ssm_race_workspace_bytes(int64_t n_trials, int n_particles) {
    return ssm::race_ws_bytes(n_trials, n_particles);
}

int ssm_race_model(const float *v, const float *z, const float *t, const float *s,
                   const float *deadline, int64_t n_trials, int64_t n_samples, int n_particles,
                   const int64_t *sample_offsets, float max_t, float delta_t, int bound_kind,
                   const float *a, const float *bound_p1, const float *bound_p2,
                   const float *bound_table, int64_t table_stride, int64_t table_len,
                   uint64_t seed, int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                   const float *noise_unif, float *rts, int32_t *choices, int32_t *steps,
                   float *traj, int64_t traj_len, const ssm_launch *launch, void *workspace,
                   size_t workspace_bytes, void *stream) {
    return ssm::run_race(ssm::FAM_RACE, v, z, t, s, deadline, nullptr, nullptr, n_trials, n_samples,
                         n_particles, sample_offsets, max_t, delta_t, bound_kind, a, bound_p1,
                         bound_p2, bound_table, table_stride, table_len, seed, smooth_unif,
                         noise_rows, noise_row_len, noise_unif, rts, choices, steps, traj,
                         traj_len, launch, workspace, workspace_bytes, stream);
}

int ssm_lca(const float *v, const float *z, const float *g, const float *b, const float *t,
            const float *s, const float *deadline, int64_t n_trials, int64_t n_samples,
            int n_particles, const int64_t *sample_offsets, float max_t, float delta_t,
            int bound_kind, const float *a, const float *bound_p1, const float *bound_p2,
            const float *bound_table, int64_t table_stride, int64_t table_len, uint64_t seed,
            int smooth_unif, const float *noise_rows, int64_t noise_row_len,
            const float *noise_unif, float *rts, int32_t *choices, int32_t *steps, float *traj,
            int64_t traj_len, const ssm_launch *launch, void *workspace, size_t workspace_bytes,
            void *stream) {
    return ssm::run_race(ssm::FAM_LCA, v, z, t, s, deadline, g, b, n_trials, n_samples, n_particles,
                         sample_offsets, max_t, delta_t, bound_kind, a, bound_p1, bound_p2,
                         bound_table, table_stride, table_len, seed, smooth_unif, noise_rows,
                         noise_row_len, noise_unif, rts, choices, steps, traj, traj_len, launch,
                         workspace, workspace_bytes, stream);
}

int ssm_racing_diffusion(const float *v, const float *b, const float *A, const float *t, const float *s,
                         const float *deadline, int64_t n_trials, int64_t n_samples, int n_particles,
                         const int64_t *sample_offsets, float max_t, float delta_t, uint64_t seed,
                         int smooth_unif, const float *noise_rows, int64_t noise_row_len,
                         const float *noise_unif, float *rts, int32_t *choices, int32_t *steps,
                         float *traj, int64_t traj_len, const ssm_launch *launch, void *workspace,
                         size_t workspace_bytes, void *stream) {
    SSM_REQUIRE(n_trials == 0 || (b && A), "b and A are required");
    return ssm::run_race(ssm::FAM_RDM, v, A, t, s, deadline, nullptr, nullptr, n_trials, n_samples,
                         n_particles, sample_offsets, max_t, delta_t, SSM_BOUND_CONSTANT, b, nullptr,
                         nullptr, nullptr, 0, 0, seed, smooth_unif, noise_rows, noise_row_len,
                         noise_unif, rts, choices, steps, traj, traj_len, launch, workspace,
                         workspace_bytes, stream);
}

}  // extern "C"
