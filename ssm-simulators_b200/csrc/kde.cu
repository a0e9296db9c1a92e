// Batched log-rt Gaussian KDE for sm_100a: the reference's LogKDE
// (ssms/support_utils/kde_class.py) and the record layout of its
// ResampleMixtureStrategy (ssms/dataset_generators/strategies/
// resample_mixture_strategy.py:64-214), for many parameter sets at once.
//
// Layout.  Simulated data of set s occupies [soff[s], soff[s+1]) of rts /
// choices.  Group g = s * nc + c holds the log-rts of set s with choice c
// (omissions dropped) at points[poff[g] .. poff[g+1]), in sample order.
//
// Evaluation.  For a query log-rt q of group g the reference evaluates
//   log p_c + log( 1/(n h sqrt(2 pi)) sum_j exp(-(q - x_j)^2 / (2 h^2)) ) - q
// exactly (scikit-learn with atol = rtol = 0).  k_kde_eval tiles the group's
// points through shared memory, keeps QPT queries per thread in registers
// (q split into float hi + lo parts so q - x_j keeps full precision), evaluates
// each kernel term as ex2(-(d s)^2) on the SFU and sums in float over 32 terms
// before adding into a float64 accumulator.  Groups differ in cost by orders
// of magnitude (queries x points), so the work is scheduled Stream-K style
// (Osama, Merrill, Cecka, Garland & Owens, PPoPP'23): the iteration space
// (group, query tile, point tile) is cut into equal contiguous ranges, one per
// CTA of a persistent grid; query tiles cut between CTAs are finished by a
// fix-up kernel that adds the CTAs' partial sums in CTA order.
#include <algorithm>

#include "common.cuh"

namespace ssm {

constexpr int KDE_MAX_CHOICES = 16;
constexpr double KDE_LOG_2PI = 1.8378770664093453;

struct KdeFit {
    const float *rts;
    const int32_t *choices;
    int64_t n_sets;
    const int64_t *soff;
    const int32_t *cvals;
    int nc;
    const double *shift; // per-set displacement (displace_t) or nullptr
    double *bwvals;      // [total] displaced-mode bandwidth inputs, or nullptr
    int64_t *count_all;  // [G] samples with choice c, omissions included
    int64_t *n_valid;    // [G] non-omitted samples
    int64_t *poff;       // [G + 1]
    float *points;       // [total valid]
    double *h;           // [G] bandwidth (-1: no data)
    double *lognorm;     // [G] log p_c - log n - log h - log(2 pi)/2
    double *prop;        // [G] choice proportion
};

__device__ __forceinline__ int choice_index(int32_t ch, const int32_t *cvals, int nc) {
    for (int c = 0; c < nc; ++c)
        if (__ldg(cvals + c) == ch) return c;
    return -1;
}

__global__ void k_kde_count(const KdeFit a) {
    const int64_t s = blockIdx.x;
    __shared__ unsigned long long c_all[KDE_MAX_CHOICES], c_val[KDE_MAX_CHOICES];
    if (threadIdx.x < KDE_MAX_CHOICES) c_all[threadIdx.x] = c_val[threadIdx.x] = 0ull;
    __syncthreads();
    const int64_t lo = a.soff[s], hi = a.soff[s + 1];
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int ci = choice_index(a.choices[i], a.cvals, a.nc);
        if (ci >= 0) {
            atomicAdd(&c_all[ci], 1ull);
            if (a.rts[i] != -999.f) atomicAdd(&c_val[ci], 1ull);
        }
    }
    __syncthreads();
    if (threadIdx.x < a.nc) {
        a.count_all[s * a.nc + threadIdx.x] = (int64_t)c_all[threadIdx.x];
        a.n_valid[s * a.nc + threadIdx.x] = (int64_t)c_val[threadIdx.x];
    }
}

// Exclusive prefix sum of n int64 values into out[0..n] (one CTA of 1024).
__global__ void k_scan_i64(const int64_t *in, int64_t n, int64_t *out) {
    __shared__ int64_t warp_sum[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = 0; base < n; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = (i < n) ? in[i] : 0;
        int64_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int64_t w = (lane < (int)(blockDim.x >> 5)) ? warp_sum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sum[lane] = w;  // inclusive warp prefix
        }
        __syncthreads();
        const int64_t excl = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - v;
        if (i < n) out[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// Stable per-choice compaction of log(rt - shift) into the group regions.
__global__ void __launch_bounds__(256) k_kde_scatter(const KdeFit a) {
    const int64_t s = blockIdx.x;
    constexpr int W = 8;
    __shared__ int64_t base[KDE_MAX_CHOICES];
    __shared__ int wcnt[W][KDE_MAX_CHOICES];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    if (threadIdx.x < a.nc) base[threadIdx.x] = a.poff[s * a.nc + threadIdx.x];
    const double sh = a.shift ? a.shift[s] : 0.0;
    __syncthreads();
    const int64_t lo = a.soff[s], hi = a.soff[s + 1];
    for (int64_t c0 = lo; c0 < hi; c0 += blockDim.x) {
        const int64_t i = c0 + threadIdx.x;
        int ci = -1;
        float rt = 0.f;
        if (i < hi) {
            rt = a.rts[i];
            if (rt != -999.f) ci = choice_index(a.choices[i], a.cvals, a.nc);
        }
        int rank = 0;
        for (int c = 0; c < a.nc; ++c) {
            const unsigned m = __ballot_sync(0xffffffffu, ci == c);
            if (ci == c) rank = __popc(m & lt);
            if (lane == 0) wcnt[warp][c] = __popc(m);
        }
        __syncthreads();
        if (ci >= 0) {
            int64_t pos = base[ci] + rank;
            for (int w = 0; w < warp; ++w) pos += wcnt[w][ci];
            // kernels sit on float32 log of the float32 (displaced) rt; with a
            // shift the rt is displaced in float64 and stored as float32, and the
            // bandwidth uses log(exp(float32 log rt) - shift) in float64
            // (kde_class.py:174-186, 478-493)
            const float r = a.shift ? __double2float_rn((double)rt - sh) : rt;
            a.points[pos] = __double2float_rn(log((double)r));
            if (a.bwvals) a.bwvals[pos] = log(exp((double)__double2float_rn(log((double)rt))) - sh);
        }
        __syncthreads();
        if (threadIdx.x < a.nc) {
            int64_t t = 0;
            for (int w = 0; w < W; ++w) t += wcnt[w][threadIdx.x];
            base[threadIdx.x] += t;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ double block_sum_f64(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    __syncthreads();
    if (threadIdx.x == 0) red[0] = t;
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

// Silverman bandwidth (kde_class.py:508-553) and normaliser per group.
__global__ void __launch_bounds__(256) k_kde_stats(const KdeFit a) {
    const int64_t g = blockIdx.x;
    const int64_t s = g / a.nc;
    __shared__ double red[32];
    const int64_t lo = a.poff[g], n = a.poff[g + 1] - lo;
    double sum = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
        sum += a.bwvals ? a.bwvals[lo + i] : (double)a.points[lo + i];
    const double mean = block_sum_f64(sum, red) / (double)(n > 0 ? n : 1);
    double ss = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = (a.bwvals ? a.bwvals[lo + i] : (double)a.points[lo + i]) - mean;
        ss += d * d;
    }
    const double var = block_sum_f64(ss, red) / (double)(n > 0 ? n : 1);
    if (threadIdx.x == 0) {
        const int64_t N = a.soff[s + 1] - a.soff[s];
        const double p = (N > 0) ? (double)a.count_all[g] / (double)N : 0.0;
        a.prop[g] = p;
        if (n == 0) {
            a.h[g] = -1.0;
            a.lognorm[g] = 0.0;
        } else {
            double sd = (n > 1) ? sqrt(var) : 10.0;
            if (n > 1 && sd < 1e-3) sd = 1e-3;
            const double h = pow(4.0 / (3.0 * (double)n), 0.2) * sd;
            a.h[g] = h;
            a.lognorm[g] = log(p) - log((double)n) - log(h) - 0.5 * KDE_LOG_2PI;
        }
    }
}

struct KdeEval {
    const float *points;
    const int64_t *poff;
    const double *h, *lognorm;
    const int64_t *qoff;  // [G + 1] queries sorted by group
    const double *q_rt;
    double *out;
    int nc;
    int64_t G;
    const int64_t *soff;
    const double *shift;
    double lb, eps, max_t;
    // Stream-K schedule (see ssm_kde_eval): units are (group, tile of KDE_QT
    // queries); a unit's iterations are its group's point tiles.
    int64_t *uoff;     // [G + 1] first unit of each group
    int64_t *ucnt;     // [G] units per group (scan input)
    int64_t *ioff;     // [u_max + 1] first iteration of each unit
    int64_t *icnt;     // [u_max] iterations per unit (scan input)
    int64_t u_max;     // capacity of the unit arrays
    double *slots;     // [P][2][KDE_QT] partial sums of units split between CTAs
    int64_t P;         // CTAs of the evaluation grid
};

constexpr int KDE_TILE = 2048;
constexpr int KDE_QPT = 4;
constexpr int KDE_THREADS = 128;
constexpr int KDE_QT = KDE_QPT * KDE_THREADS;

__device__ __forceinline__ int64_t upper_index(const int64_t *off, int64_t n, int64_t x) {
    // largest i in [0, n) with off[i] <= x (off non-decreasing, off[0] <= x)
    int64_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (off[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void k_kde_units(const KdeEval a) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.G; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = a.qoff[g + 1] - a.qoff[g];
        a.ucnt[g] = (m + KDE_QT - 1) / KDE_QT;
    }
}

__global__ void k_kde_unit_iters(const KdeEval a) {
    const int64_t U = min(a.uoff[a.G], a.u_max);
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < a.u_max; u += (int64_t)gridDim.x * blockDim.x) {
        int64_t it = 0;
        if (u < U) {
            const int64_t g = upper_index(a.uoff, a.G + 1, u);
            const int64_t n = a.poff[g + 1] - a.poff[g];
            it = (n > 0) ? (n + KDE_TILE - 1) / KDE_TILE : 1;
        }
        a.icnt[u] = it;
    }
}

// first iteration of CTA c: floor(c * I / P) (c <= P < 2^16 and I < 2^46, so
// the product fits in 64 bits)
__device__ __forceinline__ int64_t sk_begin(int64_t c, int64_t I, int64_t P) {
    return (c * I) / P;
}
// the CTA whose iteration range holds iteration i (empty CTAs own nothing)
__device__ __forceinline__ int64_t sk_owner(int64_t i, int64_t I, int64_t P) {
    int64_t c = (i * P) / I;
    if (c > P - 1) c = P - 1;
    while (c > 0 && sk_begin(c, I, P) > i) --c;
    while (c + 1 < P && sk_begin(c + 1, I, P) <= i) ++c;
    return c;
}

// log-likelihood of one query from its kernel sum acc (kde_class.py:188-329)
__device__ __forceinline__ double kde_finalize(const KdeEval &a, int64_t g, int64_t n, double acc,
                                               double disp, double lq) {
    const int64_t s = g / a.nc;
    double ll;
    if (n == 0) {
        // choice without base data: log(1 / n_trials) + log(1 / max_t)
        ll = -log((double)(a.soff[s + 1] - a.soff[s]) * a.max_t);
    } else if (!(disp > 0.0)) {
        ll = a.lb;
    } else {
        ll = a.lognorm[g] + log(acc) - lq;
        if (!(ll > a.lb)) ll = a.lb;
    }
    return ll;
}

// Each thread holds KDE_QPT queries of the unit (q split into float hi + lo
// parts so q - x_j keeps full precision), the group's points stream through
// shared memory one tile per iteration, and each kernel term is
// ex2(-(d s)^2) on the SFU, summed in float over 32 terms before it is added
// into a float64 accumulator.
__global__ void __launch_bounds__(KDE_THREADS, 7) k_kde_eval(const KdeEval a) {
    __shared__ __align__(16) float tile[KDE_TILE];
    const int64_t U = min(a.uoff[a.G], a.u_max);
    const int64_t I = a.ioff[a.u_max];
    const int64_t c = blockIdx.x;
    const int64_t i0 = sk_begin(c, I, a.P), i1 = sk_begin(c + 1, I, a.P);
    if (i0 >= i1) return;
    int64_t u = upper_index(a.ioff, U, i0);
    int64_t g = upper_index(a.uoff, a.G + 1, u);
    for (int64_t it = i0; it < i1;) {
        while (a.uoff[g + 1] <= u) ++g;
        const int64_t ubeg = a.ioff[u], uend = a.ioff[u + 1];
        const int64_t lo = it, hi = (uend < i1) ? uend : i1;
        const int64_t q0 = a.qoff[g] + (u - a.uoff[g]) * KDE_QT, q1 = a.qoff[g + 1];
        const int64_t p0 = a.poff[g], n = a.poff[g + 1] - p0;
        const double hg = a.h[g];
        const double sh = a.shift ? a.shift[g / a.nc] : 0.0;
        // 2^(-(d*sc)^2) = exp(-d^2 / (2 h^2))
        const float sc = (n > 0) ? (float)(0.8493218002880191 / hg) : 0.f;  // sqrt(log2(e)/2) / h
        float qhi[KDE_QPT], qlo[KDE_QPT], part[KDE_QPT];
        double acc[KDE_QPT];
#pragma unroll
        for (int j = 0; j < KDE_QPT; ++j) {
            const int64_t qi = q0 + threadIdx.x + (int64_t)j * KDE_THREADS;
            const double lq = log(fmax((qi < q1) ? a.q_rt[qi] - sh : 1.0, a.eps));
            qhi[j] = (float)lq;
            qlo[j] = (float)(lq - (double)qhi[j]);
            part[j] = 0.f;
            acc[j] = 0.0;
        }
        for (int64_t t = lo - ubeg; t < hi - ubeg && n > 0; ++t) {
            const int64_t b0 = t * KDE_TILE;
            const int cnt = (int)min((int64_t)KDE_TILE, n - b0);
            __syncthreads();
            for (int i = threadIdx.x; i < KDE_TILE; i += KDE_THREADS)
                tile[i] = (i < cnt) ? __ldg(a.points + p0 + b0 + i) : qhi[0] + 1e30f;  // padding: zero weight
            __syncthreads();
            const float4 *t4 = reinterpret_cast<const float4 *>(tile);
            const int n4 = (cnt + 3) >> 2;
            for (int k0 = 0; k0 < n4; k0 += 8) {
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) {
                    const float4 x = t4[min(k0 + kk, KDE_TILE / 4 - 1)];
                    const bool live = (k0 + kk) < n4;
#pragma unroll
                    for (int j = 0; j < KDE_QPT; ++j) {
                        float d, e, r0, r1, r2, r3;
                        d = ((qhi[j] - x.x) + qlo[j]) * sc; e = -d * d;
                        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(e));
                        d = ((qhi[j] - x.y) + qlo[j]) * sc; e = -d * d;
                        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(e));
                        d = ((qhi[j] - x.z) + qlo[j]) * sc; e = -d * d;
                        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r2) : "f"(e));
                        d = ((qhi[j] - x.w) + qlo[j]) * sc; e = -d * d;
                        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r3) : "f"(e));
                        if (live) part[j] += (r0 + r1) + (r2 + r3);
                    }
                }
#pragma unroll
                for (int j = 0; j < KDE_QPT; ++j) {
                    acc[j] += (double)part[j];
                    part[j] = 0.f;
                }
            }
        }
        if (lo == ubeg && hi == uend) {
#pragma unroll
            for (int j = 0; j < KDE_QPT; ++j) {
                const int64_t qi = q0 + threadIdx.x + (int64_t)j * KDE_THREADS;
                if (qi < q1) {
                    const double disp = a.q_rt[qi] - sh;
                    a.out[qi] = kde_finalize(a, g, n, acc[j], disp, log(fmax(disp, a.eps)));
                }
            }
        } else {
            // split unit: slot 0 (head) if it began in an earlier CTA, else slot 1 (tail)
            double *slot = a.slots + (c * 2 + (ubeg < i0 ? 0 : 1)) * KDE_QT;
#pragma unroll
            for (int j = 0; j < KDE_QPT; ++j) slot[threadIdx.x + j * KDE_THREADS] = acc[j];
        }
        it = hi;
        ++u;
    }
}

// Units split between CTAs: their partial sums are added in CTA order (a fixed
// order, so results do not depend on timing) and finalised.
__global__ void __launch_bounds__(KDE_THREADS) k_kde_fixup(const KdeEval a) {
    const int64_t U = min(a.uoff[a.G], a.u_max);
    const int64_t I = a.ioff[a.u_max];
    for (int64_t u = blockIdx.x; u < U; u += gridDim.x) {
        const int64_t ubeg = a.ioff[u], uend = a.ioff[u + 1];
        const int64_t c0 = sk_owner(ubeg, I, a.P), c1 = sk_owner(uend - 1, I, a.P);
        if (c0 == c1) continue;
        const int64_t g = upper_index(a.uoff, a.G + 1, u);
        const int64_t q0 = a.qoff[g] + (u - a.uoff[g]) * KDE_QT, q1 = a.qoff[g + 1];
        const int64_t n = a.poff[g + 1] - a.poff[g];
        const double sh = a.shift ? a.shift[g / a.nc] : 0.0;
        for (int j = 0; j < KDE_QPT; ++j) {
            const int r = threadIdx.x + j * KDE_THREADS;
            const int64_t qi = q0 + r;
            if (qi >= q1) continue;
            double acc = a.slots[(c0 * 2 + 1) * KDE_QT + r];
            for (int64_t cc = c0 + 1; cc <= c1; ++cc)
                if (sk_begin(cc, I, a.P) < sk_begin(cc + 1, I, a.P)) acc += a.slots[(cc * 2) * KDE_QT + r];
            const double disp = a.q_rt[qi] - sh;
            a.out[qi] = kde_finalize(a, g, n, acc, disp, log(fmax(disp, a.eps)));
        }
    }
}

// Queries / samples per group: slots [o[g], o[g] + nk[g]) get KDE samples
// (point j ~ U{0..n-1}, log-rt + h N(0,1), exponentiated, plus the shift);
// the following nu[g] slots get U(ulo, uhi) rts.  Groups without data draw
// their KDE part from U(0, max_t) as the reference does.
struct KdeSample {
    PhiloxKeys key;
    const float *points;
    const int64_t *poff;
    const double *h;
    const int64_t *ooff;    // [G + 1] output slots per group
    const int64_t *nkde;    // [G] KDE samples at the start of each group's slots
    int64_t n_groups;
    const double *shift;
    int nc;
    double max_t, ulo, uhi;
    double *out_rt;
};

__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

__global__ void k_kde_sample(const KdeSample a) {
    const int64_t total = a.ooff[a.n_groups];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = a.n_groups;  // ooff[lo] <= i < ooff[hi]
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (a.ooff[mid] <= i) lo = mid; else hi = mid;
        }
        const int64_t g = lo, j = i - a.ooff[g];
        const uint4 r = philox10(make_uint4((uint32_t)j, (uint32_t)g, (uint32_t)(g >> 32), 7u), a.key);
        const double sh = a.shift ? a.shift[g / a.nc] : 0.0;
        const int64_t n = a.poff[g + 1] - a.poff[g];
        double rt;
        if (j < a.nkde[g]) {
            if (n > 0) {
                int64_t idx = (int64_t)(u53(r.x, r.y) * (double)n);
                if (idx >= n) idx = n - 1;
                const float2 z = box_muller(r.z, r.w);
                rt = exp((double)a.points[a.poff[g] + idx] + a.h[g] * (double)z.x) + sh;
            } else {
                rt = u53(r.x, r.y) * a.max_t + sh;
            }
        } else {
            rt = a.ulo + u53(r.x, r.y) * (a.uhi - a.ulo);
        }
        a.out_rt[i] = rt;
    }
}

// Training records (ResampleMixtureStrategy layout): per set s, rows
// [theta_0..theta_{P-1}, rt, choice, loglik] as float32.  The evaluated
// queries of the set's groups come first, then n_down rows with
// rt ~ U(-1, 0.0001), a uniformly drawn choice and loglik = neg_ll; rows are
// shuffled within the set (Fisher-Yates driven by Philox).
struct KdeRecords {
    PhiloxKeys key;
    const float *theta;  // [S, P]
    int P;
    int64_t n_sets;
    const int64_t *qoff;  // [G + 1]
    const double *q_rt, *q_ll;
    const int32_t *cvals;
    int nc;
    int64_t n_down;  // per set
    int64_t rows_per_set;
    float neg_ll;
    float *out;      // [S * rows_per_set, P + 3]
};

__global__ void __launch_bounds__(256) k_kde_records(const KdeRecords a) {
    extern __shared__ int perm[];
    const int64_t s = blockIdx.x;
    const int64_t M = a.rows_per_set;
    const int64_t qa = a.qoff[s * a.nc], qb = a.qoff[(s + 1) * a.nc];
    for (int64_t i = threadIdx.x; i < M; i += blockDim.x) perm[i] = (int)i;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int64_t i = M - 1; i > 0; --i) {
            const uint4 r = philox10(make_uint4((uint32_t)i, (uint32_t)s, (uint32_t)(s >> 32), 9u), a.key);
            const int64_t j = (int64_t)(u53(r.x, r.y) * (double)(i + 1));
            const int tmp = perm[i];
            perm[i] = perm[j <= i ? j : i];
            perm[j <= i ? j : i] = tmp;
        }
    }
    __syncthreads();
    const int W = a.P + 3;
    for (int64_t i = threadIdx.x; i < M; i += blockDim.x) {
        float *row = a.out + (s * M + perm[i]) * W;
        for (int p = 0; p < a.P; ++p) row[p] = a.theta[s * a.P + p];
        float rt, ch, ll;
        const int64_t q = qa + i;
        if (q < qb) {
            int64_t c = 0;  // group of query q within this set
            while (c + 1 < a.nc && a.qoff[s * a.nc + c + 1] <= q) ++c;
            rt = (float)a.q_rt[q];
            ch = (float)a.cvals[c];
            ll = (float)a.q_ll[q];
        } else {
            const uint4 r = philox10(make_uint4((uint32_t)i, (uint32_t)s, (uint32_t)(s >> 32), 11u), a.key);
            rt = (float)(-1.0 + u53(r.x, r.y) * (0.0001 + 1.0));
            ch = (float)a.cvals[min((int)(u53(r.z, r.w) * a.nc), a.nc - 1)];
            ll = a.neg_ll;
        }
        row[a.P] = rt;
        row[a.P + 1] = ch;
        row[a.P + 2] = ll;
    }
}

// Per-set summaries for the auxiliary labels of the data pipeline
// (simulation_pipeline.py:262-351): choice counts, the pipeline's omission
// count (choices equal to -999), no-go count ((choice != max choice) or rt ==
// -999) and per-choice rt histograms over np.linspace(0, max_t, nb + 1) with
// numpy's index rules (right edge inclusive in the last bin, float64 edges,
// +-1 corrections at the edges), omissions excluded.
struct SetSummary {
    const float *rts;
    const int32_t *choices;
    const int64_t *soff;
    const int32_t *cvals;
    int nc;
    double max_t;
    int64_t *counts, *nogo, *omit;
    int nb_a, nb_b;
    float *hist_a, *hist_b;
};

__device__ __forceinline__ int np_hist_index(double v, double max_t, int nb) {
    if (!(v >= 0.0) || !(v <= max_t)) return -1;
    const double step = max_t / (double)nb;
    int i = (int)((v / max_t) * (double)nb);
    if (i == nb) i -= 1;
    const double lo = (double)i * step;
    if (v < lo) i -= 1;
    const double hi = (i + 1 == nb) ? max_t : (double)(i + 1) * step;
    if (i != nb - 1 && v >= hi) i += 1;
    return i;
}

__global__ void __launch_bounds__(256) k_set_summary(const SetSummary a) {
    extern __shared__ unsigned int sh[];  // [nc * (nb_a + nb_b)] histogram counters
    __shared__ unsigned long long cnt[KDE_MAX_CHOICES];
    __shared__ unsigned long long nogo, omit;
    const int64_t s = blockIdx.x;
    const int H = a.nc * (a.nb_a + a.nb_b);
    int32_t max_choice = __ldg(a.cvals);
    for (int c = 1; c < a.nc; ++c) max_choice = max(max_choice, __ldg(a.cvals + c));
    for (int i = threadIdx.x; i < H; i += blockDim.x) sh[i] = 0u;
    if (threadIdx.x < KDE_MAX_CHOICES) cnt[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) nogo = omit = 0ull;
    __syncthreads();
    for (int64_t i = a.soff[s] + threadIdx.x; i < a.soff[s + 1]; i += blockDim.x) {
        const int32_t ch = a.choices[i];
        const float rt = a.rts[i];
        if (ch == -999) atomicAdd(&omit, 1ull);
        if (ch != max_choice || rt == -999.f) atomicAdd(&nogo, 1ull);
        const int c = choice_index(ch, a.cvals, a.nc);
        if (c < 0) continue;
        atomicAdd(&cnt[c], 1ull);
        if (rt == -999.f) continue;
        const int ia = np_hist_index((double)rt, a.max_t, a.nb_a);
        if (ia >= 0) atomicAdd(&sh[c * a.nb_a + ia], 1u);
        const int ib = np_hist_index((double)rt, a.max_t, a.nb_b);
        if (ib >= 0) atomicAdd(&sh[a.nc * a.nb_a + c * a.nb_b + ib], 1u);
    }
    __syncthreads();
    if (threadIdx.x < a.nc) a.counts[s * a.nc + threadIdx.x] = (int64_t)cnt[threadIdx.x];
    if (threadIdx.x == 0) {
        a.nogo[s] = (int64_t)nogo;
        a.omit[s] = (int64_t)omit;
    }
    // layout [S, nb, nc] like the pipeline's binned_128 / binned_256 arrays
    for (int i = threadIdx.x; i < a.nc * a.nb_a; i += blockDim.x) {
        const int c = i / a.nb_a, b = i % a.nb_a;
        a.hist_a[(s * a.nb_a + b) * a.nc + c] = (float)sh[i];
    }
    for (int i = threadIdx.x; i < a.nc * a.nb_b; i += blockDim.x) {
        const int c = i / a.nb_b, b = i % a.nb_b;
        a.hist_b[(s * a.nb_b + b) * a.nc + c] = (float)sh[a.nc * a.nb_a + i];
    }
}

}  // namespace ssm

extern "C" {

int ssm_set_summary(const float *rts, const int32_t *choices, int64_t n_sets,
                    const int64_t *sample_offsets, const int32_t *choice_values, int n_choices,
                    double max_t, int64_t *choice_counts, int64_t *nogo_counts,
                    int64_t *omission_counts, int nbins_a, float *hist_a, int nbins_b,
                    float *hist_b, void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_sets >= 0 && n_choices >= 1 && n_choices <= KDE_MAX_CHOICES, "bad n_sets / n_choices");
    SSM_REQUIRE(nbins_a >= 1 && nbins_b >= 1 && (size_t)n_choices * (nbins_a + nbins_b) * 4 <= 48 * 1024,
                "histograms must fit in 48 KB of shared memory");
    if (n_sets == 0) return SSM_OK;
    SSM_REQUIRE(rts && choices && sample_offsets && choice_values && choice_counts && nogo_counts &&
                omission_counts && hist_a && hist_b, "all buffers are required");
    SetSummary a;
    a.rts = rts; a.choices = choices; a.soff = sample_offsets; a.cvals = choice_values;
    a.nc = n_choices; a.max_t = max_t; a.counts = choice_counts; a.nogo = nogo_counts;
    a.omit = omission_counts; a.nb_a = nbins_a; a.nb_b = nbins_b; a.hist_a = hist_a; a.hist_b = hist_b;
    const size_t smem = (size_t)n_choices * (nbins_a + nbins_b) * sizeof(unsigned int);
    k_set_summary<<<(unsigned)n_sets, 256, smem, (cudaStream_t)stream>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

int ssm_kde_fit(const float *rts, const int32_t *choices, int64_t n_sets,
                const int64_t *sample_offsets, const int32_t *choice_values, int n_choices,
                const double *displace, double *displaced_logs, int64_t *count_all,
                int64_t *n_valid, int64_t *point_offsets, float *points, double *bandwidth,
                double *log_norm, double *proportion, void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_sets >= 0, "n_sets must be >= 0");
    SSM_REQUIRE(n_choices >= 1 && n_choices <= KDE_MAX_CHOICES, "n_choices must be in [1, %d]", KDE_MAX_CHOICES);
    SSM_REQUIRE(n_sets == 0 || (rts && choices && sample_offsets && choice_values && count_all &&
                                n_valid && point_offsets && points && bandwidth && log_norm && proportion),
                "all buffers are required");
    if (n_sets == 0) return SSM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    SSM_REQUIRE(!displace || displaced_logs, "displace needs the displaced_logs buffer");
    KdeFit a{rts, choices, n_sets, sample_offsets, choice_values, n_choices, displace,
             displace ? displaced_logs : nullptr, count_all, n_valid, point_offsets, points,
             bandwidth, log_norm, proportion};
    const int64_t G = n_sets * n_choices;
    k_kde_count<<<(unsigned)n_sets, 256, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    k_scan_i64<<<1, 1024, 0, st>>>(n_valid, G, point_offsets);
    SSM_CUDA(cudaGetLastError());
    k_kde_scatter<<<(unsigned)n_sets, 256, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    k_kde_stats<<<(unsigned)G, 256, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

}  // extern "C"

namespace ssm {

// CTAs of the evaluation grid: every SM filled to the kernel's occupancy.
static int64_t kde_eval_ctas() {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kde_eval, KDE_THREADS, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    return (int64_t)per_sm * sm_count();
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct KdeEvalLayout {
    size_t uoff, ucnt, ioff, icnt, slots, total;
    int64_t u_max, P;
};

static KdeEvalLayout kde_eval_layout(int64_t G, int64_t n_queries) {
    KdeEvalLayout L;
    L.P = kde_eval_ctas();
    L.u_max = n_queries / KDE_QT + G + 1;
    L.uoff = 0;
    L.ucnt = L.uoff + align256((size_t)(G + 1) * 8);
    L.ioff = L.ucnt + align256((size_t)G * 8);
    L.icnt = L.ioff + align256((size_t)(L.u_max + 1) * 8);
    L.slots = L.icnt + align256((size_t)L.u_max * 8);
    L.total = L.slots + (size_t)L.P * 2 * KDE_QT * sizeof(double);
    return L;
}

}  // namespace ssm

extern "C" {

size_t ssm_kde_eval_workspace_bytes(int64_t n_sets, int n_choices, int64_t n_queries) {
    if (n_sets < 0 || n_choices < 1 || n_queries < 0) return 0;
    return ssm::kde_eval_layout(n_sets * n_choices, n_queries).total;
}

int ssm_kde_eval(const float *points, const int64_t *point_offsets, const double *bandwidth,
                 const double *log_norm, int64_t n_sets, int n_choices,
                 const int64_t *sample_offsets, const double *displace,
                 const int64_t *query_offsets, const double *query_rt, int64_t n_queries, double lb,
                 double eps, double max_t, void *workspace, size_t workspace_bytes,
                 double *out_loglik, void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_sets >= 0 && n_choices >= 1 && n_choices <= KDE_MAX_CHOICES, "bad n_sets / n_choices");
    SSM_REQUIRE(n_queries >= 0, "n_queries must be >= 0");
    if (n_sets == 0 || n_queries == 0) return SSM_OK;
    SSM_REQUIRE(points && point_offsets && bandwidth && log_norm && sample_offsets && query_offsets &&
                query_rt && out_loglik && workspace, "all buffers are required");
    const int64_t G = n_sets * n_choices;
    const KdeEvalLayout L = kde_eval_layout(G, n_queries);
    SSM_REQUIRE(workspace_bytes >= L.total, "workspace too small: %zu bytes, need %zu (ssm_kde_eval_workspace_bytes)",
                workspace_bytes, L.total);
    SSM_REQUIRE(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
    uint8_t *ws = static_cast<uint8_t *>(workspace);
    KdeEval a;
    a.points = points; a.poff = point_offsets; a.h = bandwidth; a.lognorm = log_norm;
    a.qoff = query_offsets; a.q_rt = query_rt; a.out = out_loglik; a.nc = n_choices; a.G = G;
    a.soff = sample_offsets; a.shift = displace; a.lb = lb; a.eps = eps; a.max_t = max_t;
    a.uoff = reinterpret_cast<int64_t *>(ws + L.uoff);
    a.ucnt = reinterpret_cast<int64_t *>(ws + L.ucnt);
    a.ioff = reinterpret_cast<int64_t *>(ws + L.ioff);
    a.icnt = reinterpret_cast<int64_t *>(ws + L.icnt);
    a.u_max = L.u_max;
    a.slots = reinterpret_cast<double *>(ws + L.slots);
    a.P = L.P;
    cudaStream_t st = (cudaStream_t)stream;
    const int ng = (int)std::min<int64_t>((G + 255) / 256, 4096);
    k_kde_units<<<ng, 256, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    k_scan_i64<<<1, 1024, 0, st>>>(a.ucnt, G, a.uoff);
    SSM_CUDA(cudaGetLastError());
    const int nu = (int)std::min<int64_t>((L.u_max + 255) / 256, 4096);
    k_kde_unit_iters<<<nu, 256, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    k_scan_i64<<<1, 1024, 0, st>>>(a.icnt, L.u_max, a.ioff);
    SSM_CUDA(cudaGetLastError());
    k_kde_eval<<<(unsigned)L.P, KDE_THREADS, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    k_kde_fixup<<<(unsigned)std::min<int64_t>(L.u_max, 65535), KDE_THREADS, 0, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

int ssm_kde_sample(const float *points, const int64_t *point_offsets, const double *bandwidth,
                   int64_t n_sets, int n_choices, const double *displace,
                   const int64_t *out_offsets, const int64_t *n_kde, uint64_t seed, double max_t,
                   double unif_lo, double unif_hi, double *out_rt, void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_sets >= 0 && n_choices >= 1 && n_choices <= KDE_MAX_CHOICES, "bad n_sets / n_choices");
    if (n_sets == 0) return SSM_OK;
    SSM_REQUIRE(points && point_offsets && bandwidth && out_offsets && n_kde && out_rt, "all buffers are required");
    KdeSample a;
    a.key = philox_keys(seed);
    a.points = points; a.poff = point_offsets; a.h = bandwidth; a.ooff = out_offsets; a.nkde = n_kde;
    a.n_groups = n_sets * n_choices; a.shift = displace; a.nc = n_choices; a.max_t = max_t;
    a.ulo = unif_lo; a.uhi = unif_hi; a.out_rt = out_rt;
    k_kde_sample<<<sm_count() * 8, 256, 0, (cudaStream_t)stream>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

int ssm_kde_records(const float *theta, int n_params, int64_t n_sets, int n_choices,
                    const int32_t *choice_values, const int64_t *query_offsets,
                    const double *query_rt, const double *query_loglik, int64_t n_down,
                    int64_t rows_per_set, float negative_rt_loglik, uint64_t seed, float *out,
                    void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_sets >= 0 && n_params >= 1 && n_choices >= 1 && n_choices <= KDE_MAX_CHOICES, "bad sizes");
    SSM_REQUIRE(rows_per_set >= 1 && rows_per_set <= 12288, "rows_per_set must be in [1, 12288]");
    if (n_sets == 0) return SSM_OK;
    SSM_REQUIRE(theta && choice_values && query_offsets && query_rt && query_loglik && out, "all buffers are required");
    KdeRecords a;
    a.key = philox_keys(seed);
    a.theta = theta; a.P = n_params; a.n_sets = n_sets; a.qoff = query_offsets; a.q_rt = query_rt;
    a.q_ll = query_loglik; a.cvals = choice_values; a.nc = n_choices; a.n_down = n_down;
    a.rows_per_set = rows_per_set; a.neg_ll = negative_rt_loglik; a.out = out;
    k_kde_records<<<(unsigned)n_sets, 256, rows_per_set * sizeof(int), (cudaStream_t)stream>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

}  // extern "C"
