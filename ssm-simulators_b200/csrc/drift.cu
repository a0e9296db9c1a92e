// Drift tables v(t_i) of the registered drift functions, evaluated on the device.
//
// ddm_flex reads one float32 drift value per trial and time step.  The
// reference evaluates drift_fun(t=t_s, **params_k) in numpy once per trial
// (src/cssm/ddm_models.pyx:1063-1066) -- about 0.1 ms of host time per trial
// on the 20 001-point grid.  Here every (trial, time) entry is one thread.
// Each formula follows the dtype flow of the reference's numpy code
// (ssms/basic_simulators/drift_functions.py): float32 parameters and grid,
// float32 arithmetic without contraction, float64 where scipy's normal
// distribution functions take over (the attention drifts).  The math library
// differs from numpy's, so values agree to a few float32 ulps, not bit for
// bit; the bit-exact noise-injection path keeps the host tables.
#include <math.h>

#include "common.cuh"

namespace ssm {

struct DriftArgs {
    int kind;
    const float *params;  // [n_params][n_trials]
    int n_params;
    int64_t n_trials;
    const float *t_s;
    int64_t t_len;
    float *table;         // [n_trials][stride]
    int64_t stride;
};

// target / distractor course: (init - fix) exp(-(slope t)) + fix in float32
__device__ __forceinline__ float ds_course(float init, float fix, float slope, float t) {
    return __fadd_rn(__fmul_rn(__fsub_rn(init, fix), expf(-__fmul_rn(slope, t))), fix);
}

// numpy.stimflex_support: coh on onset <= t <= offset, 0 elsewhere
__device__ __forceinline__ float pulse(float t, float onset, float offset, float coh) {
    return (t >= onset && t <= offset) ? coh : 0.f;
}

// scipy.stats.norm.cdf(x, loc=0, scale=w) in float64
__device__ __forceinline__ double norm_cdf(double x, double w) { return 0.5 * erfc(-(x / w) * 0.70710678118654752440); }

__device__ __forceinline__ float drift_value(const DriftArgs &a, int64_t k, float t, float t_end) {
    const float *P = a.params + k;
    auto prm = [&](int j) { return __ldg(P + (int64_t)j * a.n_trials); };
    switch (a.kind) {
        case SSM_DRIFT_CONSTANT:
            return prm(0);
        case SSM_DRIFT_GAMMA: {
            // v + c * (t^(shape-1) exp(-t/scale)) / ((shape-1)^(shape-1) scale^(shape-1) exp(-(shape-1)))
            const float v = prm(0), s1 = __fsub_rn(prm(1), 1.f), scale = prm(2), c = prm(3);
            const float pulse_ = __fmul_rn(powf(t, s1), expf(__fdiv_rn(-t, scale)));
            const float peak = __fmul_rn(__fmul_rn(powf(s1, s1), powf(scale, s1)), expf(-s1));
            return __fadd_rn(v, __fmul_rn(c, __fdiv_rn(pulse_, peak)));
        }
        case SSM_DRIFT_CONFLICT_DS: {
            // v + ((target * tcoh) + (distractor * dcoh)); params v, tinit, dinit, tslope, dslope, tfixedp, tcoh, dcoh
            const float target = ds_course(prm(1), prm(5), prm(3), t);
            const float distractor = ds_course(prm(2), 0.f, prm(4), t);
            return __fadd_rn(prm(0), __fadd_rn(__fmul_rn(target, prm(6)), __fmul_rn(distractor, prm(7))));
        }
        case SSM_DRIFT_CONFLICT_DSSTIMFLEX: {
            // as conflict_ds with target / distractor switched on at their onsets, relative to the first
            float ton = prm(8), don = prm(9);
            const float first = fminf(ton, don);
            ton = __fsub_rn(ton, first);
            don = __fsub_rn(don, first);
            const float target = ds_course(prm(1), prm(5), prm(3), t);
            const float distractor = ds_course(prm(2), 0.f, prm(4), t);
            return __fadd_rn(prm(0), __fadd_rn(__fmul_rn(target, pulse(t, ton, t_end, prm(6))),
                                               __fmul_rn(distractor, pulse(t, don, t_end, prm(7)))));
        }
        case SSM_DRIFT_CONFLICT_STIMFLEX:
        case SSM_DRIFT_CONFLICT_STIMFLEXREL1: {
            // v + (vt * target pulse + vd * distractor pulse); params v, vt, vd, tcoh, dcoh, tonset, donset
            float ton = prm(5), don = prm(6);
            if (a.kind == SSM_DRIFT_CONFLICT_STIMFLEXREL1) {
                const float first = fminf(ton, don);
                ton = __fsub_rn(ton, first);
                don = __fsub_rn(don, first);
            }
            return __fadd_rn(prm(0), __fadd_rn(__fmul_rn(prm(1), pulse(t, ton, t_end, prm(3))),
                                               __fmul_rn(prm(2), pulse(t, don, t_end, prm(4)))));
        }
        case SSM_DRIFT_ATTEND: {
            // spotlight width w = max(sda - r t, 0.001) in float32, then float64;
            // params v, ptarget, pouter, pinner, r, sda
            const double w = (double)fmaxf(__fsub_rn(prm(5), __fmul_rn(prm(4), t)), 0.001f);
            const double outer = 0.5 * erfc((1.5 / w) * 0.70710678118654752440);
            const double inner = norm_cdf(1.5, w) - norm_cdf(0.5, w);
            const double target = norm_cdf(0.5, w) - norm_cdf(-0.5, w);
            const double s = ((double)(2.f * prm(2)) * outer + (double)(2.f * prm(3)) * inner) + (double)prm(1) * target;
            return (float)((double)prm(0) + s);
        }
        case SSM_DRIFT_ATTEND_SIMPLE: {
            // params v, ptarget, pouter, r, sda
            const double w = (double)fmaxf(__fsub_rn(prm(4), __fmul_rn(prm(3), t)), 0.001f);
            const double outer = 1.0 - norm_cdf(0.5, w);
            const double target = norm_cdf(0.5, w) - 0.5;
            const double s = (double)(2.f * prm(2)) * outer + (double)(2.f * prm(1)) * target;
            return (float)((double)prm(0) + s);
        }
        default:
            return 0.f;
    }
}

__global__ void k_drift_table(const DriftArgs a) {
    const float t_end = __ldg(a.t_s + a.t_len - 1);  // np.max of the increasing grid
    const int64_t n = a.n_trials * a.stride;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / a.stride, j = i - k * a.stride;
        a.table[i] = (j < a.t_len) ? drift_value(a, k, __ldg(a.t_s + j), t_end) : 0.f;
    }
}

static int n_drift_params(int kind) {
    switch (kind) {
        case SSM_DRIFT_CONSTANT: return 1;
        case SSM_DRIFT_GAMMA: return 4;
        case SSM_DRIFT_CONFLICT_DS: return 8;
        case SSM_DRIFT_CONFLICT_DSSTIMFLEX: return 10;
        case SSM_DRIFT_CONFLICT_STIMFLEX:
        case SSM_DRIFT_CONFLICT_STIMFLEXREL1: return 7;
        case SSM_DRIFT_ATTEND: return 6;
        case SSM_DRIFT_ATTEND_SIMPLE: return 5;
        default: return -1;
    }
}

}  // namespace ssm

extern "C" int ssm_drift_table(int kind, const float *params, int n_params, int64_t n_trials, const float *t_s,
                               int64_t t_len, float *table, int64_t stride, void *stream) {
    const int need = ssm::n_drift_params(kind);
    SSM_REQUIRE(need > 0, "ssm_drift_table: unknown drift kind %d", kind);
    SSM_REQUIRE(n_params == need, "ssm_drift_table: drift kind %d takes %d parameters (got %d)", kind, need,
                n_params);
    SSM_REQUIRE(n_trials >= 0 && t_len >= 1 && stride >= t_len, "ssm_drift_table: bad sizes");
    if (n_trials == 0) return SSM_OK;
    SSM_REQUIRE(params && t_s && table, "ssm_drift_table: null pointer");
    ssm::DriftArgs a{kind, params, n_params, n_trials, t_s, t_len, table, stride};
    const int64_t n = n_trials * stride;
    const int64_t cap = (int64_t)ssm::sm_count() * 8;
    const int grid = (int)((n + 255) / 256 < cap ? (n + 255) / 256 : cap);
    ssm::k_drift_table<<<grid, 256, 0, (cudaStream_t)stream>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}
