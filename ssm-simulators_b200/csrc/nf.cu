// First-passage-time log-density of the Wiener diffusion model and its
// analytic gradient, in float64, one thread per query: the exact reference
// the constant-bound DDM simulator and the surrogate's theta-gradient are
// judged against.  The reference has no analytic density.
//
// Navarro & Fuss (2009), J. Math. Psychol. 53:222-230: the lower-barrier
// density for drift v, separation A, relative start w, unit noise is
//     f(T) = A^-2 exp(-v A w - v^2 T / 2) g(T / A^2, w)
// with g from the small-time series (2 pi u^3)^-1/2 sum_k (w + 2k) exp(-(w + 2k)^2 / 2u)
// or the large-time series pi sum_k k exp(-k^2 pi^2 u / 2) sin(k pi w),
// whichever needs fewer terms by the paper's bounds (eps = 1e-14 here, plus
// four guard terms).  The upper barrier is v -> -v, w -> 1 - w; noise s
// enters as v / s and A / s.
//
// Parameterisation of the reference's ddm / ddm_flexbound with a constant
// bound (src/cssm/ddm_models.pyx): bounds +-a, start -a + 2 z a, choice +1
// at the upper bound, non-decision time t -- i.e. A = 2a, w = z, T = rt - t.
#include <math.h>

#include "common.cuh"

namespace ssm {
namespace nf {

constexpr double PI = 3.141592653589793238462643383279502884;

// log g and the ratios (dg/du) / g, (dg/dw) / g.  Each series is summed
// relative to its leading term (exp(-w^2 / 2u) small-time, exp(-pi^2 u / 2)
// large-time), so log g stays finite where g itself would underflow.
struct LogG {
    double logg, ru, rw;
};

__device__ LogG g_series(double u, double w, double eps) {
    LogG r;
    // term counts (Navarro & Fuss truncation bounds for the two series)
    double kl = 1.0 / (PI * sqrt(u));
    if (PI * u * eps < 1.0) kl = fmax(kl, sqrt(fmax(-2.0 * log(PI * u * eps) / (PI * PI * u), 0.0)));
    double ks = sqrt(u) + 1.0;
    const double arg = 2.0 * sqrt(2.0 * PI * u) * eps;
    ks = fmax(ks, arg < 1.0 ? 2.0 + sqrt(fmax(-2.0 * u * log(arg), 0.0)) : 2.0);
    if (ks < kl) {
        const int K = (int)ceil(ks) + 4;
        double s0 = 0.0, sw = 0.0, su = 0.0;
        for (int k = -K; k <= K; ++k) {
            const double c = w + 2.0 * k;
            const double e = exp(-(c * c - w * w) / (2.0 * u));
            s0 += c * e;
            sw += (1.0 - c * c / u) * e;
            su += c * e * (c * c / (2.0 * u * u) - 1.5 / u);
        }
        r.logg = -0.5 * log(2.0 * PI * u * u * u) - w * w / (2.0 * u) + log(s0);
        r.rw = sw / s0;
        r.ru = su / s0;
    } else {
        const int K = (int)ceil(kl) + 4;
        double s0 = 0.0, sw = 0.0, su = 0.0;
        for (int k = 1; k <= K; ++k) {
            const double kk = (double)k;
            const double e = exp(-(kk * kk - 1.0) * PI * PI * u / 2.0);
            double sn, cs;
            sincospi(kk * w, &sn, &cs);
            s0 += kk * e * sn;
            sw += kk * e * kk * PI * cs;
            su += kk * e * sn * (-kk * kk * PI * PI / 2.0);
        }
        r.logg = log(PI) - PI * PI * u / 2.0 + log(s0);
        r.rw = sw / s0;
        r.ru = su / s0;
    }
    return r;
}

// grad layout per query: d/dv, d/da, d/dz, d/dt
__global__ void k_ddm_nf(const double *__restrict__ rt, const int32_t *__restrict__ choice,
                         const double *__restrict__ v, const double *__restrict__ a, const double *__restrict__ z,
                         const double *__restrict__ t, const double *__restrict__ s, int64_t n, int64_t pstride,
                         double eps, double *__restrict__ out, double *__restrict__ grad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t j = pstride ? i : 0;
    const double T = rt[i] - t[j];
    const bool up = choice[i] > 0;
    const double sc = s ? s[j] : 1.0;
    const double vv = (up ? -v[j] : v[j]) / sc;
    const double ww = up ? 1.0 - z[j] : z[j];
    const double A = 2.0 * a[j] / sc;
    if (!(T > 0.0)) {
        out[i] = -INFINITY;
        if (grad)
            for (int q = 0; q < 4; ++q) grad[4 * i + q] = NAN;
        return;
    }
    const double u = T / (A * A);
    const LogG r = g_series(u, ww, eps);
    out[i] = -vv * A * ww - vv * vv * T / 2.0 + r.logg - 2.0 * log(A);
    if (grad) {
        // d log f w.r.t. the lower-barrier arguments, then chained to (v, a, z, t)
        const double d_vv = -A * ww - vv * T;
        const double d_A = -2.0 / A - vv * ww + r.ru * (-2.0 * T / (A * A * A));
        const double d_ww = -vv * A + r.rw;
        const double d_T = -vv * vv / 2.0 + r.ru / (A * A);
        const double sg = up ? -1.0 : 1.0;
        grad[4 * i + 0] = sg * d_vv / sc;
        grad[4 * i + 1] = 2.0 * d_A / sc;
        grad[4 * i + 2] = sg * d_ww;
        grad[4 * i + 3] = -d_T;
    }
}

}  // namespace nf
}  // namespace ssm

extern "C" int ssm_ddm_nf_loglik(const double *rt, const int32_t *choice, const double *v, const double *a,
                                 const double *z, const double *t, const double *s, int64_t n,
                                 int per_query_params, double eps, double *out_loglik, double *out_grad,
                                 void *stream) {
    SSM_REQUIRE(n >= 0, "ssm_ddm_nf_loglik: n < 0");
    if (n == 0) return SSM_OK;
    SSM_REQUIRE(rt && choice && v && a && z && t && out_loglik, "ssm_ddm_nf_loglik: null pointer");
    SSM_REQUIRE(eps > 0 && eps < 1, "ssm_ddm_nf_loglik: eps must be in (0, 1)");
    const int threads = 128;
    ssm::nf::k_ddm_nf<<<(unsigned)((n + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(
        rt, choice, v, a, z, t, s, n, per_query_params ? 1 : 0, eps, out_loglik, out_grad);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}
