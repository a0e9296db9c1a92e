// Linear ballistic accumulator (cssm.lba_vanilla, src/cssm/lba_models.pyx:36-139)
// for sm_100a.  Closed form per sample: start_j ~ U(0, A), drift_j = |N(v_j, sd_j)|,
// finishing time x_j = (b - start_j) / drift_j; choice = argmin_j x_j (first
// minimum), rt = min_j x_j + t, rt = -999 when rt >= deadline.  One thread per
// sample; Philox4x32-10 words give the uniforms and (Box-Muller) normals.
#include "common.cuh"

namespace ssm {

struct LbaParams {
    PhiloxKeys key;
    const float *v, *a, *z, *sd, *t, *deadline;  // v, sd: [K, nact]; a, z (=A), t, deadline: [K]
    const int64_t *offsets;
    int64_t n_trials, total;
    int nact;
    const float *noise_u, *noise_g;  // injected U(0,1) and N(0,1) draws, [total, nact]
    float *rts;
    int32_t *choices;
};

__device__ __forceinline__ int64_t lba_find(const int64_t *off, int64_t K, int64_t w) {
    int64_t lo = 0, hi = K;  // off[lo] <= w < off[hi]
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= w) lo = mid; else hi = mid;
    }
    return lo;
}

template <bool NOISE>
__global__ void __launch_bounds__(256) k_lba(const __grid_constant__ LbaParams p) {
    const int64_t total = (p.total >= 0) ? p.total : __ldg(p.offsets + p.n_trials);
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total;
         w += (int64_t)gridDim.x * blockDim.x) {
        int64_t k, n;
        if (p.offsets == nullptr) {
            k = w % p.n_trials;
            n = w / p.n_trials;
        } else {
            k = lba_find(p.offsets, p.n_trials, w);
            n = w - __ldg(p.offsets + k);
        }
        const float bk = __ldg(p.a + k), Ak = __ldg(p.z + k);
        float best = 0.f;
        int arg = 0;
        for (int j = 0; j < p.nact; ++j) {
            float u, g;
            if (NOISE) {
                u = __ldg(p.noise_u + w * p.nact + j);
                g = __ldg(p.noise_g + w * p.nact + j);
            } else {
                // one Philox call per accumulator: words x, y -> normal, z -> uniform
                const uint4 r = philox10(make_uint4((uint32_t)j, (uint32_t)n, (uint32_t)k, 5u), p.key);
                g = box_muller(r.x, r.y).x;
                u = uniform_co(r.z);
            }
            const float zs = __fmul_rn(u, Ak);
            const float vs = fabsf(__fadd_rn(__ldg(p.v + k * p.nact + j), __fmul_rn(__ldg(p.sd + k * p.nact + j), g)));
            const float x = __fdiv_rn(__fsub_rn(bk, zs), vs);
            if (j == 0 || x < best) {
                best = x;
                arg = j;
            }
        }
        float rt = __fadd_rn(best, __ldg(p.t + k));
        if (rt >= __ldg(p.deadline + k)) rt = -999.f;
        p.rts[w] = rt;
        p.choices[w] = arg;
    }
}

}  // namespace ssm

extern "C" int ssm_lba_vanilla(const float *v, const float *a, const float *z,
                               const float *deadline, const float *sd, const float *t,
                               int64_t n_trials, int64_t n_samples, int nact,
                               const int64_t *sample_offsets, uint64_t seed, const float *noise_u,
                               const float *noise_g, float *rts, int32_t *choices, void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_trials >= 0 && n_samples >= 0, "n_trials and n_samples must be >= 0");
    SSM_REQUIRE(nact >= 1, "nact must be >= 1");
    SSM_REQUIRE(n_trials == 0 || (v && a && z && deadline && sd && t), "v, a, z, deadline, sd, t are required");
    SSM_REQUIRE(!noise_u == !noise_g, "noise_u and noise_g go together");
    SSM_REQUIRE((rts && choices) || (!sample_offsets && n_trials * n_samples == 0), "rts and choices outputs are required");
    const int64_t total = sample_offsets ? -1 : n_trials * n_samples;
    if (n_trials == 0 || total == 0) return SSM_OK;
    LbaParams p;
    p.key = philox_keys(seed);
    p.v = v; p.a = a; p.z = z; p.sd = sd; p.t = t; p.deadline = deadline;
    p.offsets = sample_offsets; p.n_trials = n_trials; p.total = total; p.nact = nact;
    p.noise_u = noise_u; p.noise_g = noise_g; p.rts = rts; p.choices = choices;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = sm_count() * 8;
    if (noise_u) k_lba<true><<<grid, 256, 0, st>>>(p);
    else k_lba<false><<<grid, 256, 0, st>>>(p);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}
