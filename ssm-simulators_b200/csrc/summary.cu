// Per-trial choice statistics and pooled rt histograms of a simulator output
// in the reference layout (output n * n_trials + k): the derived outputs of
// simulator() (ssms/basic_simulators/simulator.py:806-863 -- choice_p,
// choice_p_no_omission, omission_p, nogo_p, go_p) and its binned_128 /
// binned_256 histograms (bin_simulator_output, simulator.py:435-497), which the
// reference computes in host loops over trials.
//
// Grid (n_trials, slices): each CTA counts one slice of one trial's samples in
// shared memory and adds its non-zero counters to the global ones, which the
// entry point clears first.  Histogram bins follow numpy.histogram: bin i holds
// edges[i] <= x < edges[i+1], the last bin also x == edges[nbins]; values
// outside [edges[0], edges[nbins]] and omissions are not counted.
#include "common.cuh"

namespace ssm {

constexpr int SUM_MAX_CHOICES = 16;
constexpr int SUM_MAX_BINS = 1024;

struct SimSummary {
    const float *rts;
    const int32_t *choices;
    int64_t n_samples, n_trials, per_slice;
    const int32_t *cvals;
    int nc;
    const double *edges_a, *edges_b;
    int nb_a, nb_b;
    unsigned long long *choice_counts, *kept_counts, *omit_counts, *nogo_counts, *hist_a, *hist_b;
};

__device__ __forceinline__ int edge_bin(const double *edges, int nb, double x) {
    if (!(x >= edges[0]) || !(x <= edges[nb])) return -1;
    if (x == edges[nb]) return nb - 1;
    int lo = 0, hi = nb;  // edges[lo] <= x < edges[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (edges[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_sim_summary(const SimSummary a) {
    extern __shared__ unsigned int hs[];  // [nc * (nb_a + nb_b)]
    __shared__ unsigned int cc[SUM_MAX_CHOICES], kc[SUM_MAX_CHOICES], om, ng;
    const int64_t k = blockIdx.x;
    const int H = a.nc * (a.nb_a + a.nb_b);
    // the largest choice value is the "go" response (simulator.py:846-853)
    int32_t max_choice = __ldg(a.cvals);
    for (int j = 1; j < a.nc; ++j) max_choice = max(max_choice, __ldg(a.cvals + j));
    for (int i = threadIdx.x; i < H; i += blockDim.x) hs[i] = 0u;
    if (threadIdx.x < SUM_MAX_CHOICES) cc[threadIdx.x] = kc[threadIdx.x] = 0u;
    if (threadIdx.x == 0) om = ng = 0u;
    __syncthreads();
    const int64_t n0 = (int64_t)blockIdx.y * a.per_slice;
    const int64_t n1 = min(n0 + a.per_slice, a.n_samples);
    for (int64_t n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
        const int64_t i = n * a.n_trials + k;
        const float rt = a.rts[i];
        const int32_t ch = a.choices[i];
        const bool omitted = (rt == -999.f);
        if (omitted) atomicAdd(&om, 1u);
        if (ch != max_choice || omitted) atomicAdd(&ng, 1u);
        int c = -1;
        for (int j = 0; j < a.nc; ++j)
            if (__ldg(a.cvals + j) == ch) c = j;
        if (c < 0) continue;
        atomicAdd(&cc[c], 1u);
        if (omitted) continue;
        atomicAdd(&kc[c], 1u);
        const int ia = edge_bin(a.edges_a, a.nb_a, (double)rt);
        if (ia >= 0) atomicAdd(&hs[c * a.nb_a + ia], 1u);
        const int ib = edge_bin(a.edges_b, a.nb_b, (double)rt);
        if (ib >= 0) atomicAdd(&hs[a.nc * a.nb_a + c * a.nb_b + ib], 1u);
    }
    __syncthreads();
    if (threadIdx.x < a.nc) {
        if (cc[threadIdx.x]) atomicAdd(a.choice_counts + k * a.nc + threadIdx.x, (unsigned long long)cc[threadIdx.x]);
        if (kc[threadIdx.x]) atomicAdd(a.kept_counts + k * a.nc + threadIdx.x, (unsigned long long)kc[threadIdx.x]);
    }
    if (threadIdx.x == 0) {
        if (om) atomicAdd(a.omit_counts + k, (unsigned long long)om);
        if (ng) atomicAdd(a.nogo_counts + k, (unsigned long long)ng);
    }
    // pooled histograms, laid out [bin, choice] like the reference's arrays
    for (int i = threadIdx.x; i < a.nc * a.nb_a; i += blockDim.x) {
        if (hs[i]) {
            const int c = i / a.nb_a, b = i % a.nb_a;
            atomicAdd(a.hist_a + (int64_t)b * a.nc + c, (unsigned long long)hs[i]);
        }
    }
    for (int i = threadIdx.x; i < a.nc * a.nb_b; i += blockDim.x) {
        const unsigned int v = hs[a.nc * a.nb_a + i];
        if (v) {
            const int c = i / a.nb_b, b = i % a.nb_b;
            atomicAdd(a.hist_b + (int64_t)b * a.nc + c, (unsigned long long)v);
        }
    }
}

}  // namespace ssm

extern "C" {

int ssm_simulator_summary(const float *rts, const int32_t *choices, int64_t n_samples, int64_t n_trials,
                          const int32_t *choice_values, int n_choices, const double *edges_a, int nbins_a,
                          const double *edges_b, int nbins_b, int64_t *choice_counts, int64_t *kept_counts,
                          int64_t *omission_counts, int64_t *nogo_counts, int64_t *hist_a, int64_t *hist_b,
                          void *stream) {
    using namespace ssm;
    SSM_REQUIRE(n_samples >= 0 && n_trials >= 0, "n_samples and n_trials must be >= 0");
    SSM_REQUIRE(n_choices >= 1 && n_choices <= SUM_MAX_CHOICES, "n_choices must be in [1, %d]", SUM_MAX_CHOICES);
    SSM_REQUIRE(nbins_a >= 1 && nbins_b >= 1 && nbins_a + nbins_b <= SUM_MAX_BINS, "bad bin counts");
    SSM_REQUIRE(choice_values && edges_a && edges_b && choice_counts && kept_counts && omission_counts &&
                nogo_counts && hist_a && hist_b, "all buffers are required");
    cudaStream_t st = (cudaStream_t)stream;
    SSM_CUDA(cudaMemsetAsync(choice_counts, 0, sizeof(int64_t) * n_trials * n_choices, st));
    SSM_CUDA(cudaMemsetAsync(kept_counts, 0, sizeof(int64_t) * n_trials * n_choices, st));
    SSM_CUDA(cudaMemsetAsync(omission_counts, 0, sizeof(int64_t) * n_trials, st));
    SSM_CUDA(cudaMemsetAsync(nogo_counts, 0, sizeof(int64_t) * n_trials, st));
    SSM_CUDA(cudaMemsetAsync(hist_a, 0, sizeof(int64_t) * nbins_a * n_choices, st));
    SSM_CUDA(cudaMemsetAsync(hist_b, 0, sizeof(int64_t) * nbins_b * n_choices, st));
    if (n_samples == 0 || n_trials == 0) return SSM_OK;
    SSM_REQUIRE(rts && choices, "rts and choices are required");
    SSM_REQUIRE(n_trials < (1ll << 31), "too many trials for one launch");
    const size_t smem = sizeof(unsigned int) * n_choices * (nbins_a + nbins_b);
    SSM_REQUIRE(smem <= 48 * 1024, "histograms must fit in 48 KB of shared memory");
    SimSummary a;
    a.rts = rts; a.choices = choices; a.n_samples = n_samples; a.n_trials = n_trials;
    a.cvals = choice_values; a.nc = n_choices;
    a.edges_a = edges_a; a.edges_b = edges_b; a.nb_a = nbins_a; a.nb_b = nbins_b;
    a.choice_counts = reinterpret_cast<unsigned long long *>(choice_counts);
    a.kept_counts = reinterpret_cast<unsigned long long *>(kept_counts);
    a.omit_counts = reinterpret_cast<unsigned long long *>(omission_counts);
    a.nogo_counts = reinterpret_cast<unsigned long long *>(nogo_counts);
    a.hist_a = reinterpret_cast<unsigned long long *>(hist_a);
    a.hist_b = reinterpret_cast<unsigned long long *>(hist_b);
    // slices of >= 4096 samples, enough CTAs to fill the GPU
    const int64_t want = (int64_t)sm_count() * 8;
    int64_t slices = (want + n_trials - 1) / n_trials;
    const int64_t max_slices = (n_samples + 4095) / 4096;
    if (slices > max_slices) slices = max_slices;
    if (slices < 1) slices = 1;
    if (slices > 65535) slices = 65535;
    a.per_slice = (n_samples + slices - 1) / slices;
    dim3 grid((unsigned)n_trials, (unsigned)slices);
    k_sim_summary<<<grid, 256, smem, st>>>(a);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

}  // extern "C"
