// Shared device/host helpers for the sm_100a simulators: status handling,
// the counter-based Philox4x32-10 generator and normal/uniform transforms.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ssm_b200.h"

namespace ssm {

// ---------------------------------------------------------------- host side
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *where);
int sm_count();

#define SSM_CUDA(call)                                         \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return ::ssm::cuda_fail(e_, #call); \
    } while (0)

#define SSM_REQUIRE(cond, ...)          \
    do {                                \
        if (!(cond)) {                  \
            ::ssm::set_error(__VA_ARGS__); \
            return SSM_ERR_ARG;         \
        }                               \
    } while (0)

// Trajectories a persistent simulator warp claims per queue access: the
// caller's chunk, cut (to a multiple of the warp's walk slots -- 32, or 32 / W
// with W lanes per walk -- and at least one slot per walk) so that every warp
// of the grid gets work when the launch is small.
__device__ __forceinline__ int64_t warp_chunk(int chunk, int64_t total, int slots = 32) {
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t fair = ((total + warps - 1) / warps + slots - 1) / slots * slots;
    return max((int64_t)slots, min((int64_t)chunk, fair));
}

// Ended walks a persistent simulator warp collects before it writes their
// results and restarts those lanes (ssm_launch.refill_min = 0).  Batching
// pays where a step is cheap next to the restart (single accumulator, 4:
// 10-12 % faster than 1 on the angle and full_ddm batches).  The race kernel,
// whose steps cost more, restarts two at a time by default: with windows of
// steps drawn ahead, 1 024-set launches measured 2.4 % (LCA) and 7.9 %
// (racing diffusion) faster with 2 than with 1, and the race model 8.3 %
// with 6 (its tuned value, like the others', is in the launch-option store).
#ifndef SSM_REFILL_MIN
#define SSM_REFILL_MIN 4
#endif
#ifndef SSM_REFILL_MIN_RACE
#define SSM_REFILL_MIN_RACE 2
#endif

// Workspace header shared by every persistent kernel: a work counter and an
// error word.  It sits at the start of the caller's workspace and is cleared
// by the launching entry point (cudaMemsetAsync) before each launch.
struct alignas(256) WorkspaceHeader {
    unsigned long long counter;  // next unclaimed trajectory index
    int err;                     // first error code raised on the device (0 = none)
    int err_detail;              // e.g. the trajectory that overran its noise row
    unsigned long long aux[4];
};
static_assert(sizeof(WorkspaceHeader) == 256, "header must stay 256 B");

// Philox4x32-10 round keys.  The key schedule depends only on the seed, so it
// is expanded once on the host and travels in the kernel parameter block
// (constant bank): each round's key XOR is then a free constant operand.
struct PhiloxKeys {
    uint32_t k0[10];
    uint32_t k1[10];
};

inline PhiloxKeys philox_keys(uint64_t seed) {
    PhiloxKeys k;
    uint32_t a = (uint32_t)seed, b = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        k.k0[r] = a;
        k.k1[r] = b;
        a += 0x9E3779B9u;  // Weyl increments of the Philox key schedule
        b += 0xBB67AE85u;
    }
    return k;
}

// ---------------------------------------------------------------- device side
// Philox4x32 with 10 rounds (Salmon, Moraes, Dror & Shaw, "Parallel Random
// Numbers: As Easy as 1, 2, 3", SC'11).  One call maps a 128-bit counter to
// 128 random bits; we key it by the seed and count over (step block, sample,
// trial, stream) so every trajectory owns an independent stream.
__device__ __forceinline__ uint4 philox10(uint4 c, const PhiloxKeys &key) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // one 32x32->64 multiply (IMAD.WIDE.U32) per product gives both halves
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ key.k0[r], (uint32_t)p1,
                       (uint32_t)(p0 >> 32) ^ c.w ^ key.k1[r], (uint32_t)p0);
    }
    return c;
}

// 23 random bits -> float in [1, 2) by exponent stuffing (two integer ops, no
// int->float conversion, which runs at quarter rate).
__device__ __forceinline__ float bits_to_1_2(uint32_t x) {
    return __uint_as_float(0x3f800000u | (x >> 9));
}
// Uniform on the open interval (0, 1): values j*2^-23 + 2^-24, j = 0..2^23-1.
__device__ __forceinline__ float uniform_open(uint32_t x) {
    return bits_to_1_2(x) - 0.99999994f;  // 1 - 2^-24; exact in float32
}
// Uniform on [0, 1) with 24-bit resolution (used once per trajectory).
__device__ __forceinline__ float uniform_co(uint32_t x) {
    return (float)(x >> 8) * 5.9604645e-08f;  // 2^-24
}

// SFU approximations in their flush-to-zero forms.  Every argument the
// generators pass is a normal float (uniforms are at least 2^-24, angles 0 or
// at least 2^-21), for which these give the same results as the non-ftz
// forms, without the extra instructions that rescale subnormal inputs.
__device__ __forceinline__ float lg2_ftz(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ void sincos_ftz(float x, float &s, float &c) {
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(x));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(x));
}

// Box-Muller transform of two 32-bit words into two N(0,1) variates
// (r = sqrt(-2 ln u1), phase 2 pi u2).  Uses the SFU approximations of log2,
// rsqrt, sin and cos: 4 MUFU operations per pair (u1 >= 2^-24 and the phase
// is 0 or at least 2 pi 2^-23: normal floats, so the ftz forms apply).
__device__ __forceinline__ float2 box_muller(uint32_t a, uint32_t b) {
    const float u1 = uniform_open(a);
    const float u2 = bits_to_1_2(b) - 1.0f;
    const float e = -1.3862944f * lg2_ftz(u1);  // -2 ln u1 > 0
    const float r = e * rsqrtf(e);
    float s, c;
    sincos_ftz(6.2831853f * u2, s, c);
    return make_float2(r * c, r * s);
}

// Six increments from one Philox4x32-10 call (128 bits): three Box-Muller pairs whose
// radii take 23-bit uniforms from the low bits of x, y and z, and whose phases
// take the low 23 bits of w, and 18 bits each from the top nine bits of (w, x)
// and of (y, z).  The radius resolution is that of the four-per-call layout
// (uniforms on a 2^-23 grid, so |N| <= 5.6); an 18-bit phase puts the pair on
// one of 262 144 rays, far below what a one-dimensional increment can show.
// Compared with two pairs per call this takes a third less Philox work per
// increment.  c2 = -2 ln(2) scale^2 scales the radius, so each output is
// drift + scale * N(0,1) (scale 1, drift 0: standard normals).  Pair i (outputs
// 2i, 2i+1) takes its own c2[i] and drift[i] (bm6_increment: the same for all).
__device__ __forceinline__ void bm6_increment_pairs(uint4 b, const float (&c2)[3], const float (&drift)[3],
                                                    float *g) {
    const uint32_t rad[3] = {b.x, b.y, b.z};
    const uint32_t ph[3] = {b.w & 0x007fffffu, ((b.w >> 9) & 0x7fc000u) | ((b.x >> 18) & 0x3fe0u),
                            ((b.y >> 9) & 0x7fc000u) | ((b.z >> 18) & 0x3fe0u)};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float u1 = __uint_as_float(0x3f800000u | (rad[i] & 0x007fffffu)) - 0.99999994f;  // (0, 1)
        const float ang = fmaf(__uint_as_float(0x3f800000u | ph[i]), 6.2831853f, -6.2831853f);
        const float e = c2[i] * lg2_ftz(u1);
        float r;
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e));
        float sn, cs;
        sincos_ftz(ang, sn, cs);
        g[2 * i] = fmaf(r, cs, drift[i]);
        g[2 * i + 1] = fmaf(r, sn, drift[i]);
    }
}
__device__ __forceinline__ void bm6_increment(uint4 b, float c2, float drift, float *g) {
    const float c[3] = {c2, c2, c2}, d[3] = {drift, drift, drift};
    bm6_increment_pairs(b, c, d, g);
}

__device__ __forceinline__ void raise_error(WorkspaceHeader *h, int code, int detail) {
    if (atomicCAS(&h->err, 0, code) == 0) h->err_detail = detail;
}

}  // namespace ssm
