// Likelihood-surrogate MLP 7 -> 100 -> 100 -> 120 -> 1 (tanh hidden layers) on
// the sm_100a tensor cores: forward, forward + d(out)/d(input), and the
// training gradient, each one persistent kernel that keeps the bf16 weight
// image resident in shared memory and runs its three hidden-layer GEMMs as
// tcgen05.mma (bf16 x bf16 -> fp32 in TMEM).  The reference has no network of
// its own: it only emits the (theta, rt, choice, log-lik) training records
// (ssms/dataset_generators/lan_mlp.py); this file is the learned part built on
// those records.
//
// Shapes (rows of a tile = batch rows, M = 128 per warpgroup):
//   layer 1  [128 x 16 ] x W1^T [16 x 112]   -> acc 112 cols   (7 inputs split hi/lo)
//   layer 2  [128 x 112] x W2^T [112 x 112]  -> acc 112 cols
//   layer 3  [128 x 112] x W3^T [112 x 128]  -> acc 128 cols
//   output   h3 . w4 + b4 on the FP32 pipe (120 terms, fp32 weights)
// Inputs are normalised x~ = (x - c) * s and split x~ = hi + lo into two bf16
// columns each, so the first layer sees ~16 significant bits of rt.  The
// hidden layers' biases ride in the GEMMs the same way: every layer input
// carries two ones columns (14 and 15 of the input tile, 100 and 101 of the
// hidden tiles) against weight columns holding bf16(b) and bf16(b - bf16(b)),
// so the fp32 accumulator starts from b to ~16 bits and the epilogues, whose
// shared-memory and SFU queue is the forward pass's bottleneck, add nothing.
//
// Shared-memory operand layout ("chunk-major", no swizzle): an R x C bf16 tile
// stores element (r, c) at byte (c / 8) * (R * 16) + r * 16 + (c % 8) * 2, i.e.
// each 8-column chunk is a contiguous stack of 16-byte row pieces and every
// 8 x 8 core matrix is 128 contiguous bytes.  The same bytes serve as a
// K-major operand (rows = M/N, cols = K) and, transposed, as an MN-major
// operand (rows = K, cols = M/N); backward and weight-gradient GEMMs use the
// transposed views instead of copying.
//
// Synchronisation: per warpgroup one mbarrier tracks its MMAs (tcgen05.commit),
// epilogue stores are published to the async proxy with
// fence.proxy.async.shared::cta + a named barrier, and TMEM reads are ordered
// against the next MMA by tcgen05.fence::before/after_thread_sync.  Every
// mbarrier wait is bounded (about one second); on expiry the kernel records
// SSM_MLP_ERR_TIMEOUT, leaves its tile loop and frees its TMEM.
#include <cuda_bf16.h>

#include "common.cuh"

namespace ssm {
namespace mlp {

constexpr int DIN = 7, H1 = 100, H2 = 100, H3 = 120;
constexpr int K0 = 16, N1 = 112, N2 = 112, N3 = 128;
constexpr int ONES1 = 100, ONES3 = 120, ONES0 = 14;  // ones columns (bias terms and bias gradients)

// bf16 weight image (device global and shared memory), byte offsets
constexpr int OFF_W1 = 0;                       // 112 rows x 16 cols
constexpr int OFF_W2 = OFF_W1 + N1 * K0 * 2;    // 112 x 112
constexpr int OFF_W3 = OFF_W2 + N2 * N1 * 2;    // 128 x 112
constexpr int OFF_B1 = OFF_W3 + N3 * N2 * 2;    // fp32 [112] (the biases in fp32; the kernels use the
                                                // bf16 hi/lo columns of W1-W3)
constexpr int OFF_B2 = OFF_B1 + N1 * 4;         // fp32 [112]
constexpr int OFF_B3 = OFF_B2 + N2 * 4;         // fp32 [128]
constexpr int OFF_W4 = OFF_B3 + N3 * 4;         // fp32 [128]
constexpr int OFF_B4 = OFF_W4 + N3 * 4;         // fp32 [4]
constexpr int IMAGE_BYTES = OFF_B4 + 16;
static_assert(IMAGE_BYTES == SSM_MLP_IMAGE_BYTES, "image size mismatch with the header");
static_assert(OFF_W2 % 16 == 0 && OFF_W3 % 16 == 0 && OFF_B1 % 16 == 0 && IMAGE_BYTES % 16 == 0, "align");

// master parameter vector (fp32, torch nn.Linear order: weight [out, in] then bias)
constexpr int P_W1 = 0, P_B1 = P_W1 + H1 * DIN, P_W2 = P_B1 + H1, P_B2 = P_W2 + H2 * H1,
              P_W3 = P_B2 + H2, P_B3 = P_W3 + H3 * H2, P_W4 = P_B3 + H3, P_B4 = P_W4 + H3,
              NPARAMS = P_B4 + 1;
static_assert(NPARAMS == SSM_MLP_NPARAMS, "parameter count mismatch with the header");
constexpr int PSTRIDE = SSM_MLP_PARTIAL_STRIDE;  // floats per per-CTA gradient partial

// shared memory map
constexpr int SM_BAR = 59392;                   // mbarriers (8 x 8 B) + TMEM slot
constexpr int SM_WG = SM_BAR + 128;             // per-warpgroup operand buffers
static_assert(SM_BAR >= IMAGE_BYTES, "image overlaps barriers");
constexpr int TILE_X = 128 * K0 * 2;            // 4096
constexpr int TILE_H = 128 * N1 * 2;            // 28672 (112 cols)
constexpr int TILE_G = 128 * 128 * 2;           // 32768 (128 cols)
constexpr int CHUNK = 128 * 16;                 // bytes per 8-column chunk of a 128-row tile

enum Mode { FWD = 0, FWD_DX = 1, TRAIN = 2 };
template <int MODE> struct Cfg;
template <> struct Cfg<FWD> {
    static constexpr int NWG = 4;
    static constexpr int WG_BYTES = TILE_X + TILE_H;                   // X, B0
};
template <> struct Cfg<FWD_DX> {
    static constexpr int NWG = 2;
    static constexpr int WG_BYTES = TILE_X + TILE_G + TILE_H;          // X, B0, B1
};
template <> struct Cfg<TRAIN> {
    static constexpr int NWG = 1;
    static constexpr int WG_BYTES = TILE_X + 2 * TILE_H + 2 * TILE_G + TILE_X;  // X H1 H2 H3 G GO
};
template <int MODE> constexpr int smem_bytes() { return SM_WG + Cfg<MODE>::NWG * Cfg<MODE>::WG_BYTES; }
static_assert(smem_bytes<FWD>() <= 232448 && smem_bytes<FWD_DX>() <= 232448 &&
              smem_bytes<TRAIN>() <= 232448, "shared memory budget");

// TMEM columns (512 allocated; one CTA per SM is forced by the shared memory size)
constexpr uint32_t T_DW2 = 128, T_DW3 = 256, T_DW1 = 384, T_DW4 = 416;

struct Norm {
    float c[8];
    float s[8];
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// true when the phase with the given parity has completed; gives up after ~1 s
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    uint32_t done = 0;
    uint64_t t0 = 0;
    for (uint32_t it = 0;; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255u) == 0) {
            const uint64_t now = globaltimer();
            if (it == 0) t0 = now;
            else if (now - t0 > 1000000000ull) return false;
        }
    }
}

__device__ __forceinline__ void bar_sync(int id, int n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// named barrier that also ORs a predicate over the participating threads
__device__ __forceinline__ int bar_or(int id, int n, int pred) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(pred), "r"(id), "r"(n)
        : "memory");
    return r;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle: start, leading-dimension byte
// offset (between K-adjacent core matrices), stride byte offset (between
// M/N-adjacent core matrices), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor for kind::f16 with bf16 A/B and fp32 D.
__host__ __device__ constexpr uint32_t idesc(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t dt, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(dt), "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// One chain of K-steps into TMEM column dt.  a/b: start address, LBO, SBO and
// the byte advance per K-step of 16.
struct Op {
    uint32_t base, lbo, sbo, step;
};
__device__ __forceinline__ void mma_chain(uint32_t dt, Op a, Op b, int ksteps, uint32_t id, bool acc0) {
    for (int k = 0; k < ksteps; ++k)
        umma(dt, sdesc(a.base + k * a.step, a.lbo, a.sbo), sdesc(b.base + k * b.step, b.lbo, b.sbo), id,
             (k > 0 || acc0) ? 1u : 0u);
}
// operand views of a chunk-major tile with R rows
__device__ __forceinline__ Op kmajor(uint32_t base, int R) { return {base, (uint32_t)R * 16u, 128u, (uint32_t)R * 32u}; }
__device__ __forceinline__ Op mnmajor(uint32_t base, int R) { return {base, 128u, (uint32_t)R * 16u, 256u}; }

// 16 consecutive fp32 TMEM columns of this thread's lane; the wait is in the
// same statement so the registers are valid when it returns.
__device__ __forceinline__ void tmem_ld16(uint32_t ta, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta)
        : "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t ta, uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(ta)
        : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t ta, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(ta), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

constexpr uint32_t BF16_ONE = 0x3F80u;

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ float2 unpack2(uint32_t u) {
    return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162 *>(&u));
}

__device__ __forceinline__ void st_row(uint8_t *tile, int chunk, int r, uint4 v) {
    *reinterpret_cast<uint4 *>(tile + chunk * CHUNK + r * 16) = v;
}
__device__ __forceinline__ uint4 ld_row(const uint8_t *tile, int chunk, int r) {
    return *reinterpret_cast<const uint4 *>(tile + chunk * CHUNK + r * 16);
}

// ------------------------------------------------------------ epilogue pieces
// x row -> normalised, split hi/lo -> X tile (cols 0-6 hi, 7-13 lo, 14 = 15 = 1).
__device__ __forceinline__ void stage_x(uint8_t *X, int r, const float *xr, bool valid, const Norm &nm) {
    float hi[7], lo[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        const float v = valid ? (xr[j] - nm.c[j]) * nm.s[j] : 0.f;
        hi[j] = __bfloat162float(__float2bfloat16_rn(v));
        lo[j] = v - hi[j];
    }
    uint4 c0 = {pack2(hi[0], hi[1]), pack2(hi[2], hi[3]), pack2(hi[4], hi[5]), pack2(hi[6], lo[0])};
    uint4 c1 = {pack2(lo[1], lo[2]), pack2(lo[3], lo[4]), pack2(lo[5], lo[6]), pack2(1.f, 1.f)};
    st_row(X, 0, r, c0);
    st_row(X, 1, r, c1);
}

// Hidden layers 1 and 2: tanh(acc) in fp32 (tanh.approx.f32; the bias is in
// acc already), rounded to bf16 pairs -> bf16 tile.  Columns from H (the real
// width) on are padding: written as zeros without a tanh, except the two ones
// columns.  Optionally the packed pairs are also stashed in TMEM at ts.
// (tanh.approx.bf16x2 was measured: it costs the XU pipe as much as two fp32
// tanh, so it buys nothing.)
template <bool EDGE, int H, int ONES, bool STASH>
__device__ __forceinline__ void hidden_chunk(int c, uint32_t ta, uint8_t *dst, int r, uint32_t ts) {
    float v[16];
    tmem_ld16(ta + 16 * c, v);
    uint32_t p[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int col = 16 * c + 4 * q;
        if (EDGE && col >= H) {
            p[2 * q] = p[2 * q + 1] = 0u;
        } else {
            p[2 * q] = pack2(tanh_fast(v[4 * q]), tanh_fast(v[4 * q + 1]));
            p[2 * q + 1] = pack2(tanh_fast(v[4 * q + 2]), tanh_fast(v[4 * q + 3]));
        }
        if (EDGE) {
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (col + e == ONES || col + e == ONES + 1) {
                    uint32_t &w = p[2 * q + e / 2];
                    w = (e & 1) ? ((w & 0x0000FFFFu) | (BF16_ONE << 16)) : ((w & 0xFFFF0000u) | BF16_ONE);
                }
        }
    }
    st_row(dst, 2 * c, r, make_uint4(p[0], p[1], p[2], p[3]));
    st_row(dst, 2 * c + 1, r, make_uint4(p[4], p[5], p[6], p[7]));
    if (STASH) tmem_st8(ts + 8 * c, p);
}

template <int NC, int H, int ONES, bool STASH>
__device__ __forceinline__ void epi_hidden(uint32_t ta, uint8_t *dst, int r, uint32_t ts) {
    static_assert(H > NC - 16 && ONES >= NC - 16 && ONES + 1 < NC, "padding and ones columns lie in the last chunk");
#pragma unroll 1
    for (int c = 0; c < NC / 16 - 1; ++c) hidden_chunk<false, H, ONES, STASH>(c, ta, dst, r, ts);
    hidden_chunk<true, H, ONES, STASH>(NC / 16 - 1, ta, dst, r, ts);
}

// G = D (TMEM, NC cols) * (1 - h^2) with h read from this row of H; G -> dst
// (which may alias H); columns [NC, NCPAD) of dst are zeroed.
template <int NC, int NCPAD>
__device__ __forceinline__ void epi_dtanh(uint32_t ta, const uint8_t *H, uint8_t *dst, int r) {
#pragma unroll 1
    for (int c = 0; c < NC / 16; ++c) {
        float v[16];
        tmem_ld16(ta + 16 * c, v);
        const uint4 h0 = ld_row(H, 2 * c, r), h1 = ld_row(H, 2 * c + 1, r);
        const uint32_t hh[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
        uint32_t p[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float2 h = unpack2(hh[j]);
            p[j] = pack2(v[2 * j] * (1.f - h.x * h.x), v[2 * j + 1] * (1.f - h.y * h.y));
        }
        st_row(dst, 2 * c, r, make_uint4(p[0], p[1], p[2], p[3]));
        st_row(dst, 2 * c + 1, r, make_uint4(p[4], p[5], p[6], p[7]));
    }
#pragma unroll
    for (int c = NC / 8; c < NCPAD / 8; ++c) st_row(dst, c, r, make_uint4(0, 0, 0, 0));
}

// same, with h taken from the packed bf16 stash in TMEM
__device__ __forceinline__ void epi_dtanh_stash(uint32_t ta, uint32_t ts, uint8_t *dst, int r) {
#pragma unroll 1
    for (int c = 0; c < N1 / 16; ++c) {
        float v[16];
        tmem_ld16(ta + 16 * c, v);
        uint32_t hh[8];
        tmem_ld8(ts + 8 * c, hh);
        uint32_t p[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float2 h = unpack2(hh[j]);
            p[j] = pack2(v[2 * j] * (1.f - h.x * h.x), v[2 * j + 1] * (1.f - h.y * h.y));
        }
        st_row(dst, 2 * c, r, make_uint4(p[0], p[1], p[2], p[3]));
        st_row(dst, 2 * c + 1, r, make_uint4(p[4], p[5], p[6], p[7]));
    }
}

// Layer-3 epilogue: h3 = tanh(acc) in fp32 (b3 is in acc), out = b4 + h3 . w4 (fp32),
// and per KIND: 0 nothing else, 1 G3 = w4 (1 - h3^2) -> dst (d out / d acc3),
// 2 bf16 h3 with the ones column -> dst (training operand).
template <int KIND, bool EDGE>
__device__ __forceinline__ void out_chunk(int c, uint32_t ta, const float4 *w4v, float &o, uint8_t *dst, int r) {
    float v[16];
    tmem_ld16(ta + 16 * c, v);
    uint32_t p[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int col = 16 * c + 4 * q;
        float h[4] = {0.f, 0.f, 0.f, 0.f}, w[4] = {0.f, 0.f, 0.f, 0.f};
        if (!EDGE || col < H3) {
            const float4 ww = w4v[col / 4];
            h[0] = tanh_fast(v[4 * q]);
            h[1] = tanh_fast(v[4 * q + 1]);
            h[2] = tanh_fast(v[4 * q + 2]);
            h[3] = tanh_fast(v[4 * q + 3]);
            w[0] = ww.x; w[1] = ww.y; w[2] = ww.z; w[3] = ww.w;
#pragma unroll
            for (int e = 0; e < 4; ++e) o = fmaf(w[e], h[e], o);
        }
        if (KIND == 1) {
            p[2 * q] = pack2(w[0] * (1.f - h[0] * h[0]), w[1] * (1.f - h[1] * h[1]));
            p[2 * q + 1] = pack2(w[2] * (1.f - h[2] * h[2]), w[3] * (1.f - h[3] * h[3]));
        }
        if (KIND == 2) {
            if (EDGE && col == ONES3) h[0] = 1.f;
            p[2 * q] = pack2(h[0], h[1]);
            p[2 * q + 1] = pack2(h[2], h[3]);
        }
    }
    if (KIND != 0) {
        st_row(dst, 2 * c, r, make_uint4(p[0], p[1], p[2], p[3]));
        st_row(dst, 2 * c + 1, r, make_uint4(p[4], p[5], p[6], p[7]));
    }
}

template <int KIND>
__device__ __forceinline__ float epi_out(uint32_t ta, const float *w4, float b4, uint8_t *dst, int r) {
    static_assert(H3 > N3 - 16 && ONES3 >= N3 - 16, "padding and ones column lie in the last chunk");
    const float4 *w4v = reinterpret_cast<const float4 *>(w4);
    float o = b4;
#pragma unroll 1
    for (int c = 0; c < N3 / 16 - 1; ++c) out_chunk<KIND, false>(c, ta, w4v, o, dst, r);
    out_chunk<KIND, true>(N3 / 16 - 1, ta, w4v, o, dst, r);
    return o;
}

__device__ __forceinline__ void flag_error(int *status, int code) {
    if (status) atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------- the kernel
template <int MODE>
__global__ void __launch_bounds__(128 * Cfg<MODE>::NWG, 1)
k_mlp(const uint8_t *__restrict__ image, const float *__restrict__ x, int64_t n, int x_stride, Norm nm,
      float *__restrict__ out, float *__restrict__ dx, int dx_stride, int loss_kind, float inv_batch,
      float *__restrict__ part, float *__restrict__ part_loss, int *__restrict__ status) {
    constexpr int NWG = Cfg<MODE>::NWG;
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, wg = tid >> 7, r = tid & 127, warp = tid >> 5;
    const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t s0 = su32(sm);
    const uint32_t wbar = s0 + SM_BAR, mbar = s0 + SM_BAR + 8 * (1 + wg);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + SM_BAR + 64);
    const float *w4 = reinterpret_cast<const float *>(sm + OFF_W4);

    if (tid == 0) {
        mbar_init(wbar, 1);
        for (int w = 0; w < NWG; ++w) mbar_init(s0 + SM_BAR + 8 * (1 + w), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(su32(tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tbase = *tslot;

    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(wbar), "r"(IMAGE_BYTES)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(s0),
            "l"(image), "r"(IMAGE_BYTES), "r"(wbar)
            : "memory");
    }
    int bad = !mbar_wait(wbar, 0);
    bad = __syncthreads_or(bad);
    const float bias4 = *reinterpret_cast<const float *>(sm + OFF_B4);

    uint8_t *wbuf = sm + SM_WG + wg * Cfg<MODE>::WG_BYTES;
    const uint32_t sw = su32(wbuf);
    const uint32_t w1s = s0 + OFF_W1, w2s = s0 + OFF_W2, w3s = s0 + OFF_W3;
    const int bid = 1 + wg;
    uint32_t phase = 0;
    float loss_acc = 0.f;
    bool any_tile = false;

    constexpr uint32_t ID_L12 = idesc(128, 112, 0, 0), ID_L3 = idesc(128, 128, 0, 0);
    constexpr uint32_t ID_B112 = idesc(128, 112, 0, 1), ID_B16 = idesc(128, 16, 0, 1);
    constexpr uint32_t ID_W112 = idesc(128, 112, 1, 1), ID_W16 = idesc(128, 16, 1, 1);

    const int64_t n_tiles = (n + 127) / 128;
    if (!bad) {
        const uint32_t twork = tbase + (MODE == FWD_DX ? 256u * wg : 128u * wg);
        const uint32_t tw = twork + lane;  // this warp's lanes of the work columns
        for (int64_t tile = (int64_t)blockIdx.x * NWG + wg; tile < n_tiles; tile += (int64_t)gridDim.x * NWG) {
            const int64_t row = tile * 128 + r;
            const bool valid = row < n;
            const float *xr = x + (valid ? row : 0) * (int64_t)x_stride;
            uint8_t *X = wbuf;
            const uint32_t Xs = sw;
            int late = 0;
            stage_x(X, r, xr, valid, nm);
            fence_async_smem();
            bar_sync(bid, 128);

            if (MODE != TRAIN) {
                // ---------------- inference: forward (and d out / d x)
                uint8_t *B0 = wbuf + TILE_X;
                const uint32_t B0s = sw + TILE_X;
                uint8_t *B1 = wbuf + TILE_X + TILE_G;
                const uint32_t B1s = sw + TILE_X + TILE_G;
                uint8_t *Hb = (MODE == FWD) ? B0 : B1;   // h2 buffer
                const uint32_t Hbs = (MODE == FWD) ? B0s : B1s;
                const uint32_t tstash = twork + 128u + lane;

                if (r == 0) {
                    tc_after();
                    mma_chain(twork, kmajor(Xs, 128), kmajor(w1s, N1), 1, ID_L12, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                epi_hidden<N1, H1, ONES1, MODE == FWD_DX>(tw, B0, r, tstash);
                if (MODE == FWD_DX) tmem_wait_st();
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    mma_chain(twork, kmajor(B0s, 128), kmajor(w2s, N1), N1 / 16, ID_L12, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                epi_hidden<N2, H2, ONES1, false>(tw, Hb, r, 0);
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    mma_chain(twork, kmajor(Hbs, 128), kmajor(w3s, N3), N2 / 16, ID_L3, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                // layer 3 epilogue: h3, output, and (FWD_DX) G3 = w4 (1 - h3^2) -> B0
                const float o = epi_out<MODE == FWD_DX ? 1 : 0>(tw, w4, bias4, B0, r);
                if (valid) out[row] = o;
                tc_before();
                if (MODE == FWD_DX) {
                    fence_async_smem();
                    bar_sync(bid, 128);
                    // D2 = G3 W3 (K = 128 over layer-3 units)
                    if (r == 0) {
                        tc_after();
                        mma_chain(twork, kmajor(B0s, 128), mnmajor(w3s, N3), N3 / 16, ID_B112, false);
                        umma_commit(mbar);
                    }
                    late |= !mbar_wait(mbar, phase); phase ^= 1;
                    tc_after();
                    epi_dtanh<N2, N2>(tw, B1, B1, r);   // G2 over h2, in place
                    tc_before();
                    fence_async_smem();
                    bar_sync(bid, 128);
                    // D1 = G2 W2 (K = 112)
                    if (r == 0) {
                        tc_after();
                        mma_chain(twork, kmajor(B1s, 128), mnmajor(w2s, N2), N2 / 16, ID_B112, false);
                        umma_commit(mbar);
                    }
                    late |= !mbar_wait(mbar, phase); phase ^= 1;
                    tc_after();
                    epi_dtanh_stash(tw, tstash, B0, r);  // G1 over h1 (stash) -> B0
                    tc_before();
                    fence_async_smem();
                    bar_sync(bid, 128);
                    // D0 = G1 W1 (K = 112, N = 16)
                    if (r == 0) {
                        tc_after();
                        mma_chain(twork, kmajor(B0s, 128), mnmajor(w1s, N1), N1 / 16, ID_B16, false);
                        umma_commit(mbar);
                    }
                    late |= !mbar_wait(mbar, phase); phase ^= 1;
                    tc_after();
                    float v[16];
                    tmem_ld16(tw, v);
                    if (valid) {
                        float *d = dx + row * (int64_t)dx_stride;
#pragma unroll
                        for (int j = 0; j < DIN; ++j) d[j] = v[j] * nm.s[j];
                    }
                    tc_before();
                }
            } else {
                // ---------------- training: forward, loss gradient, backward, dW
                uint8_t *H1t = wbuf + TILE_X, *H2t = H1t + TILE_H, *H3t = H2t + TILE_H;
                uint8_t *Gt = H3t + TILE_G, *GOt = Gt + TILE_G;
                const uint32_t H1s = su32(H1t), H2s = su32(H2t), H3s = su32(H3t), Gs = su32(Gt), GOs = su32(GOt);
                const bool acc_dw = any_tile;
                any_tile = true;

                if (r == 0) {
                    tc_after();
                    mma_chain(twork, kmajor(Xs, 128), kmajor(w1s, N1), 1, ID_L12, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                epi_hidden<N1, H1, ONES1, false>(tw, H1t, r, 0);
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    mma_chain(twork, kmajor(H1s, 128), kmajor(w2s, N1), N1 / 16, ID_L12, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                epi_hidden<N2, H2, ONES1, false>(tw, H2t, r, 0);
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    mma_chain(twork, kmajor(H2s, 128), kmajor(w3s, N3), N2 / 16, ID_L3, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                const float o = epi_out<2>(tw, w4, bias4, H3t, r);
                const float y = valid ? xr[DIN] : 0.f;
                const float e = o - y;
                float g, l;
                if (loss_kind == 0) {  // Huber, delta 1
                    const float ae = fabsf(e);
                    l = ae <= 1.f ? 0.5f * e * e : ae - 0.5f;
                    g = fminf(fmaxf(e, -1.f), 1.f);
                } else {               // squared error
                    l = e * e;
                    g = 2.f * e;
                }
                if (!valid) { l = 0.f; g = 0.f; }
                loss_acc += l;
                g *= inv_batch;
                if (valid && out) out[row] = o;
                // G3 = g w4 (1 - h3^2) -> G ; Gout = (g, 0, ...) -> GO
#pragma unroll 1
                for (int c = 0; c < N3 / 8; ++c) {
                    const uint4 h = ld_row(H3t, c, r);
                    const uint32_t hh[4] = {h.x, h.y, h.z, h.w};
                    uint32_t p[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 f = unpack2(hh[j]);
                        const int col = 8 * c + 2 * j;
                        p[j] = pack2(g * w4[col] * (1.f - f.x * f.x), g * w4[col + 1] * (1.f - f.y * f.y));
                    }
                    st_row(Gt, c, r, make_uint4(p[0], p[1], p[2], p[3]));
                }
                st_row(GOt, 0, r, make_uint4(pack2(g, 0.f), 0, 0, 0));
                st_row(GOt, 1, r, make_uint4(0, 0, 0, 0));
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    // dW4 += H3^T Gout, dW3 += G3^T H2 (K = 128 rows), D2 = G3 W3
                    mma_chain(tbase + T_DW4, mnmajor(H3s, 128), mnmajor(GOs, 128), 8, ID_W16, acc_dw);
                    mma_chain(tbase + T_DW3, mnmajor(Gs, 128), mnmajor(H2s, 128), 8, ID_W112, acc_dw);
                    mma_chain(twork, kmajor(Gs, 128), mnmajor(w3s, N3), N3 / 16, ID_B112, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                epi_dtanh<N2, 128>(tw, H2t, Gt, r);   // G2 -> G (cols 112..127 zero)
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    mma_chain(tbase + T_DW2, mnmajor(Gs, 128), mnmajor(H1s, 128), 8, ID_W112, acc_dw);
                    mma_chain(twork, kmajor(Gs, 128), mnmajor(w2s, N2), N2 / 16, ID_B112, false);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
                epi_dtanh<N1, 128>(tw, H1t, Gt, r);   // G1 -> G
                tc_before();
                fence_async_smem();
                bar_sync(bid, 128);

                if (r == 0) {
                    tc_after();
                    mma_chain(tbase + T_DW1, mnmajor(Gs, 128), mnmajor(Xs, 128), 8, ID_W16, acc_dw);
                    umma_commit(mbar);
                }
                late |= !mbar_wait(mbar, phase); phase ^= 1;
                tc_after();
            }
            // every thread of the warpgroup leaves together if any wait expired
            if (bar_or(bid, 128, late)) {
                bad = 1;
                break;
            }
        }
    }
    if (bad) flag_error(status, SSM_MLP_ERR_TIMEOUT);

    if (MODE == TRAIN && !bad) {
        // per-CTA gradient partials out of TMEM; thread r owns output unit r
        float *pp = part + (int64_t)blockIdx.x * PSTRIDE;
        const uint32_t tl = tbase + lane;
        const bool have = any_tile;
#pragma unroll 1
        for (int c = 0; c < N2 / 16; ++c) {
            float v[16];
            tmem_ld16(tl + T_DW2 + 16 * c, v);
            if (r < H2) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int i = 16 * c + j;
                    if (i < H1) pp[P_W2 + r * H1 + i] = have ? v[j] : 0.f;
                    else if (i == ONES1) pp[P_B2 + r] = have ? v[j] : 0.f;
                }
            }
            tmem_ld16(tl + T_DW3 + 16 * c, v);
            if (r < H3) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int i = 16 * c + j;
                    if (i < H2) pp[P_W3 + r * H2 + i] = have ? v[j] : 0.f;
                    else if (i == ONES1) pp[P_B3 + r] = have ? v[j] : 0.f;
                }
            }
        }
        {
            float v[16];
            tmem_ld16(tl + T_DW1, v);
            if (r < H1) {
#pragma unroll
                for (int j = 0; j < DIN; ++j) pp[P_W1 + r * DIN + j] = have ? v[j] + v[j + DIN] : 0.f;  // hi + lo
                pp[P_B1 + r] = have ? v[ONES0] : 0.f;
            }
            tmem_ld16(tl + T_DW4, v);
            if (r < H3) pp[P_W4 + r] = have ? v[0] : 0.f;
            if (r == ONES3) pp[P_B4] = have ? v[0] : 0.f;
        }
        // CTA loss sum (one warpgroup): warp shuffle, then four warp sums
        float s = loss_acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        float *red = reinterpret_cast<float *>(sm + SM_BAR + 96);
        if ((tid & 31) == 0) red[warp] = s;
        bar_sync(1, 128);
        if (tid == 0) part_loss[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
    }

    tc_before();
    __syncthreads();
    tc_after();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase) : "memory");
    }
}

// ------------------------------------------------------------ image packing
__device__ __forceinline__ int img_index(int R, int row, int col) {  // bf16 element index in a tile
    return (col >> 3) * (R * 8) + row * 8 + (col & 7);
}

// bias b as the bf16 pair (hi, lo) of its two weight columns: hi + lo = b to ~16 bits
__device__ __forceinline__ float bias_part(float b, bool lo) {
    const float hi = __bfloat162float(__float2bfloat16_rn(b));
    return lo ? b - hi : hi;
}

// full image from the master parameters (pads are zero)
__global__ void k_mlp_pack(const float *__restrict__ p, uint8_t *__restrict__ image) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int NB = (OFF_B1 - OFF_W1) / 2, NF = (IMAGE_BYTES - OFF_B1) / 4;
    if (e < NB) {
        int base, R, off;
        if (e < N1 * K0) { base = 0; R = N1; off = OFF_W1; }
        else if (e < N1 * K0 + N2 * N1) { base = N1 * K0; R = N2; off = OFF_W2; }
        else { base = N1 * K0 + N2 * N1; R = N3; off = OFF_W3; }
        const int le = e - base, cb = le / (R * 8), rem = le % (R * 8);
        const int row = rem / 8, col = cb * 8 + rem % 8;
        float v = 0.f;
        if (off == OFF_W1) {
            if (row < H1 && col < DIN) v = p[P_W1 + row * DIN + col];
            else if (row < H1 && col >= DIN && col < 2 * DIN) v = p[P_W1 + row * DIN + col - DIN];
            else if (row < H1 && (col == ONES0 || col == ONES0 + 1)) v = bias_part(p[P_B1 + row], col != ONES0);
        } else if (off == OFF_W2) {
            if (row < H2 && col < H1) v = p[P_W2 + row * H1 + col];
            else if (row < H2 && (col == ONES1 || col == ONES1 + 1)) v = bias_part(p[P_B2 + row], col != ONES1);
        } else {
            if (row < H3 && col < H2) v = p[P_W3 + row * H2 + col];
            else if (row < H3 && (col == ONES1 || col == ONES1 + 1)) v = bias_part(p[P_B3 + row], col != ONES1);
        }
        reinterpret_cast<__nv_bfloat16 *>(image + off)[le] = __float2bfloat16_rn(v);
    } else if (e < NB + NF) {
        const int f = e - NB;  // fp32 word index from OFF_B1
        const int byte = OFF_B1 + 4 * f;
        float v = 0.f;
        if (byte < OFF_B2) { const int i = f; if (i < H1) v = p[P_B1 + i]; }
        else if (byte < OFF_B3) { const int i = (byte - OFF_B2) / 4; if (i < H2) v = p[P_B2 + i]; }
        else if (byte < OFF_W4) { const int i = (byte - OFF_B3) / 4; if (i < H3) v = p[P_B3 + i]; }
        else if (byte < OFF_B4) { const int i = (byte - OFF_W4) / 4; if (i < H3) v = p[P_W4 + i]; }
        else { if (byte == OFF_B4) v = p[P_B4]; }
        reinterpret_cast<float *>(image)[OFF_B1 / 4 + f] = v;
    }
}

// Adam over the summed per-CTA partials (fixed CTA order: deterministic), then
// refresh the parameter's places in the bf16 image.
__global__ void k_mlp_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ part, int n_part, float lr, float b1, float b2, float eps,
                           float bc1, float bc2, uint8_t *__restrict__ image) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAMS) return;
    float g = 0.f;
    for (int c = 0; c < n_part; ++c) g += part[(int64_t)c * PSTRIDE + i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float w = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    p[i] = w;
    __nv_bfloat16 *w1 = reinterpret_cast<__nv_bfloat16 *>(image + OFF_W1);
    __nv_bfloat16 *w2 = reinterpret_cast<__nv_bfloat16 *>(image + OFF_W2);
    __nv_bfloat16 *w3 = reinterpret_cast<__nv_bfloat16 *>(image + OFF_W3);
    float *f = reinterpret_cast<float *>(image);
    const __nv_bfloat16 wb = __float2bfloat16_rn(w);
    if (i < P_B1) {
        const int o = i / DIN, j = i % DIN;
        w1[img_index(N1, o, j)] = wb;
        w1[img_index(N1, o, j + DIN)] = wb;
    } else if (i < P_W2) {
        const int o = i - P_B1;
        f[OFF_B1 / 4 + o] = w;
        w1[img_index(N1, o, ONES0)] = __float2bfloat16_rn(bias_part(w, false));
        w1[img_index(N1, o, ONES0 + 1)] = __float2bfloat16_rn(bias_part(w, true));
    } else if (i < P_B2) { const int o = (i - P_W2) / H1, c = (i - P_W2) % H1; w2[img_index(N2, o, c)] = wb; }
    else if (i < P_W3) {
        const int o = i - P_B2;
        f[OFF_B2 / 4 + o] = w;
        w2[img_index(N2, o, ONES1)] = __float2bfloat16_rn(bias_part(w, false));
        w2[img_index(N2, o, ONES1 + 1)] = __float2bfloat16_rn(bias_part(w, true));
    } else if (i < P_B3) { const int o = (i - P_W3) / H2, c = (i - P_W3) % H2; w3[img_index(N3, o, c)] = wb; }
    else if (i < P_W4) {
        const int o = i - P_B3;
        f[OFF_B3 / 4 + o] = w;
        w3[img_index(N3, o, ONES1)] = __float2bfloat16_rn(bias_part(w, false));
        w3[img_index(N3, o, ONES1 + 1)] = __float2bfloat16_rn(bias_part(w, true));
    }
    else if (i < P_B4) f[OFF_W4 / 4 + (i - P_W4)] = w;
    else f[OFF_B4 / 4] = w;
}

template <int MODE>
static int launch(const void *image, const float *x, int64_t n, int x_stride, const float *nc, const float *ns,
                  float *out, float *dx, int dx_stride, int loss_kind, float inv_batch, float *part,
                  float *part_loss, int grid, int *status, cudaStream_t st) {
    static bool configured[64] = {false};
    int dev = 0;
    SSM_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && !configured[dev]) {
        SSM_CUDA(cudaFuncSetAttribute(k_mlp<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes<MODE>()));
        configured[dev] = true;
    }
    Norm nm;
    for (int j = 0; j < 8; ++j) {
        nm.c[j] = (j < DIN && nc) ? nc[j] : 0.f;
        nm.s[j] = (j < DIN && ns) ? ns[j] : 1.f;
    }
    k_mlp<MODE><<<grid, 128 * Cfg<MODE>::NWG, smem_bytes<MODE>(), st>>>(
        (const uint8_t *)image, x, n, x_stride, nm, out, dx, dx_stride, loss_kind, inv_batch, part, part_loss,
        status);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

}  // namespace mlp
}  // namespace ssm

using namespace ssm;
using namespace ssm::mlp;

extern "C" {

int ssm_mlp_pack(const float *params, void *image, void *stream) {
    SSM_REQUIRE(params && image, "ssm_mlp_pack: null pointer");
    constexpr int total = (OFF_B1 - OFF_W1) / 2 + (IMAGE_BYTES - OFF_B1) / 4;
    k_mlp_pack<<<(total + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, (uint8_t *)image);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

int ssm_mlp_forward(const void *image, const float *x, int64_t n, int x_stride, const float *norm_c,
                    const float *norm_s, float *out, float *dx, int dx_stride, int max_ctas, int *status,
                    void *stream) {
    SSM_REQUIRE(n >= 0, "ssm_mlp_forward: n < 0");
    if (n == 0) return SSM_OK;
    SSM_REQUIRE(image && x && out, "ssm_mlp_forward: null pointer");
    SSM_REQUIRE(((uintptr_t)image & 15) == 0, "ssm_mlp_forward: image must be 16-byte aligned");
    SSM_REQUIRE(x_stride >= DIN, "ssm_mlp_forward: x_stride < 7");
    SSM_REQUIRE(!dx || dx_stride >= DIN, "ssm_mlp_forward: dx_stride < 7");
    const int64_t tiles = (n + 127) / 128;
    const int nwg = dx ? Cfg<FWD_DX>::NWG : Cfg<FWD>::NWG;
    int grid = (int)std::min<int64_t>((tiles + nwg - 1) / nwg, (int64_t)sm_count());
    if (max_ctas > 0) grid = std::min(grid, max_ctas);
    cudaStream_t st = (cudaStream_t)stream;
    if (dx)
        return launch<FWD_DX>(image, x, n, x_stride, norm_c, norm_s, out, dx, dx_stride, 0, 0.f, nullptr, nullptr,
                              grid, status, st);
    return launch<FWD>(image, x, n, x_stride, norm_c, norm_s, out, nullptr, 0, 0, 0.f, nullptr, nullptr, grid,
                       status, st);
}

int ssm_mlp_train_grad(const void *image, const float *records, int64_t n, int rec_stride, const float *norm_c,
                       const float *norm_s, int loss_kind, float inv_batch, float *out, float *partials,
                       float *loss_partials, int n_ctas, int *status, void *stream) {
    SSM_REQUIRE(n > 0, "ssm_mlp_train_grad: empty batch");
    SSM_REQUIRE(image && records && partials && loss_partials, "ssm_mlp_train_grad: null pointer");
    SSM_REQUIRE(((uintptr_t)image & 15) == 0, "ssm_mlp_train_grad: image must be 16-byte aligned");
    SSM_REQUIRE(rec_stride >= DIN + 1, "ssm_mlp_train_grad: rec_stride < 8");
    SSM_REQUIRE(loss_kind == 0 || loss_kind == 1, "ssm_mlp_train_grad: loss_kind must be 0 (huber) or 1 (mse)");
    SSM_REQUIRE(n_ctas > 0, "ssm_mlp_train_grad: n_ctas must be positive");
    return launch<TRAIN>(image, records, n, rec_stride, norm_c, norm_s, out, nullptr, 0, loss_kind, inv_batch,
                         partials, loss_partials, n_ctas, status, (cudaStream_t)stream);
}

int ssm_mlp_adam(float *params, float *m, float *v, const float *partials, int n_partials, float lr, float beta1,
                 float beta2, float eps, float bias_corr1, float bias_corr2, void *image, void *stream) {
    SSM_REQUIRE(params && m && v && partials && image, "ssm_mlp_adam: null pointer");
    SSM_REQUIRE(n_partials > 0, "ssm_mlp_adam: n_partials must be positive");
    k_mlp_adam<<<(NPARAMS + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        params, m, v, partials, n_partials, lr, beta1, beta2, eps, bias_corr1, bias_corr2, (uint8_t *)image);
    SSM_CUDA(cudaGetLastError());
    return SSM_OK;
}

}  // extern "C"
