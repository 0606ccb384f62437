// Per-vertex MLP of the learned smoother: 9 features -> 64 -> 64 -> 3, GELU,
// BF16 weights and activations as tensor-core operands, FP32 accumulation.
//
//   inference  k_mlp_tc: tcgen05.mma (kind::f16, BF16 x BF16 -> FP32 in TMEM),
//              operands staged in shared memory by bulk async copies (TMA
//              engine), one CTA per 128-row tile, the three layers chained
//              through TMEM -> registers (bias, GELU) -> shared memory.
//   training   k_mlp_fwd_bwd: SIMT forward + hand-written backward with the same
//              BF16 rounding of the weights and activations, FP32 math;
//              per-block gradient partials summed in a fixed order.
//
// Parameter vector (FP32 master copy, 4,995 floats):
//   W1[64][9]  b1[64]  W2[64][64]  b2[64]  W3[3][64]  b3[3]
// Device image for the tensor cores (bf16, K-major, no swizzle, "interleaved"
// core matrices of 8 rows x 16 bytes):
//   W1 64x16 (K padded 9->16 with zeros) | W2 64x64 | W3 16x64 (rows padded
//   3->16 with zeros) | b1[64] b2[64] b3[16] (fp32)
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace mgsb {
namespace {

constexpr int kMlpIn = 9, kMlpInPad = 16, kMlpHid = 64, kMlpOut = 3, kMlpOutPad = 16;
constexpr int kMlpTile = 128;   // rows per tensor-core tile (MMA M)
constexpr int kMlpParams = kMlpHid * kMlpIn + kMlpHid + kMlpHid * kMlpHid + kMlpHid + kMlpOut * kMlpHid + kMlpOut;
// parameter offsets
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpHid * kMlpIn, kOffW2 = kOffB1 + kMlpHid,
              kOffB2 = kOffW2 + kMlpHid * kMlpHid, kOffW3 = kOffB2 + kMlpHid, kOffB3 = kOffW3 + kMlpOut * kMlpHid;
static_assert(kOffB3 + kMlpOut == kMlpParams, "parameter layout");
// image offsets (bytes)
constexpr int kImgW1 = 0, kImgW2 = kImgW1 + kMlpHid * kMlpInPad * 2, kImgW3 = kImgW2 + kMlpHid * kMlpHid * 2,
              kImgB = kImgW3 + kMlpOutPad * kMlpHid * 2, kImgBytes = kImgB + (2 * kMlpHid + kMlpOutPad) * 4;
constexpr int kTileBytes = kMlpTile * kMlpInPad * 2;   // one feature tile: 4 KiB

// Byte offset of element (row, k) in a K-major interleaved tile of K columns:
// 8-row groups of (K/8) core matrices, each core matrix 8 rows x 16 bytes.
__host__ __device__ constexpr int interleaved_offset(int row, int k, int K) {
    return (row >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// GELU in its tanh form (Hendrycks & Gimpel 2016):
//   g(x) = x/2 (1 + tanh(u)),  u = sqrt(2/pi) (x + 0.044715 x^3),
// with the hardware tanh.approx.f32 (well below the BF16 rounding of the
// activations that follows), the same in inference and in training.
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluC = 0.7978845608028654f, kGeluA = 0.044715f;
// u = x (C + C A x^2), g = h + h t with h = x/2: six instructions (the
// epilogues apply it to every hidden activation).
__device__ __forceinline__ float gelu(float x) {
    const float t = tanh_hw(x * fmaf(kGeluC * kGeluA, x * x, kGeluC));
    const float h = 0.5f * x;
    return fmaf(h, t, h);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float t = tanh_hw(x * fmaf(kGeluC * kGeluA, x * x, kGeluC));
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * kGeluC * fmaf(3.f * kGeluA, x * x, 1.f);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// ---------------------------------------------------------------------------
// Packing: FP32 parameters -> BF16 tensor-core image (+ FP32 biases)
// ---------------------------------------------------------------------------
__global__ void k_mlp_pack(const float* __restrict__ prm, uint8_t* __restrict__ img) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    __nv_bfloat16* w1 = reinterpret_cast<__nv_bfloat16*>(img + kImgW1);
    __nv_bfloat16* w2 = reinterpret_cast<__nv_bfloat16*>(img + kImgW2);
    __nv_bfloat16* w3 = reinterpret_cast<__nv_bfloat16*>(img + kImgW3);
    float* bias = reinterpret_cast<float*>(img + kImgB);
    if (t < kMlpHid * kMlpInPad) {
        const int n = t / kMlpInPad, k = t % kMlpInPad;
        const float v = k < kMlpIn ? prm[kOffW1 + n * kMlpIn + k] : 0.f;
        w1[interleaved_offset(n, k, kMlpInPad) / 2] = __float2bfloat16_rn(v);
    }
    if (t < kMlpHid * kMlpHid) {
        const int n = t / kMlpHid, k = t % kMlpHid;
        w2[interleaved_offset(n, k, kMlpHid) / 2] = __float2bfloat16_rn(prm[kOffW2 + n * kMlpHid + k]);
    }
    if (t < kMlpOutPad * kMlpHid) {
        const int n = t / kMlpHid, k = t % kMlpHid;
        const float v = n < kMlpOut ? prm[kOffW3 + n * kMlpHid + k] : 0.f;
        w3[interleaved_offset(n, k, kMlpHid) / 2] = __float2bfloat16_rn(v);
    }
    if (t < kMlpHid) {
        bias[t] = prm[kOffB1 + t];
        bias[kMlpHid + t] = prm[kOffB2 + t];
    }
    if (t < kMlpOutPad) bias[2 * kMlpHid + t] = t < kMlpOut ? prm[kOffB3 + t] : 0.f;
}

// Row-major FP32 features [n][9] -> BF16 interleaved tiles (rows padded to a
// multiple of 128 with zeros).
__global__ void k_mlp_tile_features(int n, int ntiles, const float* __restrict__ x, uint8_t* __restrict__ tiles) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles * kMlpTile * kMlpInPad) return;
    const int row = t / kMlpInPad, k = t % kMlpInPad;
    const int tile = row / kMlpTile, r = row % kMlpTile;
    const float v = (row < n && k < kMlpIn) ? x[(size_t)row * kMlpIn + k] : 0.f;
    reinterpret_cast<__nv_bfloat16*>(tiles + (size_t)tile * kTileBytes)[interleaved_offset(r, k, kMlpInPad) / 2] =
        __float2bfloat16_rn(v);
}

// ---------------------------------------------------------------------------
// tcgen05 / bulk-copy / mbarrier helpers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bounded wait on phase `parity`; false when the bound ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int max_polls) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < max_polls; ++i) {
        uint32_t done = 0;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// 1-D bulk async copy global -> shared, completion counted on `bar` (16-byte
// aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// UMMA shared-memory descriptor, K-major, no swizzle: LBO = byte stride between
// the two 16-byte K chunks of one MMA, SBO = byte stride between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(const void* p, uint32_t lbo, uint32_t sbo) {
    const uint64_t addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
           (1ull << 46);   // version 1 (sm100), base offset 0, layout SWIZZLE_NONE
}
// Instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 32 lanes x 32-bit, 16 consecutive columns per thread.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Inference: one CTA (4 warps) per 128-row tile, grid-strided over tiles.
//   out_mode 0: y[row] = (y0, y1, y2, 0)
//   out_mode 1: e[row] += scale[row] * (y0, y1, y2)   (learned smoothing sweep)
// err (optional): set to 1 when a bounded wait ran out; the kernel then stops.
// ---------------------------------------------------------------------------
constexpr int kMlpThreads = 256;   // 8 warps: warp w serves TMEM lanes 32 (w % 4).. and hidden columns 32 (w / 4)..
constexpr int kTmemCols = 256;     // D1 cols [0,64), D2 [64,128), D3 [128,144)
constexpr int kMaxPolls = 1 << 22;

struct MlpSmem {
    alignas(128) uint8_t x[kTileBytes];                          // 128 x 16 bf16
    alignas(128) uint8_t w[kImgBytes];                           // weights + biases
    alignas(128) uint8_t h[kMlpTile * kMlpHid * 2];              // 128 x 64 bf16 (layer 2 and 3 A operand)
    alignas(8) uint64_t bar_load, bar_mma, bar_win;   // bar_win: the learned sweep's residual window
    uint32_t tmem_base;
    int stop;
};

// Dynamic shared memory of k_mlp_tc: at least 80 KiB, so that at most two CTAs
// (2 x 256 TMEM columns) are resident per SM and tcgen05.alloc never waits.
inline size_t mlp_tc_smem_bytes() { return sizeof(MlpSmem) > 80 * 1024 ? sizeof(MlpSmem) : (size_t)80 * 1024; }

// Bounded waits of one thread; the first wait that ran out is remembered so
// that it can be retried once before TMEM is released (no copy or MMA of the
// CTA is then left in flight).
struct WaitState {
    uint64_t* fail_bar = nullptr;
    uint32_t fail_par = 0;
};
__device__ __forceinline__ bool wait_bar(WaitState& ws, uint64_t* bar, uint32_t par) {
    const bool done = mbar_wait(bar, par, kMaxPolls);
    if (!done && !ws.fail_bar) {
        ws.fail_bar = bar;
        ws.fail_par = par;
    }
    return done;
}

// CTA prologue: barriers, TMEM (256 columns, warp 0) and the weight image.
// With wait_weights = false the copy is left in flight (the caller overlaps it
// with other work and calls mlp_wait_weights before the first MMA).
__device__ __forceinline__ uint32_t mlp_cta_setup(MlpSmem& S, const uint8_t* img, WaitState& ws, uint32_t& ph_load,
                                                  int32_t* err, bool wait_weights = true) {
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(&S.bar_load, 1);
        mbar_init(&S.bar_mma, 1);
        mbar_init(&S.bar_win, 1);
        S.stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&S.bar_load, kImgBytes);
        bulk_g2s(S.w, img, kImgBytes, &S.bar_load);
    }
    if (wait_weights) {
        if (!wait_bar(ws, &S.bar_load, ph_load)) {
            S.stop = 1;
            if (err) atomicExch(err, 1);
        }
        ph_load ^= 1;
    }
    return S.tmem_base;
}

// Completes a weight copy left in flight by mlp_cta_setup(..., false).
__device__ __forceinline__ bool mlp_wait_weights(MlpSmem& S, WaitState& ws, uint32_t& ph_load, int32_t* err) {
    const bool ok = wait_bar(ws, &S.bar_load, ph_load);
    ph_load ^= 1;
    if (!ok) {
        S.stop = 1;
        if (err) atomicExch(err, 1);
    }
    return ok;
}

// CTA epilogue: retry a timed-out wait once, then release TMEM.
__device__ __forceinline__ void mlp_cta_teardown(MlpSmem& S, uint32_t tmem, WaitState& ws) {
    if (ws.fail_bar) mbar_wait(ws.fail_bar, ws.fail_par, kMaxPolls);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Hidden layer epilogue: gelu(D + bias) of this warp's half of the 64 columns
// (c0 = 0 or 32) of this thread's row, from TMEM -> BF16 into S.h (K-major
// interleaved, K = 64).
__device__ __forceinline__ void mlp_hidden_epilogue(MlpSmem& S, uint32_t taddr, const float* bias, int row_in_tile,
                                                    int c0) {
    // both 16-column loads in flight before the one wait
    static_assert(kMlpHid / 2 == 32, "a warp's half of the hidden columns is two 16-column loads");
    float v[2][16];
    tmem_ld16(taddr + c0, v[0]);
    tmem_ld16(taddr + c0 + 16, v[1]);
    tmem_wait_ld();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int c = c0 + 16 * h;
        uint32_t packed[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const __nv_bfloat162 two = __floats2bfloat162_rn(gelu(v[h][2 * i] + bias[c + 2 * i]),
                                                             gelu(v[h][2 * i + 1] + bias[c + 2 * i + 1]));
            packed[i] = *reinterpret_cast<const uint32_t*>(&two);
        }
        uint8_t* base = S.h + interleaved_offset(row_in_tile, c, kMlpHid);
        *reinterpret_cast<uint4*>(base) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *reinterpret_cast<uint4*>(base + 128) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
    }
}

// The three layers on the feature tile in S.x (which the caller has made
// visible to the async proxy and synchronised); y receives this thread's row.
// Returns false when a wait ran out.
__device__ __forceinline__ bool mlp_tile_layers(MlpSmem& S, uint32_t tmem, uint32_t& ph_mma, WaitState& ws, bool ok,
                                                float (&y)[3]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp & 3, c0 = (warp >> 2) * (kMlpHid / 2);
    const int row_in_tile = grp * 32 + lane;
    const uint32_t lane_base = (uint32_t)(grp * 32) << 16;
    const float* bias = reinterpret_cast<const float*>(S.w + kImgB);
    const uint32_t id64 = umma_idesc_bf16(kMlpTile, kMlpHid), id16 = umma_idesc_bf16(kMlpTile, kMlpOutPad);
    // layer 1: D1 = X W1^T (K = 16: one MMA)
    tc_fence_after();
    if (threadIdx.x == 0 && ok) {
        umma_bf16(tmem + 0, umma_desc(S.x, 128, 256), umma_desc(S.w + kImgW1, 128, 256), id64, 0);
        umma_commit(&S.bar_mma);
    }
    ok = ok && wait_bar(ws, &S.bar_mma, ph_mma);
    ph_mma ^= 1;
    tc_fence_after();
    mlp_hidden_epilogue(S, tmem + lane_base + 0, bias, row_in_tile, c0);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // layer 2: D2 = H1 W2^T (K = 64: four MMAs)
    if (threadIdx.x == 0 && ok) {
#pragma unroll
        for (int k = 0; k < kMlpHid / 16; ++k)
            umma_bf16(tmem + 64, umma_desc(S.h + k * 256, 128, 1024), umma_desc(S.w + kImgW2 + k * 256, 128, 1024), id64,
                      k > 0 ? 1u : 0u);
        umma_commit(&S.bar_mma);
    }
    ok = ok && wait_bar(ws, &S.bar_mma, ph_mma);
    ph_mma ^= 1;
    tc_fence_after();
    // H2 overwrites H1: layer 2 has finished reading it
    mlp_hidden_epilogue(S, tmem + lane_base + 64, bias + kMlpHid, row_in_tile, c0);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // layer 3: D3 = H2 W3^T (N = 16, 3 used)
    if (threadIdx.x == 0 && ok) {
#pragma unroll
        for (int k = 0; k < kMlpHid / 16; ++k)
            umma_bf16(tmem + 128, umma_desc(S.h + k * 256, 128, 1024), umma_desc(S.w + kImgW3 + k * 256, 128, 1024),
                      id16, k > 0 ? 1u : 0u);
        umma_commit(&S.bar_mma);
    }
    ok = ok && wait_bar(ws, &S.bar_mma, ph_mma);
    ph_mma ^= 1;
    tc_fence_after();
    float v[16];
    tmem_ld16(tmem + lane_base + 128, v);   // every warp (the .sync.aligned load is warp-wide); warps 0-3 use it
    tmem_wait_ld();
    tc_fence_before();
    y[0] = v[0] + bias[2 * kMlpHid];
    y[1] = v[1] + bias[2 * kMlpHid + 1];
    y[2] = v[2] + bias[2 * kMlpHid + 2];
    return ok;
}

// Inference over feature tiles in global memory: one CTA (4 warps) per
// 128-row tile, grid-strided.
//   out_mode 0: y[row] = (y0, y1, y2, 0)
//   out_mode 1: e[row] += scale[row] * (y0, y1, y2)
// err (optional): set to 1 when a bounded wait ran out; the kernel then stops.
__global__ void __launch_bounds__(kMlpThreads) k_mlp_tc(int n, int ntiles, const uint8_t* __restrict__ tiles,
                                                        const uint8_t* __restrict__ img, int out_mode,
                                                        float4* __restrict__ y, float4* __restrict__ e,
                                                        const float* __restrict__ scale, int32_t* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
    WaitState ws;
    uint32_t ph_load = 0, ph_mma = 0;
    const uint32_t tmem = mlp_cta_setup(S, img, ws, ph_load, err);
    const int row_in_tile = threadIdx.x;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        if (S.stop) break;
        if (threadIdx.x == 0) {
            mbar_expect_tx(&S.bar_load, kTileBytes);
            bulk_g2s(S.x, tiles + (size_t)tile * kTileBytes, kTileBytes, &S.bar_load);
        }
        bool ok = wait_bar(ws, &S.bar_load, ph_load);
        ph_load ^= 1;
        float out[3];
        ok = mlp_tile_layers(S, tmem, ph_mma, ws, ok, out);
        if (!ok) {
            S.stop = 1;
            if (err) atomicExch(err, 1);
        }
        const int row = tile * kMlpTile + row_in_tile;
        if (ok && row_in_tile < kMlpTile && row < n) {
            if (out_mode == 0) {
                y[row] = make_float4(out[0], out[1], out[2], 0.f);
            } else {
                const float sc = scale[row];
                float4 q = e[row];
                q.x += sc * out[0];
                q.y += sc * out[1];
                q.z += sc * out[2];
                e[row] = q;
            }
        }
    }
    mlp_cta_teardown(S, tmem, ws);
}

// ---------------------------------------------------------------------------
// Training: forward + backward for a block of 128 samples (one thread per
// sample for the per-sample passes), FP32 math with the same BF16 rounding of
// the weights and activations as the tensor-core forward (straight-through in
// the backward).  Loss = mean over samples and the 3 outputs of (y - t)^2.
// Activations live in shared memory feature-major ([unit][sample], row stride
// 129 against bank conflicts); the weight gradients are then formed
// cooperatively as dot products over the block's samples, so every block
// writes its gradient sum to grad_part[block][kMlpParams] without atomics, and
// k_mlp_reduce sums the blocks in a fixed order (deterministic).
// ---------------------------------------------------------------------------
constexpr int kTrainThreads = 128;
constexpr int kTrainLd = kTrainThreads + 1;
constexpr size_t kTrainSmem =
    sizeof(float) * ((size_t)kMlpParams + (4 * kMlpHid + kMlpIn + kMlpOut) * (size_t)kTrainLd + kTrainThreads);

__global__ void __launch_bounds__(kTrainThreads) k_mlp_fwd_bwd(int nb, const int32_t* __restrict__ idx,
                                                               const float* __restrict__ X, const float* __restrict__ T,
                                                               const float* __restrict__ prm, float* __restrict__ grad_part,
                                                               float* __restrict__ loss_part, float inv_count) {
    extern __shared__ float tsm[];
    float* w = tsm;                                   // BF16-rounded weights, exact biases
    float* Z1 = w + kMlpParams;                       // [64][129] pre-activations, then dZ1
    float* H1 = Z1 + kMlpHid * kTrainLd;              // [64][129]
    float* Z2 = H1 + kMlpHid * kTrainLd;              // [64][129] then dZ2
    float* H2 = Z2 + kMlpHid * kTrainLd;              // [64][129]
    float* Xs = H2 + kMlpHid * kTrainLd;              // [9][129]
    float* dY = Xs + kMlpIn * kTrainLd;               // [3][129]
    float* lsum = dY + kMlpOut * kTrainLd;            // [128]
    for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x) {
        const bool is_bias = (q >= kOffB1 && q < kOffW2) || (q >= kOffB2 && q < kOffW3) || q >= kOffB3;
        w[q] = is_bias ? prm[q] : bf16r(prm[q]);
    }
    __syncthreads();
    const int s = threadIdx.x;
    const int gs = blockIdx.x * blockDim.x + s;
    const bool valid = gs < nb;
    const int row = valid ? (idx ? idx[gs] : gs) : 0;
    // ---- forward
    float loss = 0.f;
    for (int k = 0; k < kMlpIn; ++k) Xs[k * kTrainLd + s] = valid ? bf16r(X[(size_t)row * kMlpIn + k]) : 0.f;
    for (int j = 0; j < kMlpHid; ++j) {
        float a = w[kOffB1 + j];
        for (int k = 0; k < kMlpIn; ++k) a = fmaf(w[kOffW1 + j * kMlpIn + k], Xs[k * kTrainLd + s], a);
        Z1[j * kTrainLd + s] = a;
        H1[j * kTrainLd + s] = bf16r(gelu(a));
    }
    for (int j = 0; j < kMlpHid; ++j) {
        float a = w[kOffB2 + j];
        for (int k = 0; k < kMlpHid; ++k) a = fmaf(w[kOffW2 + j * kMlpHid + k], H1[k * kTrainLd + s], a);
        Z2[j * kTrainLd + s] = a;
        H2[j * kTrainLd + s] = bf16r(gelu(a));
    }
    for (int o = 0; o < kMlpOut; ++o) {
        float a = w[kOffB3 + o];
        for (int k = 0; k < kMlpHid; ++k) a = fmaf(w[kOffW3 + o * kMlpHid + k], H2[k * kTrainLd + s], a);
        const float d = valid ? a - T[(size_t)row * kMlpOut + o] : 0.f;
        loss += d * d;
        dY[o * kTrainLd + s] = 2.f * d * inv_count;
    }
    // ---- backward through layer 3 and 2 (own sample only)
    for (int k = 0; k < kMlpHid; ++k) {
        float a = 0.f;
        for (int o = 0; o < kMlpOut; ++o) a = fmaf(dY[o * kTrainLd + s], w[kOffW3 + o * kMlpHid + k], a);
        Z2[k * kTrainLd + s] = a * gelu_grad(Z2[k * kTrainLd + s]);   // dZ2
    }
    for (int k = 0; k < kMlpHid; ++k) {
        float a = 0.f;
        for (int j = 0; j < kMlpHid; ++j) a = fmaf(Z2[j * kTrainLd + s], w[kOffW2 + j * kMlpHid + k], a);
        Z1[k * kTrainLd + s] = a * gelu_grad(Z1[k * kTrainLd + s]);   // dZ1
    }
    lsum[s] = loss;
    __syncthreads();
    // ---- weight gradients: dot products over the block's samples
    float* gp = grad_part + (size_t)blockIdx.x * kMlpParams;
    for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x) {
        const float *u, *v = nullptr;
        if (q < kOffB1) {
            const int j = (q - kOffW1) / kMlpIn, i = (q - kOffW1) % kMlpIn;
            u = Z1 + j * kTrainLd;
            v = Xs + i * kTrainLd;
        } else if (q < kOffW2) {
            u = Z1 + (q - kOffB1) * kTrainLd;
        } else if (q < kOffB2) {
            const int j = (q - kOffW2) / kMlpHid, k = (q - kOffW2) % kMlpHid;
            u = Z2 + j * kTrainLd;
            v = H1 + k * kTrainLd;
        } else if (q < kOffW3) {
            u = Z2 + (q - kOffB2) * kTrainLd;
        } else if (q < kOffB3) {
            const int o = (q - kOffW3) / kMlpHid, k = (q - kOffW3) % kMlpHid;
            u = dY + o * kTrainLd;
            v = H2 + k * kTrainLd;
        } else {
            u = dY + (q - kOffB3) * kTrainLd;
        }
        float a = 0.f;
        if (v)
            for (int t = 0; t < kTrainThreads; ++t) a = fmaf(u[t], v[t], a);
        else
            for (int t = 0; t < kTrainThreads; ++t) a += u[t];
        gp[q] = a;
    }
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < kTrainThreads; ++i) t += lsum[i];
        loss_part[blockIdx.x] = t;
    }
}

// grad[q] = sum_b grad_part[b][q] (fixed order); loss = sum_b loss_part[b] * inv_count.
__global__ void k_mlp_reduce(int nblk, const float* __restrict__ grad_part, const float* __restrict__ loss_part,
                             float inv_count, float* __restrict__ grad, float* __restrict__ loss) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < kMlpParams) {
        float a = 0.f;
        for (int b = 0; b < nblk; ++b) a += grad_part[(size_t)b * kMlpParams + q];
        grad[q] = a;
    }
    if (q == 0) {
        float l = 0.f;
        for (int b = 0; b < nblk; ++b) l += loss_part[b];
        *loss = l * inv_count;
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; step t >= 1.
__global__ void k_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kMlpParams) return;
    const float gq = grad[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    prm[q] -= lr * (mq / bc1) / (sqrtf(vq / bc2) + eps);
}

// Uniform sample indices in [0, n) from a counter-based hash (splitmix64).
__global__ void k_sample_indices(int nb, int n, uint64_t seed, uint64_t step, int32_t* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nb) return;
    uint64_t z = seed + (step * 0x9E3779B97F4A7C15ull) + (uint64_t)s * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    idx[s] = (int32_t)(z % (uint64_t)n);
}

}  // namespace
}  // namespace mgsb
