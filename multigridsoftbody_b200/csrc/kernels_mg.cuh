// Multigrid global-step kernels (sm_100a).  Included by solver.cu only.
//
// SpMV layout: sliced ELL with slice height S = 32/G; entry k of row r of
// slice s sits at slice_ptr[s] + k*S + (r mod S).  A warp covers S rows with
// G lanes per row; lane l handles entries k = l/S, l/S + G, ... so a warp
// reads 32 consecutive entries per step, and the G partial sums of a row are
// combined with xor-shuffles over lane offsets S, 2S, ..., 16.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace mgsb {

namespace cg = cooperative_groups;

constexpr int kMaxLevels = 12;
constexpr int kLanesL0 = 4;   // lanes per row at level 0 (slice height 8)
constexpr int kLanesC = 8;    // lanes per row on coarse levels (slice height 4)

struct LevelView {
    int n;
    const int32_t* slice_ptr;
    const int32_t* col;
    const float* val;
    const float* dfull;
    const float* dinv;
    float4* r;
    float4* e;
    float4* e2;
    float4* res;
    const int4* pid;      // prolongation rows of the next finer level
    const float4* pw;
    const int32_t* rptr;  // restriction: children in the next finer level
    const int32_t* rcol;
    const float* rw;
    const int32_t* op_slice_ptr;   // OP = Off * P(next coarser level), sliced ELL
    const int32_t* op_col;
    const float* op_val;
};

struct CoarseArgs {
    int L;
    int pre, post;
    int fuse_l0;             // level-0 residual and prolongation inside the kernel
    int first;               // shared-memory kernel: first level it owns (>= 1); input lv[first-1].res, output lv[first].e
    int fuse_prolong;        // prolongation + first post-sweep in one phase (OP = Off P), as k_prolong_sweep
    const int2* range;       // [nbody * L]: (first row, rows) of each body on each level
    const int32_t* dense_off;
    const float* Ainv;       // coarsest inverse blocks (row-major per body)
    const double* Ainv64;    // FP64 coarsest inverse (mixed precision), else null
    const float4* b;         // level-0 right-hand side
    float4* d;               // level-0 unknown (displacement)
    const int32_t* gate;     // if set, the kernel runs only when *gate != 0 (learned-smoother fallback)
    // level-1 right-hand side straight from level 0 (host launches only): with res0_b set, level 1's
    // restriction forms R (res0_b - D0 d) - RO d, RO = R Off(level 0), and lv[0].res is not read
    const float4* res0_b;
    const int32_t* ro_ptr;
    const int32_t* ro_col;
    const float* ro_val;
    LevelView lv[kMaxLevels];
};

__device__ __forceinline__ float4 f4z() { return make_float4(0.f, 0.f, 0.f, 0.f); }

// Block sum: warp xor-shuffles, then thread 0 adds the warp sums in order.
// Every thread of the block calls it; the result is valid in thread 0.
__device__ __forceinline__ float block_sum_f(float v, float* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;
}

// Load of a vector that may have been written earlier in the same kernel by
// another CTA of the cluster: a plain (coherent) load, never the read-only path.
template <bool kReadOnly>
__device__ __forceinline__ float4 vload(const float4* p) {
    if constexpr (kReadOnly)
        return __ldg(p);
    else
        return *p;
}

// Partial off-diagonal product of `row` for this lane (sub = lane / S), then
// reduced over the G lanes of the row.  Every lane of the warp must call it.
// kReadOnly: x is not written during the calling kernel.
template <int G, bool kReadOnly = true>
__device__ __forceinline__ float4 rg_offdiag(int row, bool valid, int lane, const int32_t* __restrict__ sp,
                                             const int32_t* __restrict__ col, const float* __restrict__ val,
                                             const float4* x) {
    constexpr int S = 32 / G;
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (valid) {
        const int slice = row / S;
        const int beg = __ldg(sp + slice), end = __ldg(sp + slice + 1);
#pragma unroll 2
        for (int e = beg + (lane / S) * S + (row - slice * S); e < end; e += 32) {
            const float a = __ldg(val + e);
            const float4 xv = vload<kReadOnly>(x + __ldg(col + e));
            ax = fmaf(a, xv.x, ax);
            ay = fmaf(a, xv.y, ay);
            az = fmaf(a, xv.z, az);
        }
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    return make_float4(ax, ay, az, 0.f);
}

// Sum of w * v[idx] over a CSR row split across the G lanes of the row.
template <int G, bool kReadOnly = true>
__device__ __forceinline__ float4 rg_csr_sum(bool valid, int lane, int beg, int end, const int32_t* __restrict__ idx,
                                             const float* __restrict__ w, const float4* v) {
    constexpr int S = 32 / G;
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (valid) {
#pragma unroll 2
        for (int q = beg + lane / S; q < end; q += G) {
            const float c = __ldg(w + q);
            const float4 t = vload<kReadOnly>(v + __ldg(idx + q));
            ax = fmaf(c, t.x, ax);
            ay = fmaf(c, t.y, ay);
            az = fmaf(c, t.z, az);
        }
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    return make_float4(ax, ay, az, 0.f);
}

// ---------------------------------------------------------------------------
// Row structure held in registers.  The sliced-ELL and CSR arrays of every
// level (columns, values, children, weights, parents) are uploaded once at
// set-up and never written by a kernel, so a kernel may load this lane's
// share of its row's entries before the dependency wait (while the previous
// kernel still runs): after the wait, only the loads of the vector that the
// previous kernel wrote remain on the critical path.  The first K entries of
// the lane are held; a longer row reads the rest after the wait.  The sums run
// over the entries in the same order as rg_offdiag / rg_csr_sum: the same bits.
// ---------------------------------------------------------------------------
template <int K>
struct HeldEntries {
    int32_t c[K];   // column (or child); -1: none
    float v[K];
    int next, end, stride;   // first entry not held, the row's end, entry stride
};

// This lane's entries of `row` of a sliced-ELL matrix (slice height 32 / G).
template <int G, int K>
__device__ __forceinline__ void hold_ell_row(HeldEntries<K>& h, int row, bool valid, int lane,
                                             const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                             const float* __restrict__ val) {
    constexpr int S = 32 / G;
    int e = 0, end = 0;
    if (valid) {
        const int slice = row / S;
        end = __ldg(sp + slice + 1);
        e = __ldg(sp + slice) + (lane / S) * S + (row - slice * S);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const bool ok = e + 32 * k < end;
        h.c[k] = ok ? __ldg(col + e + 32 * k) : -1;
        h.v[k] = ok ? __ldg(val + e + 32 * k) : 0.f;
    }
    h.next = e + 32 * K;
    h.end = end;
    h.stride = 32;
}

// This lane's entries [beg, end) of a CSR row split across G lanes.
template <int G, int K>
__device__ __forceinline__ void hold_csr_row(HeldEntries<K>& h, bool valid, int lane, int beg, int end,
                                             const int32_t* __restrict__ idx, const float* __restrict__ w) {
    constexpr int S = 32 / G;
    const int q = beg + lane / S;
    if (!valid) end = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const bool ok = q + G * k < end;
        h.c[k] = ok ? __ldg(idx + q + G * k) : -1;
        h.v[k] = ok ? __ldg(w + q + G * k) : 0.f;
    }
    h.next = q + G * K;
    h.end = end;
    h.stride = G;
}

// Sum of v * x[c] over the held entries and the row's tail, reduced over the
// G lanes of the row.  Every lane of the warp must call it.
template <int G, int K, bool kReadOnly = true>
__device__ __forceinline__ float4 held_sum(const HeldEntries<K>& h, int lane, const int32_t* __restrict__ idx,
                                           const float* __restrict__ w, const float4* x) {
    constexpr int S = 32 / G;
    float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (h.c[k] >= 0) {
            const float4 xv = vload<kReadOnly>(x + h.c[k]);
            ax = fmaf(h.v[k], xv.x, ax);
            ay = fmaf(h.v[k], xv.y, ay);
            az = fmaf(h.v[k], xv.z, az);
        }
    }
    for (int e = h.next; e < h.end; e += h.stride) {
        const float a = __ldg(w + e);
        const float4 xv = vload<kReadOnly>(x + __ldg(idx + e));
        ax = fmaf(a, xv.x, ax);
        ay = fmaf(a, xv.y, ay);
        az = fmaf(a, xv.z, az);
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    return make_float4(ax, ay, az, 0.f);
}

constexpr int kHeldL0 = 4;   // level-0 entries held per lane (4 lanes per row: 16 per row)
constexpr int kHeldC = 6;    // coarse-level entries held per lane (8 lanes per row: 48 per row)

// Sum of the contiguous float4 slots [beg, end) split across the G lanes.
template <int G>
__device__ __forceinline__ float4 rg_slot_sum(bool valid, int lane, int beg, int end, const float4* __restrict__ slots) {
    constexpr int S = 32 / G;
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (valid) {
#pragma unroll 2
        for (int q = beg + lane / S; q < end; q += G) {
            const float4 t = __ldg(slots + q);
            ax += t.x;
            ay += t.y;
            az += t.z;
        }
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    return make_float4(ax, ay, az, 0.f);
}

// ---------------------------------------------------------------------------
// Level-0 weighted-Jacobi sweep on the displacement: d' = d + dinv (b - A d).
// With gather != 0 the RHS is assembled first (b = b0 + slots) and stored.
// One warp per 8 rows, 4 lanes per row.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_l0_sweep_rg(int n, const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                                     const float* __restrict__ val, const float* __restrict__ dfull,
                                                     const float* __restrict__ dinv, const float4* __restrict__ din,
                                                     float4* __restrict__ dout, float4* __restrict__ b,
                                                     const float4* __restrict__ b0, const int32_t* __restrict__ slot_ptr,
                                                     const float4* __restrict__ slots, int gather,
                                                     const int32_t* __restrict__ gate = nullptr) {
    pdl_trigger();
    constexpr int G = kLanesL0, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    HeldEntries<kHeldL0> he;
    hold_ell_row<G>(he, row, valid, lane, sp, col, val);
    const int sbeg = (gather && valid) ? __ldg(slot_ptr + row) : 0, send = (gather && valid) ? __ldg(slot_ptr + row + 1) : 0;
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;   // gated launches run only when the learned V-cycle was rejected
    float4 bi;
    if (gather) {
        const float4 sl = rg_slot_sum<G>(valid, lane, sbeg, send, slots);
        const float4 bb = valid ? __ldg(b0 + row) : f4z();
        bi = make_float4(bb.x + sl.x, bb.y + sl.y, bb.z + sl.z, 0.f);
        if (valid && lane < S) b[row] = bi;
    } else {
        bi = valid ? b[row] : f4z();
    }
    const float4 off = held_sum<G>(he, lane, col, val, din);
    if (!valid || lane >= S) return;
    const float4 di4 = __ldg(din + row);
    const float D = __ldg(dfull + row), w = __ldg(dinv + row);
    dout[row] = make_float4(fmaf(w, bi.x - fmaf(D, di4.x, off.x), di4.x), fmaf(w, bi.y - fmaf(D, di4.y, off.y), di4.y),
                            fmaf(w, bi.z - fmaf(D, di4.z, off.z), di4.z), 0.f);
}

// Level-0 residual res = b - A d (used when the coarse kernel does not fuse it).
__global__ void __launch_bounds__(256) k_l0_residual_rg(int n, const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                                        const float* __restrict__ val, const float* __restrict__ dfull,
                                                        const float4* __restrict__ dvec, const float4* __restrict__ b,
                                                        float4* __restrict__ res, const int32_t* __restrict__ gate = nullptr) {
    pdl_trigger();
    constexpr int G = kLanesL0, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    HeldEntries<kHeldL0> he;
    hold_ell_row<G>(he, row, valid, lane, sp, col, val);
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;
    const float4 off = held_sum<G>(he, lane, col, val, dvec);
    if (!valid || lane >= S) return;
    const float4 x = __ldg(dvec + row), bi = __ldg(b + row);
    const float D = __ldg(dfull + row);
    res[row] = make_float4(bi.x - fmaf(D, x.x, off.x), bi.y - fmaf(D, x.y, off.y), bi.z - fmaf(D, x.z, off.z), 0.f);
}

// Level-0 prolongation d += P e1 (used when the coarse kernel does not fuse it).
__global__ void k_l0_prolong(int n, const int4* __restrict__ pid, const float4* __restrict__ pw,
                             const float4* __restrict__ ec, float4* __restrict__ v, const int32_t* __restrict__ gate = nullptr) {
    pdl_enter();
    if (gate && __ldg(gate) == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 id = __ldg(pid + i);
    const float4 w = __ldg(pw + i);
    const float4 e0 = __ldg(ec + id.x), e1 = __ldg(ec + id.y), e2 = __ldg(ec + id.z), e3 = __ldg(ec + id.w);
    float4 vi = v[i];
    vi.x += w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x;
    vi.y += w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y;
    vi.z += w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z;
    v[i] = vi;
}

// ---------------------------------------------------------------------------
// One coarse level as grid-wide kernels (levels below the cluster kernel's
// first level when the hierarchy is split): every body's rows of the level in
// one launch per phase, 8 lanes per row.  Same arithmetic per row as the
// cluster kernel's phases.
// ---------------------------------------------------------------------------

// r = R res_fine (children of each row, CSR); e = dinv r (the first Jacobi
// sweep from zero), or 0 when dinv is null (no pre-smoothing).
__global__ void __launch_bounds__(256) k_lvl_restrict(int n, const int32_t* __restrict__ rptr, const int32_t* __restrict__ rcol,
                                                      const float* __restrict__ rw, const float4* __restrict__ res_fine,
                                                      const float* __restrict__ dinv, float4* __restrict__ r,
                                                      float4* __restrict__ e, const int32_t* __restrict__ gate) {
    pdl_trigger();
    constexpr int G = kLanesC, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    const int beg = valid ? __ldg(rptr + row) : 0, end = valid ? __ldg(rptr + row + 1) : 0;
    HeldEntries<kHeldC> he;
    hold_csr_row<G>(he, valid, lane, beg, end, rcol, rw);
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;
    const float4 s = held_sum<G>(he, lane, rcol, rw, res_fine);
    if (!valid || lane >= S) return;
    r[row] = s;
    const float di = dinv ? __ldg(dinv + row) : 0.f;
    e[row] = make_float4(di * s.x, di * s.y, di * s.z, 0.f);
}

// Level 1's restriction without the level-0 residual: with res0 = b0 - D0 d0 -
// Off0 d0 and RO = R Off0 (precomputed, CSR over level-1 rows),
//     r = R res0 = R (b0 - D0 d0) - RO d0,
// so the level-0 residual launch is not needed (its rows are formed by the
// post-smoothing kernel, k_prolong_sweep, where it needs them).  e = dinv r as
// k_lvl_restrict.  8 lanes per row; children and RO entries held before the wait.
constexpr int kHeldRO = 16;   // RO entries held per lane (128 per row; config 1: ~125)
__global__ void __launch_bounds__(256) k_lvl_restrict_res0(int n, const int32_t* __restrict__ rptr,
                                                           const int32_t* __restrict__ rcol,
                                                           const float* __restrict__ rw,
                                                           const int32_t* __restrict__ roptr,
                                                           const int32_t* __restrict__ rocol,
                                                           const float* __restrict__ roval,
                                                           const float4* __restrict__ b0, const float* __restrict__ dfull0,
                                                           const float4* __restrict__ d0, const float* __restrict__ dinv,
                                                           float4* __restrict__ r, float4* __restrict__ e,
                                                           const int32_t* __restrict__ gate) {
    pdl_trigger();
    constexpr int G = kLanesC, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    const int beg = valid ? __ldg(rptr + row) : 0, end = valid ? __ldg(rptr + row + 1) : 0;
    const int obeg = valid ? __ldg(roptr + row) : 0, oend = valid ? __ldg(roptr + row + 1) : 0;
    HeldEntries<kHeldC> hc;
    hold_csr_row<G>(hc, valid, lane, beg, end, rcol, rw);
    HeldEntries<kHeldRO> ho;
    hold_csr_row<G>(ho, valid, lane, obeg, oend, rocol, roval);
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;
    // R (b0 - D0 d0): this lane's children, in the order of hold_csr_row
    float ax = 0.f, ay = 0.f, az = 0.f;
    auto child = [&](int i, float w) {
        const float4 bb = __ldg(b0 + i), dd = __ldg(d0 + i);
        const float D = __ldg(dfull0 + i);
        ax = fmaf(w, bb.x - D * dd.x, ax);
        ay = fmaf(w, bb.y - D * dd.y, ay);
        az = fmaf(w, bb.z - D * dd.z, az);
    };
#pragma unroll
    for (int k = 0; k < kHeldC; ++k)
        if (hc.c[k] >= 0) child(hc.c[k], hc.v[k]);
    for (int q = hc.next; q < hc.end; q += hc.stride) child(__ldg(rcol + q), __ldg(rw + q));
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    const float4 q = held_sum<G>(ho, lane, rocol, roval, d0);
    if (!valid || lane >= S) return;
    const float4 s = make_float4(ax - q.x, ay - q.y, az - q.z, 0.f);
    r[row] = s;
    const float di = dinv ? __ldg(dinv + row) : 0.f;
    e[row] = make_float4(di * s.x, di * s.y, di * s.z, 0.f);
}

// eout = ein + dinv (r - A ein)
__global__ void __launch_bounds__(256) k_lvl_sweep(int n, const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                                   const float* __restrict__ val, const float* __restrict__ dfull,
                                                   const float* __restrict__ dinv, const float4* __restrict__ r,
                                                   const float4* __restrict__ ein, float4* __restrict__ eout,
                                                   const int32_t* __restrict__ gate) {
    pdl_trigger();
    constexpr int G = kLanesC, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    HeldEntries<kHeldC> he;
    hold_ell_row<G>(he, row, valid, lane, sp, col, val);
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;
    const float4 off = held_sum<G>(he, lane, col, val, ein);
    if (!valid || lane >= S) return;
    const float4 x = __ldg(ein + row), ri = __ldg(r + row);
    const float D = __ldg(dfull + row), w = __ldg(dinv + row);
    eout[row] = make_float4(fmaf(w, ri.x - fmaf(D, x.x, off.x), x.x), fmaf(w, ri.y - fmaf(D, x.y, off.y), x.y),
                            fmaf(w, ri.z - fmaf(D, x.z, off.z), x.z), 0.f);
}

// res = r - A e
__global__ void __launch_bounds__(256) k_lvl_residual(int n, const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                                      const float* __restrict__ val, const float* __restrict__ dfull,
                                                      const float4* __restrict__ r, const float4* __restrict__ e,
                                                      float4* __restrict__ res, const int32_t* __restrict__ gate) {
    pdl_trigger();
    constexpr int G = kLanesC, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    HeldEntries<kHeldC> he;
    hold_ell_row<G>(he, row, valid, lane, sp, col, val);
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;
    const float4 off = held_sum<G>(he, lane, col, val, e);
    if (!valid || lane >= S) return;
    const float4 x = __ldg(e + row), ri = __ldg(r + row);
    const float D = __ldg(dfull + row);
    res[row] = make_float4(ri.x - fmaf(D, x.x, off.x), ri.y - fmaf(D, x.y, off.y), ri.z - fmaf(D, x.z, off.z), 0.f);
}

// dst = cur + P ec (P: 4 coarse parents per row); dst may be cur.
__global__ void k_lvl_prolong(int n, const int4* __restrict__ pid, const float4* __restrict__ pw,
                              const float4* __restrict__ ec, const float4* cur, float4* dst,
                              const int32_t* __restrict__ gate) {
    pdl_enter();
    if (gate && __ldg(gate) == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 id = __ldg(pid + i);
    const float4 w = __ldg(pw + i);
    const float4 e0 = __ldg(ec + id.x), e1 = __ldg(ec + id.y), e2 = __ldg(ec + id.z), e3 = __ldg(ec + id.w);
    float4 v = cur[i];
    v.x += w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x;
    v.y += w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y;
    v.z += w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z;
    dst[i] = v;
}

// ---------------------------------------------------------------------------
// Prolongation fused with the first post-smoothing sweep.  With the level's
// operator A = D + Off, pe = P e_c (this row's 4 parents on the coarser level)
// and OP = Off P precomputed,
//     A (d + pe) = (b - res) + D pe + OP e_c,
// where res = b - A d is the residual the descent already formed, so
//     dout = d + pe + dinv (res - D pe - OP e_c)
// needs no neighbour of the prolonged vector: one launch instead of two.
// G lanes per row over OP's sliced-ELL row; dout may be din.  With ls_r set
// (the learned cycle) the output is instead the post-smoothing residual
// ls_r = fix (res - D pe - OP e_c), and dout = din + pe.  With res null the
// kernel forms its rows of res = b - A din itself (the level's own sliced ELL
// sp0 / col0 / val0, same arithmetic as k_l0_residual_rg): din must then not
// be dout.
// ---------------------------------------------------------------------------
template <int G>
__global__ void __launch_bounds__(256) k_prolong_sweep(int n, const int4* __restrict__ pid, const float4* __restrict__ pw,
                                                       const float4* __restrict__ ec, const int32_t* __restrict__ sp,
                                                       const int32_t* __restrict__ col, const float* __restrict__ val,
                                                       const float* __restrict__ dfull, const float* __restrict__ dinv,
                                                       const float4* __restrict__ res, const float4* din, float4* dout,
                                                       const float* __restrict__ fixf, float4* __restrict__ ls_r,
                                                       const int32_t* __restrict__ gate, const float4* __restrict__ b,
                                                       const int32_t* __restrict__ sp0, const int32_t* __restrict__ col0,
                                                       const float* __restrict__ val0) {
    pdl_trigger();
    constexpr int S = 32 / G;
    const bool form_res = res == nullptr;   // uniform over the launch
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    HeldEntries<G == kLanesL0 ? kHeldL0 : kHeldC> he, ha;
    hold_ell_row<G>(he, row, valid, lane, sp, col, val);
    if (form_res) hold_ell_row<G>(ha, row, valid, lane, sp0, col0, val0);
    const bool own = valid && lane < S;
    const int4 id = own ? __ldg(pid + row) : make_int4(0, 0, 0, 0);
    const float4 w = own ? __ldg(pw + row) : f4z();
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;
    const float4 q = held_sum<G>(he, lane, col, val, ec);
    const float4 offd = form_res ? held_sum<G>(ha, lane, col0, val0, din) : f4z();
    if (!own) return;
    const float4 e0 = __ldg(ec + id.x), e1 = __ldg(ec + id.y), e2 = __ldg(ec + id.z), e3 = __ldg(ec + id.w);
    const float4 pe = make_float4(w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x,
                                  w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y,
                                  w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z, 0.f);
    const float D = __ldg(dfull + row);
    float4 r0;
    if (form_res) {
        const float4 xd = __ldg(din + row), bi = __ldg(b + row);
        r0 = make_float4(bi.x - fmaf(D, xd.x, offd.x), bi.y - fmaf(D, xd.y, offd.y), bi.z - fmaf(D, xd.z, offd.z), 0.f);
    } else {
        r0 = __ldg(res + row);
    }
    const float rx = r0.x - fmaf(D, pe.x, q.x), ry = r0.y - fmaf(D, pe.y, q.y), rz = r0.z - fmaf(D, pe.z, q.z);
    float4 x = din[row];
    x.x += pe.x;
    x.y += pe.y;
    x.z += pe.z;
    if (ls_r) {
        const float fx = __ldg(fixf + row);
        ls_r[row] = make_float4(fx * rx, fx * ry, fx * rz, 0.f);
        dout[row] = x;
    } else {
        const float wi = __ldg(dinv + row);
        dout[row] = make_float4(fmaf(wi, rx, x.x), fmaf(wi, ry, x.y), fmaf(wi, rz, x.z), 0.f);
    }
}

// ---------------------------------------------------------------------------
// Coarse part of the V-cycle, one thread-block cluster per body; phases are
// separated by cluster barriers (release/acquire on global memory).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_coarse_vcycle(const CoarseArgs A) {
    pdl_enter();
    if (A.gate && __ldg(A.gate) == 0) return;   // uniform over the cluster, before any barrier
    cg::cluster_group cluster = cg::this_cluster();
    const int cs = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int body = blockIdx.x / cs;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int warp_c = rank * wpb + (threadIdx.x >> 5);
    const int nwarp = cs * wpb;
    const int tid_c = rank * blockDim.x + threadIdx.x;
    const int nthr = cs * blockDim.x;
    const int L = A.L;
    constexpr int Sc = 32 / kLanesC;
    constexpr int S0 = 32 / kLanesL0;

    // level-0 residual res0 = b - A0 d over this body's rows
    if (A.fuse_l0) {
        const int2 rg = A.range[body * L + 0];
        const LevelView& V0 = A.lv[0];
        for (int base = rg.x + warp_c * S0; base < rg.x + rg.y; base += nwarp * S0) {
            const int row = base + (lane % S0);
            const bool valid = row < rg.x + rg.y;
            const float4 off = rg_offdiag<kLanesL0, false>(row, valid, lane, V0.slice_ptr, V0.col, V0.val, A.d);
            if (valid && lane < S0) {
                const float4 x = A.d[row], bi = __ldg(A.b + row);
                const float D = __ldg(V0.dfull + row);
                V0.res[row] = make_float4(bi.x - fmaf(D, x.x, off.x), bi.y - fmaf(D, x.y, off.y), bi.z - fmaf(D, x.z, off.z), 0.f);
            }
        }
        cluster.sync();
    }
    float4* ecur[kMaxLevels];
    float4* eoth[kMaxLevels];
    // descend
    for (int l = 1; l < L - 1; ++l) {
        const LevelView& C = A.lv[l];
        const int2 rg = A.range[body * L + l];
        ecur[l] = C.e;
        eoth[l] = C.e2;
        for (int base = rg.x + warp_c * Sc; base < rg.x + rg.y; base += nwarp * Sc) {
            const int row = base + (lane % Sc);
            const bool valid = row < rg.x + rg.y;
            const int beg = valid ? __ldg(C.rptr + row) : 0, end = valid ? __ldg(C.rptr + row + 1) : 0;
            const float4 r = rg_csr_sum<kLanesC, false>(valid, lane, beg, end, C.rcol, C.rw, A.lv[l - 1].res);
            if (valid && lane < Sc) {
                C.r[row] = r;
                const float di = A.pre > 0 ? __ldg(C.dinv + row) : 0.f;
                C.e[row] = make_float4(di * r.x, di * r.y, di * r.z, 0.f);
            }
        }
        cluster.sync();
        for (int k = 1; k < A.pre; ++k) {
            for (int base = rg.x + warp_c * Sc; base < rg.x + rg.y; base += nwarp * Sc) {
                const int row = base + (lane % Sc);
                const bool valid = row < rg.x + rg.y;
                const float4 off = rg_offdiag<kLanesC, false>(row, valid, lane, C.slice_ptr, C.col, C.val, ecur[l]);
                if (valid && lane < Sc) {
                    const float4 x = ecur[l][row], ri = C.r[row];
                    const float D = __ldg(C.dfull + row), w = __ldg(C.dinv + row);
                    eoth[l][row] = make_float4(fmaf(w, ri.x - fmaf(D, x.x, off.x), x.x), fmaf(w, ri.y - fmaf(D, x.y, off.y), x.y),
                                               fmaf(w, ri.z - fmaf(D, x.z, off.z), x.z), 0.f);
                }
            }
            float4* t = ecur[l];
            ecur[l] = eoth[l];
            eoth[l] = t;
            cluster.sync();
        }
        for (int base = rg.x + warp_c * Sc; base < rg.x + rg.y; base += nwarp * Sc) {
            const int row = base + (lane % Sc);
            const bool valid = row < rg.x + rg.y;
            const float4 off = rg_offdiag<kLanesC, false>(row, valid, lane, C.slice_ptr, C.col, C.val, ecur[l]);
            if (valid && lane < Sc) {
                const float4 x = ecur[l][row], ri = C.r[row];
                const float D = __ldg(C.dfull + row);
                C.res[row] = make_float4(ri.x - fmaf(D, x.x, off.x), ri.y - fmaf(D, x.y, off.y), ri.z - fmaf(D, x.z, off.z), 0.f);
            }
        }
        cluster.sync();
    }
    // coarsest: restrict, then e = A^-1 r (dense, warp per row)
    {
        const int l = L - 1;
        const LevelView& C = A.lv[l];
        const int2 rg = A.range[body * L + l];
        for (int base = rg.x + warp_c * Sc; base < rg.x + rg.y; base += nwarp * Sc) {
            const int row = base + (lane % Sc);
            const bool valid = row < rg.x + rg.y;
            const int beg = valid ? __ldg(C.rptr + row) : 0, end = valid ? __ldg(C.rptr + row + 1) : 0;
            const float4 r = rg_csr_sum<kLanesC, false>(valid, lane, beg, end, C.rcol, C.rw, A.lv[l - 1].res);
            if (valid && lane < Sc) C.r[row] = r;
        }
        cluster.sync();
        const int n = rg.y;
        const float* Ai = A.Ainv + __ldg(A.dense_off + body);
        for (int i = warp_c; i < n; i += nwarp) {
            float ax = 0.f, ay = 0.f, az = 0.f;
            for (int k = lane; k < n; k += 32) {
                const float a = __ldg(Ai + (size_t)i * n + k);
                const float4 r = C.r[rg.x + k];
                ax = fmaf(a, r.x, ax);
                ay = fmaf(a, r.y, ay);
                az = fmaf(a, r.z, az);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ax += __shfl_xor_sync(0xffffffffu, ax, o);
                ay += __shfl_xor_sync(0xffffffffu, ay, o);
                az += __shfl_xor_sync(0xffffffffu, az, o);
            }
            if (lane == 0) C.e[rg.x + i] = make_float4(ax, ay, az, 0.f);
        }
        ecur[l] = C.e;
        cluster.sync();
    }
    // ascend
    for (int l = L - 2; l >= 1; --l) {
        const LevelView& C = A.lv[l];
        const LevelView& Cc = A.lv[l + 1];
        const int2 rg = A.range[body * L + l];
        for (int row = rg.x + tid_c; row < rg.x + rg.y; row += nthr) {
            const int4 id = __ldg(Cc.pid + row);
            const float4 w = __ldg(Cc.pw + row);
            const float4 e0 = ecur[l + 1][id.x], e1 = ecur[l + 1][id.y], e2 = ecur[l + 1][id.z], e3 = ecur[l + 1][id.w];
            float4 v = ecur[l][row];
            v.x += w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x;
            v.y += w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y;
            v.z += w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z;
            ecur[l][row] = v;
        }
        cluster.sync();
        for (int k = 0; k < A.post; ++k) {
            for (int base = rg.x + warp_c * Sc; base < rg.x + rg.y; base += nwarp * Sc) {
                const int row = base + (lane % Sc);
                const bool valid = row < rg.x + rg.y;
                const float4 off = rg_offdiag<kLanesC, false>(row, valid, lane, C.slice_ptr, C.col, C.val, ecur[l]);
                if (valid && lane < Sc) {
                    const float4 x = ecur[l][row], ri = C.r[row];
                    const float D = __ldg(C.dfull + row), w = __ldg(C.dinv + row);
                    eoth[l][row] = make_float4(fmaf(w, ri.x - fmaf(D, x.x, off.x), x.x), fmaf(w, ri.y - fmaf(D, x.y, off.y), x.y),
                                               fmaf(w, ri.z - fmaf(D, x.z, off.z), x.z), 0.f);
                }
            }
            float4* t = ecur[l];
            ecur[l] = eoth[l];
            eoth[l] = t;
            cluster.sync();
        }
    }
    // level-0 prolongation d += P1 e1
    if (A.fuse_l0) {
        const LevelView& C1 = A.lv[1];
        const int2 rg = A.range[body * L + 0];
        for (int row = rg.x + tid_c; row < rg.x + rg.y; row += nthr) {
            const int4 id = __ldg(C1.pid + row);
            const float4 w = __ldg(C1.pw + row);
            const float4 e0 = ecur[1][id.x], e1 = ecur[1][id.y], e2 = ecur[1][id.z], e3 = ecur[1][id.w];
            float4 v = A.d[row];
            v.x += w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x;
            v.y += w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y;
            v.z += w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z;
            A.d[row] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Coarse part of the V-cycle with every coarse-level vector resident in the
// cluster's distributed shared memory.  CTA `rank` of the body's cluster owns
// rows [rank*B_l, min((rank+1)*B_l, n_l)) of level l (body-local numbering)
// and keeps r, e, e2, res of those rows in its shared memory; a row of
// another CTA is read through the cluster shared-memory window.  Matrix and
// transfer operators stay in global memory (read-only, L2-resident).
// It owns levels F = A.first .. L-1 (F = 1: every coarse level; F > 1: the
// levels below F run as the grid-wide k_lvl_* kernels).  Input: the level
// F-1 residual (global).  Output: the level-F correction (global, lv[F].e)
// for the prolongation kernel of level F-1.
// ---------------------------------------------------------------------------
struct SmemLevel {
    int off, n, B, base;   // first global row, rows, rows per CTA, float4 offset of [r|e|e2|res]
};

__device__ __forceinline__ float4* dsm_ptr(cg::cluster_group& cl, float4* sm, const SmemLevel& q, int vec, int li) {
    const int rank = li / q.B;
    const int loc = li - rank * q.B;
    return cl.map_shared_rank(sm + q.base + vec * q.B + loc, rank);
}

template <int G>
__device__ __forceinline__ float4 rg_offdiag_dsm(cg::cluster_group& cl, float4* sm, const SmemLevel& q, int vec, int row,
                                                 bool valid, int lane, const int32_t* __restrict__ sp,
                                                 const int32_t* __restrict__ col, const float* __restrict__ val) {
    constexpr int S = 32 / G;
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (valid) {
        const int slice = row / S;
        const int beg = __ldg(sp + slice), end = __ldg(sp + slice + 1);
#pragma unroll 4
        for (int e = beg + (lane / S) * S + (row - slice * S); e < end; e += 32) {
            const float a = __ldg(val + e);
            const float4 xv = *dsm_ptr(cl, sm, q, vec, __ldg(col + e) - q.off);
            ax = fmaf(a, xv.x, ax);
            ay = fmaf(a, xv.y, ay);
            az = fmaf(a, xv.z, az);
        }
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    return make_float4(ax, ay, az, 0.f);
}

// Dynamic shared memory (float4 units) the kernel needs for a cluster size
// when it owns levels first..L-1.
__host__ __device__ inline int coarse_smem_float4(const int* nl, int L, int first, int cs, int ncoarsest) {
    int tot = 0;
    for (int l = first; l < L; ++l) tot += 4 * ((nl[l] + cs - 1) / cs);
    return tot + ncoarsest;
}

__global__ void __launch_bounds__(1024) k_coarse_vcycle_dsm(const CoarseArgs A) {
    pdl_enter();
    if (A.gate && __ldg(A.gate) == 0) return;   // uniform over the cluster, before any barrier
    extern __shared__ float4 smv[];
    cg::cluster_group cluster = cg::this_cluster();
    const int cs = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int body = blockIdx.x / cs;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarp = blockDim.x >> 5;
    const int L = A.L;
    constexpr int Sc = 32 / kLanesC;
    constexpr int R = 0, E = 1, E2 = 2, RES = 3;
    const int F = A.first;
    SmemLevel q[kMaxLevels];
    int base = 0;
    for (int l = F; l < L; ++l) {
        const int2 rg = A.range[body * L + l];
        q[l].off = rg.x;
        q[l].n = rg.y;
        q[l].B = (rg.y + cs - 1) / cs;
        q[l].base = base;
        base += 4 * q[l].B;
    }
    float4* rfull = smv + base;   // full coarsest right-hand side (every CTA)
    int ec[kMaxLevels];           // which of E / E2 holds the current correction
    auto first_row = [&](int l) { return rank * q[l].B; };
    auto own_rows = [&](int l) { return max(0, min(q[l].B, q[l].n - rank * q[l].B)); };
    auto loc = [&](int l, int vec, int i) -> float4& { return smv[q[l].base + vec * q[l].B + i]; };

    // ---- descend
    for (int l = F; l < L; ++l) {
        const LevelView& C = A.lv[l];
        const int r0 = first_row(l), cnt = own_rows(l);
        // restriction r = P^T res_{l-1} (level F-1 residual from global memory)
        for (int b0 = warp * Sc; b0 < cnt; b0 += nwarp * Sc) {
            const int li = b0 + (lane % Sc);
            const bool valid = li < cnt;
            const int row = q[l].off + r0 + li;
            const int beg = valid ? __ldg(C.rptr + row) : 0, end = valid ? __ldg(C.rptr + row + 1) : 0;
            float ax = 0.f, ay = 0.f, az = 0.f;
            if (valid) {
#pragma unroll 4
                for (int k = beg + lane / Sc; k < end; k += kLanesC) {
                    const float w = __ldg(C.rw + k);
                    const int ch = __ldg(C.rcol + k);
                    const float4 t = (l == F) ? __ldg(A.lv[l - 1].res + ch) : *dsm_ptr(cluster, smv, q[l - 1], RES, ch - q[l - 1].off);
                    ax = fmaf(w, t.x, ax);
                    ay = fmaf(w, t.y, ay);
                    az = fmaf(w, t.z, az);
                }
            }
#pragma unroll
            for (int o = Sc; o < 32; o <<= 1) {
                ax += __shfl_xor_sync(0xffffffffu, ax, o);
                ay += __shfl_xor_sync(0xffffffffu, ay, o);
                az += __shfl_xor_sync(0xffffffffu, az, o);
            }
            if (valid && lane < Sc) {
                loc(l, R, li) = make_float4(ax, ay, az, 0.f);
                const float di = (l < L - 1 && A.pre > 0) ? __ldg(C.dinv + row) : 0.f;
                loc(l, E, li) = make_float4(di * ax, di * ay, di * az, 0.f);
            }
        }
        ec[l] = E;
        cluster.sync();
        if (l == L - 1) break;
        for (int k = 1; k < A.pre; ++k) {
            const int src = ec[l], dst = (src == E) ? E2 : E;
            for (int b0 = warp * Sc; b0 < cnt; b0 += nwarp * Sc) {
                const int li = b0 + (lane % Sc);
                const bool valid = li < cnt;
                const int row = q[l].off + r0 + li;
                const float4 off = rg_offdiag_dsm<kLanesC>(cluster, smv, q[l], src, row, valid, lane, C.slice_ptr, C.col, C.val);
                if (valid && lane < Sc) {
                    const float4 x = loc(l, src, li), ri = loc(l, R, li);
                    const float D = __ldg(C.dfull + row), w = __ldg(C.dinv + row);
                    loc(l, dst, li) = make_float4(fmaf(w, ri.x - fmaf(D, x.x, off.x), x.x), fmaf(w, ri.y - fmaf(D, x.y, off.y), x.y),
                                                  fmaf(w, ri.z - fmaf(D, x.z, off.z), x.z), 0.f);
                }
            }
            ec[l] = dst;
            cluster.sync();
        }
        for (int b0 = warp * Sc; b0 < cnt; b0 += nwarp * Sc) {
            const int li = b0 + (lane % Sc);
            const bool valid = li < cnt;
            const int row = q[l].off + r0 + li;
            const float4 off = rg_offdiag_dsm<kLanesC>(cluster, smv, q[l], ec[l], row, valid, lane, C.slice_ptr, C.col, C.val);
            if (valid && lane < Sc) {
                const float4 x = loc(l, ec[l], li), ri = loc(l, R, li);
                const float D = __ldg(C.dfull + row);
                loc(l, RES, li) = make_float4(ri.x - fmaf(D, x.x, off.x), ri.y - fmaf(D, x.y, off.y), ri.z - fmaf(D, x.z, off.z), 0.f);
            }
        }
        cluster.sync();
    }
    // ---- coarsest: every CTA gathers the whole right-hand side, then e = A^-1 r for its rows
    {
        const int l = L - 1;
        const int n = q[l].n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) rfull[i] = *dsm_ptr(cluster, smv, q[l], R, i);
        __syncthreads();
        const int r0 = first_row(l), cnt = own_rows(l);
        if (A.Ainv64) {
            // FP64 coarsest solve (mixed precision)
            const double* Ai = A.Ainv64 + __ldg(A.dense_off + body);
            for (int li = warp; li < cnt; li += nwarp) {
                const int i = r0 + li;
                double ax = 0.0, ay = 0.0, az = 0.0;
                for (int k = lane; k < n; k += 32) {
                    const double a = __ldg(Ai + (size_t)i * n + k);
                    const float4 r = rfull[k];
                    ax = fma(a, (double)r.x, ax);
                    ay = fma(a, (double)r.y, ay);
                    az = fma(a, (double)r.z, az);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ax += __shfl_xor_sync(0xffffffffu, ax, o);
                    ay += __shfl_xor_sync(0xffffffffu, ay, o);
                    az += __shfl_xor_sync(0xffffffffu, az, o);
                }
                if (lane == 0) loc(l, E, li) = make_float4((float)ax, (float)ay, (float)az, 0.f);
            }
        } else {
            const float* Ai = A.Ainv + __ldg(A.dense_off + body);
            for (int li = warp; li < cnt; li += nwarp) {
                const int i = r0 + li;
                float ax = 0.f, ay = 0.f, az = 0.f;
                for (int k = lane; k < n; k += 32) {
                    const float a = __ldg(Ai + (size_t)i * n + k);
                    const float4 r = rfull[k];
                    ax = fmaf(a, r.x, ax);
                    ay = fmaf(a, r.y, ay);
                    az = fmaf(a, r.z, az);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ax += __shfl_xor_sync(0xffffffffu, ax, o);
                    ay += __shfl_xor_sync(0xffffffffu, ay, o);
                    az += __shfl_xor_sync(0xffffffffu, az, o);
                }
                if (lane == 0) loc(l, E, li) = make_float4(ax, ay, az, 0.f);
            }
        }
        ec[l] = E;
        cluster.sync();
    }
    // ---- ascend
    for (int l = L - 2; l >= F; --l) {
        const LevelView& C = A.lv[l];
        const LevelView& Cc = A.lv[l + 1];
        const int r0 = first_row(l), cnt = own_rows(l);
        int k0 = 0;
        if (A.fuse_prolong && A.post > 0) {
            // prolongation + first post-sweep from the descent's residual (RES) and OP = Off P:
            // no neighbour of the prolonged vector is read (the same arithmetic as k_prolong_sweep)
            const int src = ec[l], dst = (src == E) ? E2 : E;
            for (int b0 = warp * Sc; b0 < cnt; b0 += nwarp * Sc) {
                const int li = b0 + (lane % Sc);
                const bool valid = li < cnt;
                const int row = q[l].off + r0 + li;
                const float4 qv = rg_offdiag_dsm<kLanesC>(cluster, smv, q[l + 1], ec[l + 1], row, valid, lane,
                                                          C.op_slice_ptr, C.op_col, C.op_val);
                if (valid && lane < Sc) {
                    const int4 id = __ldg(Cc.pid + row);
                    const float4 w = __ldg(Cc.pw + row);
                    const float4 e0 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.x - q[l + 1].off);
                    const float4 e1 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.y - q[l + 1].off);
                    const float4 e2 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.z - q[l + 1].off);
                    const float4 e3 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.w - q[l + 1].off);
                    const float4 pe = make_float4(w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x,
                                                  w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y,
                                                  w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z, 0.f);
                    const float4 r0v = loc(l, RES, li);
                    const float D = __ldg(C.dfull + row), wi = __ldg(C.dinv + row);
                    const float rx = r0v.x - fmaf(D, pe.x, qv.x), ry = r0v.y - fmaf(D, pe.y, qv.y),
                                rz = r0v.z - fmaf(D, pe.z, qv.z);
                    float4 x = loc(l, src, li);
                    x.x += pe.x;
                    x.y += pe.y;
                    x.z += pe.z;
                    loc(l, dst, li) = make_float4(fmaf(wi, rx, x.x), fmaf(wi, ry, x.y), fmaf(wi, rz, x.z), 0.f);
                }
            }
            ec[l] = dst;
            cluster.sync();
            k0 = 1;
        } else {
            for (int li = threadIdx.x; li < cnt; li += blockDim.x) {
                const int row = q[l].off + r0 + li;
                const int4 id = __ldg(Cc.pid + row);
                const float4 w = __ldg(Cc.pw + row);
                const float4 e0 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.x - q[l + 1].off);
                const float4 e1 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.y - q[l + 1].off);
                const float4 e2 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.z - q[l + 1].off);
                const float4 e3 = *dsm_ptr(cluster, smv, q[l + 1], ec[l + 1], id.w - q[l + 1].off);
                float4& v = loc(l, ec[l], li);
                v.x += w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x;
                v.y += w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y;
                v.z += w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z;
            }
            cluster.sync();
        }
        for (int k = k0; k < A.post; ++k) {
            const int src = ec[l], dst = (src == E) ? E2 : E;
            for (int b0 = warp * Sc; b0 < cnt; b0 += nwarp * Sc) {
                const int li = b0 + (lane % Sc);
                const bool valid = li < cnt;
                const int row = q[l].off + r0 + li;
                const float4 off = rg_offdiag_dsm<kLanesC>(cluster, smv, q[l], src, row, valid, lane, C.slice_ptr, C.col, C.val);
                if (valid && lane < Sc) {
                    const float4 x = loc(l, src, li), ri = loc(l, R, li);
                    const float D = __ldg(C.dfull + row), w = __ldg(C.dinv + row);
                    loc(l, dst, li) = make_float4(fmaf(w, ri.x - fmaf(D, x.x, off.x), x.x), fmaf(w, ri.y - fmaf(D, x.y, off.y), x.y),
                                                  fmaf(w, ri.z - fmaf(D, x.z, off.z), x.z), 0.f);
                }
            }
            ec[l] = dst;
            cluster.sync();
        }
    }
    // ---- level-F correction to global memory (own rows only: no remote access after the last barrier)
    {
        const int r0 = first_row(F), cnt = own_rows(F);
        for (int li = threadIdx.x; li < cnt; li += blockDim.x) A.lv[F].e[q[F].off + r0 + li] = loc(F, ec[F], li);
    }
}

// ---------------------------------------------------------------------------
// Coarse part of the V-cycle, levels F = A.first .. L-1 of one body in ONE
// CTA: every vector of those levels in shared memory, phases separated by
// block barriers instead of cluster barriers, no remote loads.  Same lane
// layout (8 lanes per row), per-row arithmetic and summation order as the
// cluster kernel, so the two give the same bits.  Each warp carries
// kCtaRowGroups row groups (4 rows each) at once, so the load chains of
// several rows overlap.  Input: the level F-1 residual (global); output:
// the level-F correction (global, lv[F].e).
// ---------------------------------------------------------------------------
constexpr int kCtaRowGroups = 4;

struct CtaLevel {
    int off, n, base;   // first global row, rows, float4 offset of [r | e | e2 | res] (n each)
};

// Off-diagonal products of P row groups of a coarse sliced-ELL level with x
// in shared memory (body-local index col - off).  Every lane calls it.
template <int P>
__device__ __forceinline__ void cta_offdiag(const int (&row)[P], const bool (&valid)[P], int lane,
                                            const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                            const float* __restrict__ val, const float4* xs, int off,
                                            float4 (&out)[P]) {
    constexpr int S = 32 / kLanesC;
    int e[P], end[P];
    float ax[P], ay[P], az[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        ax[p] = ay[p] = az[p] = 0.f;
        e[p] = end[p] = 0;
        if (valid[p]) {
            const int slice = row[p] / S;
            e[p] = __ldg(sp + slice) + (lane / S) * S + (row[p] - slice * S);
            end[p] = __ldg(sp + slice + 1);
        }
    }
    for (bool more = true; more;) {
        more = false;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            if (e[p] < end[p]) {
                const float a = __ldg(val + e[p]);
                const float4 xv = xs[__ldg(col + e[p]) - off];
                ax[p] = fmaf(a, xv.x, ax[p]);
                ay[p] = fmaf(a, xv.y, ay[p]);
                az[p] = fmaf(a, xv.z, az[p]);
                e[p] += 32;
                more = true;
            }
        }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
        for (int o = S; o < 32; o <<= 1) {
            ax[p] += __shfl_xor_sync(0xffffffffu, ax[p], o);
            ay[p] += __shfl_xor_sync(0xffffffffu, ay[p], o);
            az[p] += __shfl_xor_sync(0xffffffffu, az[p], o);
        }
        out[p] = make_float4(ax[p], ay[p], az[p], 0.f);
    }
}

// Restriction r = sum_k w_k src[child_k - src_off] of P row groups (CSR over
// the finer level's rows, kLanesC lanes per row).  src is the finer level's
// residual in global memory (src_off 0) or in shared memory.
template <int P>
__device__ __forceinline__ void cta_restrict(const int (&row)[P], const bool (&valid)[P], int lane,
                                             const int32_t* __restrict__ rptr, const int32_t* __restrict__ rcol,
                                             const float* __restrict__ rw, const float4* src, int src_off,
                                             float4 (&out)[P]) {
    constexpr int S = 32 / kLanesC;
    int k[P], end[P];
    float ax[P], ay[P], az[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        ax[p] = ay[p] = az[p] = 0.f;
        k[p] = end[p] = 0;
        if (valid[p]) {
            k[p] = __ldg(rptr + row[p]) + lane / S;
            end[p] = __ldg(rptr + row[p] + 1);
        }
    }
    for (bool more = true; more;) {
        more = false;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            if (k[p] < end[p]) {
                const float w = __ldg(rw + k[p]);
                const float4 t = src[__ldg(rcol + k[p]) - src_off];
                ax[p] = fmaf(w, t.x, ax[p]);
                ay[p] = fmaf(w, t.y, ay[p]);
                az[p] = fmaf(w, t.z, az[p]);
                k[p] += kLanesC;
                more = true;
            }
        }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
        for (int o = S; o < 32; o <<= 1) {
            ax[p] += __shfl_xor_sync(0xffffffffu, ax[p], o);
            ay[p] += __shfl_xor_sync(0xffffffffu, ay[p], o);
            az[p] += __shfl_xor_sync(0xffffffffu, az[p], o);
        }
        out[p] = make_float4(ax[p], ay[p], az[p], 0.f);
    }
}

// Shared memory (float4 units) of the one-CTA kernel: 4 vectors of every level it owns.
__host__ __device__ inline int coarse_cta_smem_float4(const int* nl, int L, int first) {
    int tot = 0;
    for (int l = first; l < L; ++l) tot += 4 * nl[l];
    return tot;
}

__global__ void __launch_bounds__(1024) k_coarse_vcycle_cta(const CoarseArgs A) {
    pdl_enter();
    if (A.gate && __ldg(A.gate) == 0) return;
    const int body = blockIdx.x;
    extern __shared__ float4 smv[];
    constexpr int P = kCtaRowGroups;
    constexpr int Sc = 32 / kLanesC;
    constexpr int R = 0, E = 1, E2 = 2, RES = 3;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarp = blockDim.x >> 5;
    const int L = A.L, F = A.first;
    CtaLevel q[kMaxLevels];
    int base = 0;
    for (int l = F; l < L; ++l) {
        const int2 rg = A.range[body * L + l];
        q[l].off = rg.x;
        q[l].n = rg.y;
        q[l].base = base;
        base += 4 * rg.y;
    }
    auto vec = [&](int l, int v) -> float4* { return smv + q[l].base + v * q[l].n; };
    int ec[kMaxLevels];   // which of E / E2 holds the level's current correction

    // One pass of a Jacobi sweep (dst = x + w (r - D x - off)) or of the
    // residual (res = r - D x - off) over level l, P row groups per warp.
    auto sweep_or_residual = [&](int l, int src, int dst, bool residual) {
        const LevelView& C = A.lv[l];
        const int n = q[l].n, off = q[l].off;
        const int ngroups = (n + Sc - 1) / Sc;
        const float4* xs = vec(l, src);
        const float4* r = vec(l, R);
        float4* out = vec(l, dst);
        for (int g0 = warp; g0 < ngroups; g0 += nwarp * P) {
            int li[P], row[P];
            bool valid[P];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                li[p] = (g0 + p * nwarp) * Sc + (lane % Sc);
                valid[p] = li[p] < n;
                row[p] = off + li[p];
            }
            float4 o[P];
            cta_offdiag<P>(row, valid, lane, C.slice_ptr, C.col, C.val, xs, off, o);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                if (!valid[p] || lane >= Sc) continue;
                const float4 x = xs[li[p]], ri = r[li[p]];
                const float D = __ldg(C.dfull + row[p]);
                if (residual) {
                    out[li[p]] = make_float4(ri.x - fmaf(D, x.x, o[p].x), ri.y - fmaf(D, x.y, o[p].y),
                                             ri.z - fmaf(D, x.z, o[p].z), 0.f);
                } else {
                    const float w = __ldg(C.dinv + row[p]);
                    out[li[p]] = make_float4(fmaf(w, ri.x - fmaf(D, x.x, o[p].x), x.x),
                                             fmaf(w, ri.y - fmaf(D, x.y, o[p].y), x.y),
                                             fmaf(w, ri.z - fmaf(D, x.z, o[p].z), x.z), 0.f);
                }
            }
        }
    };

    // ---- descend
    for (int l = F; l < L; ++l) {
        const LevelView& C = A.lv[l];
        const int n = q[l].n, off = q[l].off;
        const int ngroups = (n + Sc - 1) / Sc;
        const float4* src = (l == F) ? A.lv[l - 1].res : vec(l - 1, RES);
        const int src_off = (l == F) ? 0 : q[l - 1].off;
        float4* r = vec(l, R);
        float4* e = vec(l, E);
        for (int g0 = warp; g0 < ngroups; g0 += nwarp * P) {
            int li[P], row[P];
            bool valid[P];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                li[p] = (g0 + p * nwarp) * Sc + (lane % Sc);
                valid[p] = li[p] < n;
                row[p] = off + li[p];
            }
            float4 t[P];
            cta_restrict<P>(row, valid, lane, C.rptr, C.rcol, C.rw, src, src_off, t);
#pragma unroll
            for (int p = 0; p < P; ++p) {
                if (!valid[p] || lane >= Sc) continue;
                r[li[p]] = t[p];
                const float di = (l < L - 1 && A.pre > 0) ? __ldg(C.dinv + row[p]) : 0.f;
                e[li[p]] = make_float4(di * t[p].x, di * t[p].y, di * t[p].z, 0.f);
            }
        }
        ec[l] = E;
        __syncthreads();
        if (l == L - 1) break;
        for (int k = 1; k < A.pre; ++k) {
            const int dst = (ec[l] == E) ? E2 : E;
            sweep_or_residual(l, ec[l], dst, false);
            ec[l] = dst;
            __syncthreads();
        }
        sweep_or_residual(l, ec[l], RES, true);
        __syncthreads();
    }
    // ---- coarsest: e = A^-1 r (dense, warp per row)
    {
        const int l = L - 1;
        const int n = q[l].n;
        const float4* rf = vec(l, R);
        float4* e = vec(l, E);
        if (A.Ainv64) {
            const double* Ai = A.Ainv64 + __ldg(A.dense_off + body);
            for (int i = warp; i < n; i += nwarp) {
                double ax = 0.0, ay = 0.0, az = 0.0;
                for (int k = lane; k < n; k += 32) {
                    const double a = __ldg(Ai + (size_t)i * n + k);
                    const float4 r = rf[k];
                    ax = fma(a, (double)r.x, ax);
                    ay = fma(a, (double)r.y, ay);
                    az = fma(a, (double)r.z, az);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ax += __shfl_xor_sync(0xffffffffu, ax, o);
                    ay += __shfl_xor_sync(0xffffffffu, ay, o);
                    az += __shfl_xor_sync(0xffffffffu, az, o);
                }
                if (lane == 0) e[i] = make_float4((float)ax, (float)ay, (float)az, 0.f);
            }
        } else {
            const float* Ai = A.Ainv + __ldg(A.dense_off + body);
            for (int i = warp; i < n; i += nwarp) {
                float ax = 0.f, ay = 0.f, az = 0.f;
                for (int k = lane; k < n; k += 32) {
                    const float a = __ldg(Ai + (size_t)i * n + k);
                    const float4 r = rf[k];
                    ax = fmaf(a, r.x, ax);
                    ay = fmaf(a, r.y, ay);
                    az = fmaf(a, r.z, az);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ax += __shfl_xor_sync(0xffffffffu, ax, o);
                    ay += __shfl_xor_sync(0xffffffffu, ay, o);
                    az += __shfl_xor_sync(0xffffffffu, az, o);
                }
                if (lane == 0) e[i] = make_float4(ax, ay, az, 0.f);
            }
        }
        ec[l] = E;
        __syncthreads();
    }
    // ---- ascend
    for (int l = L - 2; l >= F; --l) {
        const LevelView& C = A.lv[l];
        const LevelView& Cc = A.lv[l + 1];
        const int n = q[l].n, off = q[l].off, coff = q[l + 1].off;
        const float4* ecs = vec(l + 1, ec[l + 1]);
        int k0 = 0;
        if (A.fuse_prolong && A.post > 0) {
            // prolongation + first post-sweep in one phase (as in the cluster kernel)
            const int dst = (ec[l] == E) ? E2 : E;
            const float4* xs = vec(l, ec[l]);
            const float4* res = vec(l, RES);
            float4* out = vec(l, dst);
            const int ngroups = (n + Sc - 1) / Sc;
            for (int g0 = warp; g0 < ngroups; g0 += nwarp * P) {
                int li[P], row[P];
                bool valid[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    li[p] = (g0 + p * nwarp) * Sc + (lane % Sc);
                    valid[p] = li[p] < n;
                    row[p] = off + li[p];
                }
                float4 o[P];
                cta_offdiag<P>(row, valid, lane, C.op_slice_ptr, C.op_col, C.op_val, ecs, coff, o);
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    if (!valid[p] || lane >= Sc) continue;
                    const int4 id = __ldg(Cc.pid + row[p]);
                    const float4 w = __ldg(Cc.pw + row[p]);
                    const float4 e0 = ecs[id.x - coff], e1 = ecs[id.y - coff], e2 = ecs[id.z - coff],
                                 e3 = ecs[id.w - coff];
                    const float4 pe = make_float4(w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x,
                                                  w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y,
                                                  w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z, 0.f);
                    const float4 r0v = res[li[p]];
                    const float D = __ldg(C.dfull + row[p]), wi = __ldg(C.dinv + row[p]);
                    const float rx = r0v.x - fmaf(D, pe.x, o[p].x), ry = r0v.y - fmaf(D, pe.y, o[p].y),
                                rz = r0v.z - fmaf(D, pe.z, o[p].z);
                    float4 x = xs[li[p]];
                    x.x += pe.x;
                    x.y += pe.y;
                    x.z += pe.z;
                    out[li[p]] = make_float4(fmaf(wi, rx, x.x), fmaf(wi, ry, x.y), fmaf(wi, rz, x.z), 0.f);
                }
            }
            ec[l] = dst;
            __syncthreads();
            k0 = 1;
        } else {
            float4* v = vec(l, ec[l]);
            for (int li = threadIdx.x; li < n; li += blockDim.x) {
                const int row = off + li;
                const int4 id = __ldg(Cc.pid + row);
                const float4 w = __ldg(Cc.pw + row);
                const float4 e0 = ecs[id.x - coff], e1 = ecs[id.y - coff], e2 = ecs[id.z - coff], e3 = ecs[id.w - coff];
                float4 t = v[li];
                t.x += w.x * e0.x + w.y * e1.x + w.z * e2.x + w.w * e3.x;
                t.y += w.x * e0.y + w.y * e1.y + w.z * e2.y + w.w * e3.y;
                t.z += w.x * e0.z + w.y * e1.z + w.z * e2.z + w.w * e3.z;
                v[li] = t;
            }
            __syncthreads();
        }
        for (int k = k0; k < A.post; ++k) {
            const int dst = (ec[l] == E) ? E2 : E;
            sweep_or_residual(l, ec[l], dst, false);
            ec[l] = dst;
            __syncthreads();
        }
    }
    // ---- level-F correction to global memory
    {
        const float4* ef = vec(F, ec[F]);
        for (int li = threadIdx.x; li < q[F].n; li += blockDim.x) A.lv[F].e[q[F].off + li] = ef[li];
    }
}

// ---------------------------------------------------------------------------
// Dense coarse operator (one body): the V-cycle of levels F..L-1 is a linear
// map M of the level-F right-hand side, so it can be formed once per frame
// (after the coarse diagonals and the coarsest inverse are refreshed) and
// applied in every V-cycle as one restriction + one dense product instead of
// the cluster kernel's chain of barrier-separated phases.
//   k_op_*:         the V-cycle applied to the identity, all columns at once
//                   (below), leaves M in a scratch block.
//   k_coarse_apply: every CTA restricts the level-(F-1) residual to the level-F
//                   right-hand side r_F in shared memory and its warps form 16
//                   rows of e_F = M r_F (warp per row, lanes over the columns).
// When F is the coarsest level, M is its inverse itself and nothing is built.
// ---------------------------------------------------------------------------
constexpr int kDenseOpMaxRows = 1024;   // M at most 4 MiB
constexpr int kDenseApplyThreads = 512;
constexpr int kDenseApplyRows = kDenseApplyThreads / 32;   // rows of M per CTA of k_coarse_apply (one per warp)

// ---- the operator built for all columns at once ------------------------------
// M acts on the three components alike, so it is built as a scalar operator:
// the V-cycle of levels F..L-1 applied to the n_F x n_F identity, every level's
// vectors held as n_l x m row-major blocks (m = n_F columns).  One CTA per
// (row, 128 columns), one thread per column; one launch per phase of the V-cycle.
constexpr int kOpThreads = 128;   // columns per CTA: grid (rows, ceil(m / kOpThreads)), thread per column

// R = I (row i: 1 in column i), E = dinv R (the first Jacobi sweep from zero; 0 without dinv).
__global__ void __launch_bounds__(kOpThreads) k_op_init(int n, int m, const float* __restrict__ dinv,
                                                       float* __restrict__ R, float* __restrict__ E) {
    pdl_enter();
    const int i = blockIdx.x, c = blockIdx.y * blockDim.x + threadIdx.x;
    if (i >= n || c >= m) return;
    const float di = dinv ? __ldg(dinv + i) : 0.f;
    R[(size_t)i * m + c] = c == i ? 1.f : 0.f;
    E[(size_t)i * m + c] = c == i ? di : 0.f;
}

// The sweep, restriction and prolongation kernels stage the row's static
// structure (ELL or CSR entries, parents and weights, uploaded once at set-up)
// before the dependency wait, so that after it every load of the previous
// phase's block is independent of the others.
constexpr int kOpMaxEntries = 64;   // entries of one row staged in shared memory; longer rows take a tail loop

// residual == 0: Xout = Xin + dinv (R - D Xin - Off Xin); residual != 0: Xout = R - D Xin - Off Xin.
// Level of slice height 32 / kLanesC (coarse levels), off-diagonal sliced ELL.
__global__ void __launch_bounds__(kOpThreads) k_op_sweep(int n, int m, const int32_t* __restrict__ sp,
                                                        const int32_t* __restrict__ col,
                                                        const float* __restrict__ val,
                                                        const float* __restrict__ dfull,
                                                        const float* __restrict__ dinv, const float* __restrict__ R,
                                                        const float* __restrict__ Xin, float* __restrict__ Xout,
                                                        int residual) {
    pdl_trigger();
    constexpr int S = 32 / kLanesC;
    __shared__ int32_t scol[kOpMaxEntries];
    __shared__ float sval[kOpMaxEntries];
    const int i = blockIdx.x, c = blockIdx.y * blockDim.x + threadIdx.x;
    if (i >= n) return;   // CTA-uniform
    const int slice = i / S;
    const int e0 = __ldg(sp + slice) + (i - slice * S), e1 = __ldg(sp + slice + 1);
    const int cnt = (e1 - e0 + S - 1) / S, staged = min(cnt, kOpMaxEntries);
    for (int t = threadIdx.x; t < staged; t += blockDim.x) {
        scol[t] = __ldg(col + e0 + t * S);
        sval[t] = __ldg(val + e0 + t * S);
    }
    __syncthreads();
    pdl_wait();
    if (c >= m) return;
    float acc = 0.f;
#pragma unroll 16
    for (int t = 0; t < staged; ++t) acc = fmaf(sval[t], Xin[(size_t)scol[t] * m + c], acc);
    for (int e = e0 + kOpMaxEntries * S; e < e1; e += S) acc = fmaf(__ldg(val + e), Xin[(size_t)__ldg(col + e) * m + c], acc);
    const float x = Xin[(size_t)i * m + c];
    const float r = R[(size_t)i * m + c] - fmaf(__ldg(dfull + i), x, acc);
    Xout[(size_t)i * m + c] = residual ? r : fmaf(__ldg(dinv + i), r, x);
}

// Rc = restriction of Resf (children of each coarse row, CSR); Ec = dinv Rc (0 without dinv).
__global__ void __launch_bounds__(kOpThreads) k_op_restrict(int n, int m, const int32_t* __restrict__ rptr,
                                                           const int32_t* __restrict__ rcol,
                                                           const float* __restrict__ rw,
                                                           const float* __restrict__ Resf,
                                                           const float* __restrict__ dinv, float* __restrict__ Rc,
                                                           float* __restrict__ Ec) {
    pdl_trigger();
    __shared__ int32_t scol[kOpMaxEntries];
    __shared__ float sw[kOpMaxEntries];
    const int i = blockIdx.x, c = blockIdx.y * blockDim.x + threadIdx.x;
    if (i >= n) return;   // CTA-uniform
    const int k0 = __ldg(rptr + i), k1 = __ldg(rptr + i + 1);
    const int staged = min(k1 - k0, kOpMaxEntries);
    for (int t = threadIdx.x; t < staged; t += blockDim.x) {
        scol[t] = __ldg(rcol + k0 + t);
        sw[t] = __ldg(rw + k0 + t);
    }
    __syncthreads();
    pdl_wait();
    if (c >= m) return;
    float acc = 0.f;
#pragma unroll 16
    for (int t = 0; t < staged; ++t) acc = fmaf(sw[t], Resf[(size_t)scol[t] * m + c], acc);
    for (int k = k0 + kOpMaxEntries; k < k1; ++k) acc = fmaf(__ldg(rw + k), Resf[(size_t)__ldg(rcol + k) * m + c], acc);
    Rc[(size_t)i * m + c] = acc;
    Ec[(size_t)i * m + c] = (dinv ? __ldg(dinv + i) : 0.f) * acc;
}

// Coarsest level: E = Ainv R (n x n dense inverse of the one body times the
// n x m block; T = double for the FP64 inverse of the mixed kind).  A CTA forms
// a 4-row x 64-column tile of E: its 4 rows of Ainv staged in shared memory,
// the k range split over 4 thread groups (a column per thread, coalesced rows
// of R), the 4 partial sums added in shared memory.
constexpr int kOpcRows = 4, kOpcCols = 64, kOpcSplit = 4, kOpcThreads = kOpcCols * kOpcSplit;
template <typename T>
__global__ void __launch_bounds__(kOpcThreads) k_op_coarsest(int n, int m, const T* __restrict__ Ainv,
                                                            const float* __restrict__ R, float* __restrict__ E) {
    pdl_enter();
    __shared__ T As[kOpcRows][kDenseOpMaxRows];
    __shared__ T part[kOpcSplit - 1][kOpcRows][kOpcCols];
    const int i0 = blockIdx.x * kOpcRows, c0 = blockIdx.y * kOpcCols;
    const int tc = threadIdx.x % kOpcCols, kq = threadIdx.x / kOpcCols;
    for (int t = threadIdx.x; t < kOpcRows * n; t += kOpcThreads) {
        const int r = t / n, k = t - r * n;
        As[r][k] = i0 + r < n ? Ainv[(size_t)(i0 + r) * n + k] : T(0);
    }
    __syncthreads();
    const int c = c0 + tc;
    const int kb = kq * n / kOpcSplit, ke = (kq + 1) * n / kOpcSplit;
    T acc[kOpcRows];
#pragma unroll
    for (int j = 0; j < kOpcRows; ++j) acc[j] = T(0);
    if (c < m) {
#pragma unroll 12
        for (int k = kb; k < ke; ++k) {
            const T r = (T)R[(size_t)k * m + c];
#pragma unroll
            for (int j = 0; j < kOpcRows; ++j) acc[j] = fma(As[j][k], r, acc[j]);
        }
    }
    if (kq > 0)
#pragma unroll
        for (int j = 0; j < kOpcRows; ++j) part[kq - 1][j][tc] = acc[j];
    __syncthreads();
    if (kq != 0 || c >= m) return;
#pragma unroll
    for (int j = 0; j < kOpcRows; ++j) {
        T v = acc[j];
#pragma unroll
        for (int q = 0; q < kOpcSplit - 1; ++q) v += part[q][j][tc];
        if (i0 + j < n) E[(size_t)(i0 + j) * m + c] = (float)v;
    }
}

// Ef += P Ec (4 coarse parents per fine row).
__global__ void __launch_bounds__(kOpThreads) k_op_prolong(int n, int m, const int4* __restrict__ pid,
                                                          const float4* __restrict__ pw, const float* __restrict__ Ec,
                                                          float* __restrict__ Ef) {
    pdl_trigger();
    const int i = blockIdx.x, c = blockIdx.y * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 id = __ldg(pid + i);
    const float4 w = __ldg(pw + i);
    pdl_wait();
    if (c >= m) return;
    Ef[(size_t)i * m + c] += w.x * Ec[(size_t)id.x * m + c] + w.y * Ec[(size_t)id.y * m + c] +
                             w.z * Ec[(size_t)id.z * m + c] + w.w * Ec[(size_t)id.w * m + c];
}

// FP64 inverse of the coarsest level rounded to FP32: the operator when the
// dense part is the coarsest solve alone.
__global__ void __launch_bounds__(256) k_op_round(int count, const double* __restrict__ src, float* __restrict__ dst) {
    pdl_enter();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) dst[i] = (float)src[i];
}

// e_F = M r_F, r_F the restriction of the level-(F-1) residual (children of
// each level-F row, CSR).  One row of M per warp; CTAs in clusters of
// kApplyCluster.  The CTAs of a cluster split r_F: rank k forms rows
// [k c, (k+1) c), c = ceil(n_F / kApplyCluster), kApplyG lanes per row, its
// children and weights held in registers before the dependency wait and the
// children's residual rows read straight from global memory after it; after a
// cluster barrier every CTA gathers all of r_F from the cluster's shared
// memory (distributed shared memory), and a second barrier keeps every share
// alive until all reads are done.  Each warp fetches its row of M while the
// restriction runs.
constexpr int kApplyG = 4;         // lanes per restricted row
constexpr int kApplyK = 4;         // children per lane held in registers (16 per row; longer rows: tail loop)
constexpr int kApplyMRegs = 16;    // entries of the warp's row of M per lane held in registers
constexpr int kApplyCluster = 8;   // CTAs per cluster (portable size)
static_assert(kDenseOpMaxRows <= kApplyCluster * (kDenseApplyThreads / kApplyG),
              "a CTA restricts at most one row per lane group");

__host__ __device__ constexpr int coarse_apply_chunk(int nf) { return (nf + kApplyCluster - 1) / kApplyCluster; }
__host__ __device__ constexpr size_t coarse_apply_smem_bytes(int nf) {
    return (size_t)(nf + coarse_apply_chunk(nf)) * sizeof(float4);
}
// CTAs of one launch: one per kDenseApplyRows rows of M, rounded up to whole clusters
__host__ __device__ constexpr int coarse_apply_ctas(int nf) {
    return ((nf + kDenseApplyRows - 1) / kDenseApplyRows + kApplyCluster - 1) / kApplyCluster * kApplyCluster;
}

__global__ void __launch_bounds__(kDenseApplyThreads, 1) k_coarse_apply(int nf, const int32_t* __restrict__ rptr,
                                                                       const int32_t* __restrict__ rcol,
                                                                       const float* __restrict__ rw,
                                                                       const float4* __restrict__ res_fine,
                                                                       const float* __restrict__ M,
                                                                       float4* __restrict__ e,
                                                                       const int32_t* __restrict__ gate) {
    pdl_trigger();
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ float4 apply_smem[];
    const int chunk = coarse_apply_chunk(nf);
    float4* rs = apply_smem;          // r_F, nf rows (gathered)
    float4* mine = apply_smem + nf;   // this CTA's share of r_F, chunk rows
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sub = tid % kApplyG, rloc = tid / kApplyG;
    const int row = (int)cluster.block_rank() * chunk + rloc;
    const bool valid = rloc < chunk && row < nf;
    // static structure (written once at set-up): safe before the wait
    const int beg = valid ? __ldg(rptr + row) : 0, end = valid ? __ldg(rptr + row + 1) : 0;
    int cc[kApplyK];
    float cw[kApplyK];
#pragma unroll
    for (int k = 0; k < kApplyK; ++k) {
        const int q = beg + sub + k * kApplyG;
        cc[k] = q < end ? __ldg(rcol + q) : -1;
        cw[k] = q < end ? __ldg(rw + q) : 0.f;
    }
    pdl_wait();
    if (gate && __ldg(gate) == 0) return;   // uniform over the launch: every CTA of the cluster leaves
    const int i = blockIdx.x * kDenseApplyRows + warp;   // this warp's row of M
    float mr[kApplyMRegs];
#pragma unroll
    for (int j = 0; j < kApplyMRegs; ++j) {
        const int k = lane + 32 * j;
        mr[j] = (i < nf && k < nf) ? __ldg(M + (size_t)i * nf + k) : 0.f;
    }
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < kApplyK; ++k)
        if (cc[k] >= 0) acc = f4fma(cw[k], __ldg(res_fine + cc[k]), acc);
    for (int q = beg + sub + kApplyK * kApplyG; q < end; q += kApplyG)
        acc = f4fma(__ldg(rw + q), __ldg(res_fine + __ldg(rcol + q)), acc);
#pragma unroll
    for (int o = 1; o < kApplyG; o <<= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
    }
    if (sub == 0 && valid) mine[rloc] = acc;
    cluster.sync();   // every share written and visible to the cluster
    for (int r = tid; r < nf; r += kDenseApplyThreads) {
        const int owner = r / chunk;
        rs[r] = *cluster.map_shared_rank(mine + (r - owner * chunk), owner);
    }
    cluster.sync();   // r_F complete here; no share is read after this point
    if (i >= nf) return;   // warp-uniform
    float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
    for (int j = 0; j < kApplyMRegs; ++j) {
        const int k = lane + 32 * j;
        if (k < nf) {
            const float4 t = rs[k];
            ax = fmaf(mr[j], t.x, ax);
            ay = fmaf(mr[j], t.y, ay);
            az = fmaf(mr[j], t.z, az);
        }
    }
    for (int k = lane + 32 * kApplyMRegs; k < nf; k += 32) {
        const float a = __ldg(M + (size_t)i * nf + k);
        const float4 t = rs[k];
        ax = fmaf(a, t.x, ax);
        ay = fmaf(a, t.y, ay);
        az = fmaf(a, t.z, az);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    if (lane == 0) e[i] = make_float4(ax, ay, az, 0.f);
}

// ---------------------------------------------------------------------------
// Coarsest level: explicit inverse of A = A0 + diag(c) per body, refreshed
// only when the lumped contact stiffness c changed.  A0^-1 = B0 is computed
// once at set-up; with k coarsest vertices in contact (K = {i : c_i != 0}) the
// inverse follows from the Woodbury identity
//     A^-1 = B0 - U S^-1 U^T,   U = B0[:, K],   S = diag(1/c_K) + B0[K, K],
// an n*n*k update instead of a fresh O(n^3) factorisation.  Above
// kWoodburyMaxRank contacts it falls back to Cholesky + explicit inverse of A.
// One CTA of 1024 threads per body; T = float or double.
// ---------------------------------------------------------------------------
constexpr int kWoodburyMaxRank = 64;

// Shared memory (elements of T) either path needs for an n x n block.
__host__ __device__ inline size_t coarsest_smem_elems(int n) {
    const size_t k = (size_t)(n < kWoodburyMaxRank ? n : kWoodburyMaxRank);
    const size_t refactor = (size_t)n * n + n;
    const size_t woodbury = 2 * k * n + k * k;
    return refactor > woodbury ? refactor : woodbury;
}

// Cholesky (right-looking, L_jj on the diagonal), X = L^-1 in place row by
// row, then A^-1 = X^T X.
template <typename T>
__device__ void coarsest_refactor(int n, const T* __restrict__ A, const float* __restrict__ c, T* __restrict__ Ai,
                                  T* sm) {
    T* M = sm;            // n*n
    T* tmp = sm + n * n;  // n
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int i = q / n, j = q - i * n;
        T a = A[q];
        if (i == j) a += (T)c[i];
        M[q] = a;
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        const T d = sqrt(M[j * n + j]);
        const T id = T(1) / d;
        __syncthreads();
        if (threadIdx.x == 0) M[j * n + j] = d;
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) M[i * n + j] *= id;
        __syncthreads();
        const int m = n - j - 1;
        const int tot = m * (m + 1) / 2;
        for (int q = threadIdx.x; q < tot; q += blockDim.x) {
            int a = (int)((sqrtf(8.f * (float)q + 1.f) - 1.f) * 0.5f);
            while ((a + 1) * (a + 2) / 2 <= q) ++a;
            while (a * (a + 1) / 2 > q) --a;
            const int bcol = q - a * (a + 1) / 2;
            const int i = j + 1 + a, k = j + 1 + bcol;
            M[i * n + k] -= M[i * n + j] * M[k * n + j];
        }
        __syncthreads();
    }
    // X_ii = 1/L_ii, X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = 0; i < n; ++i) {
        const T xii = T(1) / M[i * n + i];
        for (int j = wid; j < i; j += nw) {
            T s = 0;
            for (int k = j + lane; k < i; k += 32) s = fma(M[i * n + k], M[k * n + j], s);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) tmp[j] = -xii * s;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < i; j += blockDim.x) M[i * n + j] = tmp[j];
        if (threadIdx.x == 0) M[i * n + i] = xii;
        __syncthreads();
    }
    // A^-1 = X^T X: (i, j) = sum_{k >= max(i,j)} X_ki X_kj
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int i = q / n, j = q - i * n;
        const int k0 = i > j ? i : j;
        T s = 0;
        for (int k = k0; k < n; ++k) s = fma(M[k * n + i], M[k * n + j], s);
        Ai[q] = s;
    }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarsest_update(const int2* __restrict__ range, int L,
                                                          const int32_t* __restrict__ dense_off,
                                                          const T* __restrict__ A0, const T* __restrict__ B0,
                                                          const float* __restrict__ c, float* __restrict__ c_prev,
                                                          T* __restrict__ Ainv, int32_t* __restrict__ valid) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T* sm = reinterpret_cast<T*>(sm_raw);
    __shared__ int changed, k;
    __shared__ int K[kWoodburyMaxRank];
    const int2 rg = range[blockIdx.x * L + (L - 1)];
    const int n = rg.y, off = rg.x;
    const T* A = A0 + dense_off[blockIdx.x];
    const T* B = B0 + dense_off[blockIdx.x];
    T* Ai = Ainv + dense_off[blockIdx.x];
    const float* cb = c + off;
    if (threadIdx.x == 0) changed = valid[blockIdx.x] ? 0 : 1;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (cb[i] != c_prev[off + i]) changed = 1;
    __syncthreads();
    if (!changed) return;
    // K in ascending order: warp 0 compacts 32 rows at a time with a ballot
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int cnt = 0;
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            const bool hit = i < n && cb[i] != 0.f;
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            const int pos = cnt + __popc(m & ((1u << lane) - 1u));
            if (hit && pos < kWoodburyMaxRank) K[pos] = i;
            cnt += __popc(m);
        }
        if (lane == 0) k = cnt;
    }
    __syncthreads();
    const int kk = k;
    if (kk > kWoodburyMaxRank) {
        coarsest_refactor<T>(n, A, cb, Ai, sm);
    } else if (kk == 0) {
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) Ai[q] = B[q];
    } else {
        T* Ut = sm;                 // kk x n: rows K of B0 (= columns, B0 symmetric)
        T* W = sm + kk * n;         // kk x n: S^-1 Ut
        T* S = sm + 2 * kk * n;     // kk x kk
        for (int q = threadIdx.x; q < kk * n; q += blockDim.x) {
            const int a = q / n, i = q - a * n;
            Ut[q] = B[K[a] * n + i];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < kk * kk; q += blockDim.x) {
            const int a = q / kk, b = q - a * kk;
            T v = Ut[a * n + K[b]];
            if (a == b) v += T(1) / (T)cb[K[a]];
            S[q] = v;
        }
        __syncthreads();
        // Cholesky of S in one warp (lower triangle, L_jj on the diagonal)
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            for (int j = 0; j < kk; ++j) {
                const T d = sqrt(S[j * kk + j]);
                __syncwarp();
                for (int i = j + 1 + lane; i < kk; i += 32) S[i * kk + j] /= d;
                __syncwarp();
                if (lane == 0) S[j * kk + j] = d;
                for (int i = j + 1 + lane; i < kk; i += 32) {
                    const T lij = S[i * kk + j];
                    for (int l = j + 1; l <= i; ++l) S[i * kk + l] -= lij * S[l * kk + j];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // W[:, i] = S^-1 Ut[:, i]: forward then backward substitution, one column per thread
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            for (int a = 0; a < kk; ++a) {
                T s = Ut[a * n + i];
                for (int b = 0; b < a; ++b) s -= S[a * kk + b] * W[b * n + i];
                W[a * n + i] = s / S[a * kk + a];
            }
            for (int a = kk - 1; a >= 0; --a) {
                T s = W[a * n + i];
                for (int b = a + 1; b < kk; ++b) s -= S[b * kk + a] * W[b * n + i];
                W[a * n + i] = s / S[a * kk + a];
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int i = q / n, j = q - i * n;
            T s = B[q];
            for (int a = 0; a < kk; ++a) s -= Ut[a * n + i] * W[a * n + j];
            Ai[q] = s;
        }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) c_prev[off + i] = cb[i];
    if (threadIdx.x == 0) valid[blockIdx.x] = 1;
}

}  // namespace mgsb
