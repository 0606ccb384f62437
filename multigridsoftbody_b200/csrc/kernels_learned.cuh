// Level-0 kernels of the learned smoother (the network itself is in
// kernels_mlp.cuh).  A learned sweep is
//     features(r) -> MLP -> d += (s_i / D_i) * MLP(x_i)
// with, per vertex i (4 lanes per row over the sliced-ELL level-0 matrix):
//     rbar_i = sum_j |a_ij| r_j / sum_j |a_ij|        (1-ring mean residual, coupling weighted)
//     dring_i = sum_j |a_ij| D_j / sum_j |a_ij|       (1-ring mean diagonal)
//     s_i = sqrt(|r_i|^2 + |rbar_i|^2)
//     x_i = [r_i / s_i (3), D_i / sum_j |a_ij|, (D_i - L_ii) / D_i, D_i / dring_i, rbar_i / s_i (3)]
// D_i = L_ii + c_i is the diagonal with this frame's contact stiffness.  Fixed
// vertices take no update and count as zero residual for their neighbours.
// Normalising by s_i makes the sweep homogeneous of degree 1 in r, like a
// linear smoother.
#pragma once

#include <cstdint>

#include "kernels_mg.cuh"
#include "kernels_mlp.cuh"

namespace mgsb {
namespace {

constexpr int kLsThreads = 256;
constexpr int kLsRowsPerBlock = kLsThreads / kLanesL0;   // 64 rows per block

// r = fix * (b - A d) on level 0; optionally dsave = d and part[block] = sum |r|^2.
// With slots set, b is first assembled as b0 + the row's RHS slots and stored
// to bgather (the right-hand side of the PD iteration, reused afterwards).
__global__ void __launch_bounds__(kLsThreads) k_ls_residual(int n, const int32_t* __restrict__ sp,
                                                            const int32_t* __restrict__ col, const float* __restrict__ val,
                                                            const float* __restrict__ dfull, const float* __restrict__ fixf,
                                                            const float4* __restrict__ d, const float4* __restrict__ b,
                                                            float4* __restrict__ r, float4* __restrict__ dsave,
                                                            float* __restrict__ part, const float4* __restrict__ b0 = nullptr,
                                                            const int32_t* __restrict__ slot_ptr = nullptr,
                                                            const float4* __restrict__ slots = nullptr,
                                                            float4* __restrict__ bgather = nullptr) {
    pdl_enter();
    __shared__ float red[kLsThreads / 32];
    constexpr int G = kLanesL0, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    float4 bg = make_float4(0.f, 0.f, 0.f, 0.f);
    if (slots) {
        const int beg = valid ? __ldg(slot_ptr + row) : 0, end = valid ? __ldg(slot_ptr + row + 1) : 0;
        const float4 sl = rg_slot_sum<G>(valid, lane, beg, end, slots);
        const float4 bb = valid ? __ldg(b0 + row) : make_float4(0.f, 0.f, 0.f, 0.f);
        bg = make_float4(bb.x + sl.x, bb.y + sl.y, bb.z + sl.z, 0.f);
        if (valid && lane < S) bgather[row] = bg;
    }
    const float4 off = rg_offdiag<G, false>(row, valid, lane, sp, col, val, d);
    float rr = 0.f;
    if (valid && lane < S) {
        const float4 x = d[row], bi = slots ? bg : b[row];
        const float D = __ldg(dfull + row), fx = __ldg(fixf + row);
        const float4 q = make_float4(fx * (bi.x - fmaf(D, x.x, off.x)), fx * (bi.y - fmaf(D, x.y, off.y)),
                                     fx * (bi.z - fmaf(D, x.z, off.z)), 0.f);
        if (r) r[row] = q;
        if (dsave) dsave[row] = x;
        rr = q.x * q.x + q.y * q.y + q.z * q.z;
    }
    if (part) {
        const float t = block_sum_f(rr, red);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}

// Features and update scale of one row from its 1-ring sums
// (sum |a| f_j r_j, sum |a|, sum |a| D_j).
__device__ __forceinline__ float ls_row_features(int row, float sx, float sy, float sz, float sa, float sd,
                                                 const float* __restrict__ dfull, const float* __restrict__ diag0,
                                                 const float* __restrict__ fixf, const float4* __restrict__ r,
                                                 float (&f)[kMlpIn]) {
    const float fx = __ldg(fixf + row);
    const float4 ri = r[row];
    const float rx = fx * ri.x, ry = fx * ri.y, rz = fx * ri.z;
    const float inv_a = sa > 0.f ? 1.f / sa : 0.f;
    const float bx = sx * inv_a, by = sy * inv_a, bz = sz * inv_a;
    const float D = __ldg(dfull + row), L = __ldg(diag0 + row);
    const float s = sqrtf(rx * rx + ry * ry + rz * rz + bx * bx + by * by + bz * bz);
    const float is = s > 0.f ? 1.f / s : 0.f;
    f[0] = rx * is;
    f[1] = ry * is;
    f[2] = rz * is;
    f[3] = D * inv_a;
    f[4] = (D - L) / D;
    f[5] = sd > 0.f ? D * sa / sd : 1.f;
    f[6] = bx * is;
    f[7] = by * is;
    f[8] = bz * is;
    return (fx != 0.f && s > 0.f) ? s / D : 0.f;
}

// 16 BF16 features (9 used) of one row into a K-major interleaved tile.
__device__ __forceinline__ void ls_store_tile_row(uint8_t* tile, int row_in_tile, const float (&f)[kMlpIn]) {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float lo = 2 * i < kMlpIn ? f[2 * i] : 0.f;
        const float hi = 2 * i + 1 < kMlpIn ? f[2 * i + 1] : 0.f;
        const __nv_bfloat162 two = __floats2bfloat162_rn(lo, hi);
        w[i] = *reinterpret_cast<const uint32_t*>(&two);
    }
    uint8_t* base = tile + interleaved_offset(row_in_tile, 0, kMlpInPad);
    *reinterpret_cast<uint4*>(base) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4*>(base + 128) = make_uint4(w[4], w[5], w[6], w[7]);
}

// Features of every row into the BF16 tensor-core tiles and the update scale
// s_i / D_i (0 for fixed vertices or a zero residual); optionally the FP32
// features row-major into xf[n][9].  4 lanes per row.
__global__ void __launch_bounds__(kLsThreads) k_ls_features(int n, const int32_t* __restrict__ sp,
                                                            const int32_t* __restrict__ col, const float* __restrict__ val,
                                                            const float* __restrict__ dfull, const float* __restrict__ diag0,
                                                            const float* __restrict__ fixf, const float4* __restrict__ r,
                                                            uint8_t* __restrict__ tiles, float* __restrict__ scale,
                                                            float* __restrict__ xf) {
    pdl_enter();
    constexpr int G = kLanesL0, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    float sx = 0.f, sy = 0.f, sz = 0.f, sa = 0.f, sd = 0.f;
    if (valid) {
        const int slice = row / S;
        const int beg = __ldg(sp + slice), end = __ldg(sp + slice + 1);
        for (int e = beg + (lane / S) * S + (row - slice * S); e < end; e += 32) {
            const float a = fabsf(__ldg(val + e));
            const int j = __ldg(col + e);
            const float4 rj = r[j];
            const float fj = __ldg(fixf + j);
            sx = fmaf(a * fj, rj.x, sx);
            sy = fmaf(a * fj, rj.y, sy);
            sz = fmaf(a * fj, rj.z, sz);
            sa += a;
            sd = fmaf(a, __ldg(dfull + j), sd);
        }
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
    }
    if (!valid || lane >= S) return;
    float f[kMlpIn];
    scale[row] = ls_row_features(row, sx, sy, sz, sa, sd, dfull, diag0, fixf, r, f);
    if (tiles) ls_store_tile_row(tiles + (size_t)(row / kMlpTile) * kTileBytes, row % kMlpTile, f);
    if (xf)
        for (int k = 0; k < kMlpIn; ++k) xf[(size_t)row * kMlpIn + k] = f[k];
}

// Per-frame row constants of the learned sweep's features, from this frame's
// diagonal D (contacts included): rc_i = (D_i / sa_i, (D_i - L_ii) / D_i,
// D_i sa_i / sd_i, 1 / sa_i) with sa_i = sum_j |a_ij| and sd_i = sum_j |a_ij| D_j
// over the level-0 off-diagonal row (4 lanes per row).  The sweep then needs
// only |a_ij| r_j from each neighbour.
__global__ void __launch_bounds__(kLsThreads) k_ls_row_consts(int n, const int32_t* __restrict__ sp,
                                                              const int32_t* __restrict__ col,
                                                              const float* __restrict__ val,
                                                              const float* __restrict__ dfull,
                                                              const float* __restrict__ diag0, float4* __restrict__ rc) {
    pdl_trigger();
    constexpr int G = kLanesL0, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    // the row's entries and its contact-free diagonal are set-up data: loaded before the wait
    HeldEntries<kHeldL0> he;
    hold_ell_row<G>(he, row, valid, lane, sp, col, val);
    const float L = (valid && lane < S) ? __ldg(diag0 + row) : 0.f;
    pdl_wait();
    float sa = 0.f, sd = 0.f;   // the entries in the order of the row's ELL loop
#pragma unroll
    for (int k = 0; k < kHeldL0; ++k) {
        if (he.c[k] >= 0) {
            const float a = fabsf(he.v[k]);
            sa += a;
            sd = fmaf(a, __ldg(dfull + he.c[k]), sd);
        }
    }
    for (int e = he.next; e < he.end; e += he.stride) {
        const float a = fabsf(__ldg(val + e));
        sa += a;
        sd = fmaf(a, __ldg(dfull + __ldg(col + e)), sd);
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
    }
    if (!valid || lane >= S) return;
    const float D = __ldg(dfull + row);
    const float inv_a = sa > 0.f ? 1.f / sa : 0.f;
    rc[row] = make_float4(D * inv_a, (D - L) / D, sd > 0.f ? D * sa / sd : 1.f, inv_a);
}

// Rows of the residual window of a 128-row tile that the learned sweep stages in
// shared memory: [win.x, win.y) holds the tile's rows and every column of their
// sliced-ELL entries (padding included); win.x == win.y: no window (gather from
// global memory).
constexpr int kLsWinRows = 3072;   // 48 KiB of float4
constexpr int kLsPerThread = 8;    // ELL entries a thread loads ahead (2 threads per row: rows up to 16 wide)

// Dynamic shared memory of k_ls_sweep_tc: the MLP's operands and barriers, then
// the residual window; at least 80 KiB (two CTAs per SM at most, so that
// tcgen05.alloc never waits).
inline size_t ls_sweep_smem_bytes() {
    const size_t b = ((sizeof(MlpSmem) + 127) / 128) * 128 + (size_t)kLsWinRows * sizeof(float4);
    return b > 80 * 1024 ? b : (size_t)80 * 1024;
}

// One learned sweep in a single kernel: per 128-row tile, each thread forms its
// row's features straight into the shared-memory operand tile, the tensor-core
// MLP runs on the tile, and the same thread applies d_i += (s_i/D_i) y_i.
// With dd64 set (the mixed kind's last sweep of a V-cycle whose residual check
// is taken by the next outer residual), the finished correction is also applied
// to the FP64 displacement, dd64_i += d_i, with its FP32 mirror d32_i: each row
// belongs to one thread, so this is the work of k_mx_update for that row.
// With din set the sweep reads the iterate from din and writes every row of d
// (d = din + update): the post-smoothing kernel before it then leaves din intact
// while it reads its neighbours.
__global__ void __launch_bounds__(kMlpThreads) k_ls_sweep_tc(int n, int ntiles, const int32_t* __restrict__ sp,
                                                             const int32_t* __restrict__ col, const float* __restrict__ val,
                                                             const float* __restrict__ dfull,
                                                             const float4* __restrict__ rc, const int2* __restrict__ win,
                                                             const float* __restrict__ fixf, const float4* __restrict__ r,
                                                             const uint8_t* __restrict__ img, float4* __restrict__ d,
                                                             int32_t* __restrict__ err, double4* __restrict__ dd64,
                                                             float4* __restrict__ d32, const float4* __restrict__ din) {
    pdl_trigger();
    constexpr int S = 32 / kLanesL0;   // level-0 slice height
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    MlpSmem& Sm = *reinterpret_cast<MlpSmem*>(smem_raw);
    float4* rwin = reinterpret_cast<float4*>(smem_raw + ((sizeof(MlpSmem) + 127) / 128) * 128);
    WaitState ws;
    uint32_t ph_load = 0, ph_mma = 0, ph_win = 0;
    // Prologue before the wait for the previous kernel: TMEM, barriers and the
    // weight copy (the weight image is not written by any kernel of a frame);
    // the copy also overlaps the first tile's feature gather.
    const uint32_t tmem = mlp_cta_setup(Sm, img, ws, ph_load, err, false);
    const int rt = threadIdx.x & (kMlpTile - 1), half = threadIdx.x >> 7;   // 2 threads per row
    // The tile's set-up structure (its residual window, this thread's ELL entries of the row -- the
    // two threads of a row take alternate entries -- and the row's fix flag) is written by no kernel:
    // the first tile's is loaded before the dependency wait, while the previous kernel runs.
    int2 wv = make_int2(0, 0);
    int e0 = 0, end = 0;
    int jc[kLsPerThread];
    float av[kLsPerThread];
    float fxr = 0.f;
    auto load_structure = [&](int tile) {
        wv = __ldg(win + tile);
        const int row = tile * kMlpTile + rt;
        e0 = end = 0;
        if (row < n) {
            const int slice = row / S;
            end = __ldg(sp + slice + 1);
            e0 = __ldg(sp + slice) + (row - slice * S) + half * S;
        }
#pragma unroll
        for (int k = 0; k < kLsPerThread; ++k) {
            const int e = e0 + k * 2 * S;
            const bool ok = e < end;
            jc[k] = ok ? __ldg(col + e) : -1;
            av[k] = ok ? fabsf(__ldg(val + e)) : 0.f;
        }
        fxr = (!half && row < n) ? __ldg(fixf + row) : 0.f;
    };
    if ((int)blockIdx.x < ntiles) load_structure(blockIdx.x);
    pdl_wait();
    bool weights_pending = true;
    __shared__ float part[3][kMlpTile];   // second half's 1-ring sums
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if (tile != (int)blockIdx.x) load_structure(tile);
        __syncthreads();
        if (Sm.stop) break;
        const bool use_win = wv.y > wv.x;
        if (use_win && threadIdx.x == 0) {   // the residual rows this tile reads, in one bulk copy
            mbar_expect_tx(&Sm.bar_win, (uint32_t)(wv.y - wv.x) * 16u);
            bulk_g2s(rwin, r + wv.x, (uint32_t)(wv.y - wv.x) * 16u, &Sm.bar_win);
        }
        const int row = tile * kMlpTile + rt;
        // the row's own data (its feature constants, diagonal, displacement) does not depend on the
        // window: loaded now, so that its latency overlaps the window copy
        float4 rcv = make_float4(0.f, 0.f, 0.f, 0.f), dq = make_float4(0.f, 0.f, 0.f, 0.f);
        float Dr = 1.f;
        double4 dv = make_double4(0.0, 0.0, 0.0, 0.0);
        if (!half && row < n) {
            rcv = __ldg(rc + row);
            Dr = __ldg(dfull + row);
            dq = din ? din[row] : d[row];
            if (dd64) dv = dd64[row];
        }
        bool win_ok = true;
        if (use_win) {
            win_ok = wait_bar(ws, &Sm.bar_win, ph_win);
            ph_win ^= 1;
            if (!win_ok) {
                Sm.stop = 1;
                if (err) atomicExch(err, 1);
            }
        }
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (win_ok) {
#pragma unroll
            for (int k = 0; k < kLsPerThread; ++k) {
                if (jc[k] >= 0) {
                    const float4 rj = use_win ? rwin[jc[k] - wv.x] : r[jc[k]];
                    sx = fmaf(av[k], rj.x, sx);
                    sy = fmaf(av[k], rj.y, sy);
                    sz = fmaf(av[k], rj.z, sz);
                }
            }
            for (int e = e0 + kLsPerThread * 2 * S; e < end; e += 2 * S) {   // rows wider than 2 x kLsPerThread
                const float a = fabsf(__ldg(val + e));
                const int j = __ldg(col + e);
                const float4 rj = use_win ? rwin[j - wv.x] : r[j];
                sx = fmaf(a, rj.x, sx);
                sy = fmaf(a, rj.y, sy);
                sz = fmaf(a, rj.z, sz);
            }
        }
        if (half) {
            part[0][rt] = sx;
            part[1][rt] = sy;
            part[2][rt] = sz;
        }
        __syncthreads();
        float sc = 0.f;
        if (!half) {
            float f[kMlpIn];
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) f[k] = 0.f;
            if (row < n && win_ok) {
                // r is zero at fixed vertices (every producer of the sweep's residual applies the fix mask)
                const float4 ri = use_win ? rwin[row - wv.x] : r[row];
                const float4 c = rcv;
                const float bx = (sx + part[0][rt]) * c.w, by = (sy + part[1][rt]) * c.w, bz = (sz + part[2][rt]) * c.w;
                const float s = sqrtf(ri.x * ri.x + ri.y * ri.y + ri.z * ri.z + bx * bx + by * by + bz * bz);
                const float is = s > 0.f ? 1.f / s : 0.f;
                f[0] = ri.x * is;
                f[1] = ri.y * is;
                f[2] = ri.z * is;
                f[3] = c.x;
                f[4] = c.y;
                f[5] = c.z;
                f[6] = bx * is;
                f[7] = by * is;
                f[8] = bz * is;
                sc = (fxr != 0.f && s > 0.f) ? s / Dr : 0.f;
            }
            ls_store_tile_row(Sm.x, rt, f);
        }
        fence_async_shared();
        tc_fence_before();
        __syncthreads();
        bool wok = true;
        if (weights_pending) {
            wok = mlp_wait_weights(Sm, ws, ph_load, err);
            weights_pending = false;
        }
        float out[3];
        const bool ok = mlp_tile_layers(Sm, tmem, ph_mma, ws, wok, out);
        if (!ok) {
            Sm.stop = 1;
            if (err) atomicExch(err, 1);
        }
        // threads 0..127 hold row rt's outputs (warps 0-3 serve TMEM lanes 0..127)
        if (ok && !half && row < n && (sc != 0.f || dd64 || din)) {
            float4 q = dq;
            if (sc != 0.f) {
                q.x += sc * out[0];
                q.y += sc * out[1];
                q.z += sc * out[2];
            }
            if (sc != 0.f || din) d[row] = q;
            if (dd64) {
                double4 v = dv;
                v.x += q.x;
                v.y += q.y;
                v.z += q.z;
                dd64[row] = v;
                d32[row] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
            }
        }
    }
    if (weights_pending) mlp_wait_weights(Sm, ws, ph_load, err);   // no copy may outlive the CTA
    mlp_cta_teardown(Sm, tmem, ws);
}

// Residual check of the learned V-cycles.  Cycle c of the frame passes when
// |r_after|^2 <= gamma^2 |r_before|^2 (both finite), r_after = fix (b - A d)
// after the cycle; the block sums of |r_before|^2 are part0_all[c * nblk +
// block] (written where the cycle started), those of |r_after|^2 are written
// here to part1_all[c * nblk + block].  The decision waits for the frame's
// last check (final != 0): its last block to finish (atomic ticket) sums
// every cycle's partials (one warp per cycle, fixed order), sets gate[0] = 1
// when some cycle failed (the frame's global solve is then repeated with the
// plain V-cycle), counts (stats[0] += cycles, stats[1] += failed cycles),
// in a CUDA graph sets the condition of the IF node that holds that solve
// (use_cond != 0), and resets the ticket for the next launch.
// With dd64 set (mixed precision) the kernel also applies the correction d to
// the FP64 displacement (dd64 += d) and writes its FP32 mirror d32, the work
// of k_mx_update.  kSetCond: the instance that can set a conditional handle
// (only the last check of a graph frame; profilers skip such kernels).
template <bool kSetCond>
__global__ void __launch_bounds__(kLsThreads) k_ls_guard_residual(
    int n, const int32_t* __restrict__ sp, const int32_t* __restrict__ col, const float* __restrict__ val,
    const float* __restrict__ dfull, const float* __restrict__ fixf, const float4* __restrict__ d,
    const float4* __restrict__ b, int cycle, int final, const float* __restrict__ part0_all, float* __restrict__ part1_all,
    float gamma2, int32_t* __restrict__ gate, unsigned long long* __restrict__ stats, cudaGraphConditionalHandle cond,
    int use_cond, unsigned int* __restrict__ ticket, double4* __restrict__ dd64, float4* __restrict__ d32) {
    pdl_enter();
    __shared__ float red[kLsThreads / 32];
    __shared__ bool last;
    __shared__ int fails;
    constexpr int G = kLanesL0, S = 32 / G;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * S + (lane % S);
    const bool valid = row < n;
    const int nblk = gridDim.x;
    const float4 off = rg_offdiag<G, false>(row, valid, lane, sp, col, val, d);
    float rr = 0.f;
    if (valid && lane < S) {
        const float4 x = d[row], bi = b[row];
        const float Dg = __ldg(dfull + row), fx = __ldg(fixf + row);
        const float qx = fx * (bi.x - fmaf(Dg, x.x, off.x)), qy = fx * (bi.y - fmaf(Dg, x.y, off.y)),
                    qz = fx * (bi.z - fmaf(Dg, x.z, off.z));
        rr = qx * qx + qy * qy + qz * qz;
        if (dd64) {
            double4 v = dd64[row];
            v.x += x.x;
            v.y += x.y;
            v.z += x.z;
            dd64[row] = v;
            d32[row] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
        }
    }
    const float t = block_sum_f(rr, red);
    if (threadIdx.x == 0) {
        part1_all[(size_t)cycle * nblk + blockIdx.x] = t;
        if (final) {
            __threadfence();
            last = atomicAdd(ticket, 1u) == gridDim.x - 1;
            fails = 0;
        }
    }
    if (!final) return;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int wl = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c = wl; c <= cycle; c += nw) {
        float a = 0.f, q = 0.f;
        for (int i = lane; i < nblk; i += 32) {
            a += part0_all[(size_t)c * nblk + i];
            q += part1_all[(size_t)c * nblk + i];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            q += __shfl_xor_sync(0xffffffffu, q, o);
        }
        if (lane == 0 && !(isfinite(a) && isfinite(q) && q <= gamma2 * a)) atomicAdd(&fails, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int fail = fails > 0 ? 1 : 0;
        gate[0] = fail;
        if constexpr (kSetCond) {
            if (use_cond) cudaGraphSetConditional(cond, (unsigned)fail);
        }
        stats[0] += (unsigned long long)(cycle + 1);
        stats[1] += (unsigned long long)fails;
        *ticket = 0u;
    }
}

// Copy of the fallback solve's result into the frame's displacement buffer.
__global__ void k_ls_copy(int n, const float4* __restrict__ src, float4* __restrict__ dst) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = src[i];
}

// Training targets in the network's output space: t_i = (e*_i - ec_i) / scale_i
// for rows with scale_i > 0 (mask_i = 1), else mask_i = 0.
// Also snorm_i = s_i (the residual scale of the row) for the host-side filter.
__global__ void k_ls_targets(int n, const float* __restrict__ scale, const float* __restrict__ dfull,
                             const float4* __restrict__ estar, const float4* __restrict__ ecoarse, float* __restrict__ t,
                             uint8_t* __restrict__ mask, float* __restrict__ snorm) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float s = scale[i];
    snorm[i] = s * dfull[i];
    const float4 a = estar[i], c = ecoarse[i];
    const bool ok = s > 0.f;
    const float is = ok ? 1.f / s : 0.f;
    t[3 * (size_t)i] = (a.x - c.x) * is;
    t[3 * (size_t)i + 1] = (a.y - c.y) * is;
    t[3 * (size_t)i + 2] = (a.z - c.z) * is;
    mask[i] = ok ? 1 : 0;
}

}  // namespace
}  // namespace mgsb
