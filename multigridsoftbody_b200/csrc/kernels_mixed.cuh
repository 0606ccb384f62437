// Mixed-precision multigrid frame (sm_100a).  Included by solver.cu only.
//
// FP64: positions, velocities, prediction s, displacement d = x - s, the
// right-hand side and the outer residual r = b - A d (level-0 matrix in FP64),
// the coarsest factor and solve.  FP32: the local step (on FP32 mirrors of s
// and d) and the V-cycle that computes each correction e ~= A^-1 r.
// Every PD iteration runs `refinement_passes` FP64-residual / FP32-correction
// passes (iterative refinement).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels_mg.cuh"

namespace mgsb {

__device__ __forceinline__ double4 d4z() { return make_double4(0.0, 0.0, 0.0, 0.0); }

// Prediction in FP64 (same form as calculateST): last = x; v = v*damp*fix + g*dt*fix;
// x = s = x + v*dt*fix.  FP32 mirrors s32 (local step) and x32 (readback).
__global__ void k_mx_predict(int n, double4* __restrict__ x, double4* __restrict__ v, double4* __restrict__ s,
                             double4* __restrict__ last, float4* __restrict__ s32, float4* __restrict__ x32,
                             const float* __restrict__ fixf, const int32_t* __restrict__ body_of,
                             const BodyDev* __restrict__ bodies, double dt) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BodyDev& B = bodies[__ldg(body_of + i)];
    double4 p = x[i], vel = v[i];
    last[i] = p;
    const double fix = __ldg(fixf + i);
    const double damp = B.damping;
    vel.x *= damp * fix; vel.y *= damp * fix; vel.z *= damp * fix;
    vel.x += (double)B.gravity[0] * dt * fix; vel.y += (double)B.gravity[1] * dt * fix; vel.z += (double)B.gravity[2] * dt * fix;
    p.x += vel.x * dt * fix; p.y += vel.y * dt * fix; p.z += vel.z * dt * fix;
    p.w = 0.0;
    x[i] = p;
    v[i] = vel;
    s[i] = p;
    const float4 f = make_float4((float)p.x, (float)p.y, (float)p.z, 0.f);
    s32[i] = f;
    x32[i] = f;
}

__device__ __forceinline__ void capsule_test64(const double4 sp, const BodyDev& B, int& flag, double4& target) {
    flag = 0;
    target = d4z();
    const double r = B.cap_r;
    if (!(r > 0.0)) return;
    const double p[3] = {sp.x, sp.y, sp.z};
    const double a[3] = {B.cap_a[0], B.cap_a[1], B.cap_a[2]}, b[3] = {B.cap_b[0], B.cap_b[1], B.cap_b[2]};
    const double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    double t = 0.0;
    if (l2 > 0.0) {
        t = ((p[0] - a[0]) * ab[0] + (p[1] - a[1]) * ab[1] + (p[2] - a[2]) * ab[2]) / l2;
        t = fmin(1.0, fmax(0.0, t));
    }
    const double q[3] = {a[0] + t * ab[0], a[1] + t * ab[1], a[2] + t * ab[2]};
    const double dv[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
    const double d = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    if (!(d < r)) return;
    double nrm[3] = {0.0, 0.0, 1.0};
    if (d > 1e-12) {
        nrm[0] = dv[0] / d; nrm[1] = dv[1] / d; nrm[2] = dv[2] / d;
    }
    flag = 1;
    target = make_double4(q[0] + r * nrm[0], q[1] + r * nrm[1], q[2] + r * nrm[2], 0.0);
}

// Contact on the FP64 prediction; b0 = c (p - s) in FP64; D, dinv (FP32, for
// the correction V-cycle); d = 0 in both precisions.  With cand set (the
// broad phase ran), only the surface vertices it flagged are tested.
__global__ void k_mx_contact_frame(int n, const double4* __restrict__ s, const float* __restrict__ fixf,
                                   const int32_t* __restrict__ body_of, const BodyDev* __restrict__ bodies,
                                   const uint8_t* __restrict__ is_surf, const uint8_t* __restrict__ cand, float kc,
                                   const float* __restrict__ diag0,
                                   float omega, int32_t* __restrict__ cflag, float* __restrict__ c0,
                                   double4* __restrict__ b0, float* __restrict__ dfull, float* __restrict__ dinv,
                                   double4* __restrict__ d64, float4* __restrict__ d32, float4* __restrict__ target,
                                   const int32_t* __restrict__ vt_ptr = nullptr,
                                   const int32_t* __restrict__ vt_idx = nullptr,
                                   const double4* __restrict__ push = nullptr) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int flag = 0;
    double4 tg = d4z();
    const double4 sv = s[i];
    if (__ldg(is_surf + i) && (!cand || cand[i])) capsule_test64(sv, bodies[__ldg(body_of + i)], flag, tg);
    Dv3 mp;   // triangle contact (vt_ptr set): s + the mean push of the touching surface triangles
    if (!flag && vt_ptr && tri_contact_gather(i, vt_ptr, vt_idx, push, mp)) {
        flag = 1;
        tg = make_double4(sv.x + mp.x, sv.y + mp.y, sv.z + mp.z, 0.0);
    }
    const bool free_v = __ldg(fixf + i) != 0.f;
    const float c = (flag && free_v) ? kc : 0.f;
    cflag[i] = flag;
    c0[i] = c;
    target[i] = make_float4((float)tg.x, (float)tg.y, (float)tg.z, 0.f);
    b0[i] = c != 0.f ? make_double4((double)c * (tg.x - sv.x), (double)c * (tg.y - sv.y), (double)c * (tg.z - sv.z), 0.0) : d4z();
    const float D = __ldg(diag0 + i) + c;
    dfull[i] = D;
    dinv[i] = free_v ? omega / D : 0.f;
    d64[i] = d4z();
    d32[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Outer FP64 residual r = b - A d with A = diag + c + off-diagonal (FP64
// values; c = this frame's contact stiffness), stored as FP32 for the correction V-cycle, fused with its first Jacobi
// sweep from a zero guess: e = dinv r.  G lanes per row (kLanesMx), 64
// rows per block (64 * G threads), so the blocks cover the rows the
// level-0 kernels' 256-thread blocks cover.
// With b0 set, b is first assembled as b0 + the row's slots (FP64, the slots
// split over the row's lanes; the first pass of a PD iteration) and stored.  With ls_r set (the
// learned V-cycle, which starts from zero), also ls_r = fix * r and
// part[block] = sum |ls_r|^2: the starting residual of that cycle.  With
// part_end set, the previous learned cycle's residual check rides on this
// product: its correction is already in d (the cycle's last sweep applied it),
// so its end residual is fix * (b_prev - A d) with b_prev the right-hand side
// before this kernel's assembly (the same b when nothing is assembled), and
// part_end[block] = sum |fix * (b_prev - A d)|^2.
constexpr int kLanesMx = 4;
constexpr int kMxThreads = 64 * kLanesMx;
__global__ void __launch_bounds__(kMxThreads, 3) k_mx_residual(int n, const int32_t* __restrict__ sp, const int32_t* __restrict__ col,
                                                     const double* __restrict__ val, const double* __restrict__ diag64,
                                                     const float* __restrict__ c, const double4* __restrict__ d, double4* __restrict__ b,
                                                     const float* __restrict__ dinv, float4* __restrict__ r32,
                                                     float4* __restrict__ e, int first_sweep,
                                                     const double4* __restrict__ b0, const int32_t* __restrict__ slot_ptr,
                                                     const float4* __restrict__ slots, const float* __restrict__ fixf,
                                                     float4* __restrict__ ls_r, float* __restrict__ part,
                                                     float* __restrict__ part_end) {
    pdl_trigger();
    __shared__ float red[kMxThreads / 32];
    constexpr int G = kLanesMx, RW = 32 / G;   // lanes per row, rows per warp
    constexpr int SH = 32 / kLanesL0;           // slice height of the level-0 sliced ELL
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int row = warp * RW + (lane % RW);
    const int j = lane / RW;                    // this lane's share of the row
    const bool valid = row < n;
    // Every load whose address is known is issued before the first sum: the row's slots (up to
    // kMxSlotsAhead per lane) and its ELL entries (up to kMxEllAhead per lane), then the neighbour
    // displacements; the sums then run in the order of the plain loops (same bits).  Rows with more
    // entries finish in the tail loops.  The set-up structure (slot and ELL offsets, columns, FP64
    // values, the contact-free diagonal, the fix mask) is written by no kernel: it is loaded before
    // the dependency wait, while the previous kernel runs.
    constexpr int kMxSlotsAhead = 6, kMxEllAhead = 4;
    int s_beg = 0, s_end = 0, q0 = 0, end = 0;
    if (valid) {
        if (b0) {
            s_beg = __ldg(slot_ptr + row) + j;
            s_end = __ldg(slot_ptr + row + 1);
        }
        const int slice = row / SH;
        q0 = __ldg(sp + slice) + j * SH + (row - slice * SH);
        end = __ldg(sp + slice + 1);
    }
    int cj[kMxEllAhead];
    double av[kMxEllAhead];
#pragma unroll
    for (int k = 0; k < kMxEllAhead; ++k) {
        const int q = q0 + k * G * SH;
        const bool ok = q < end;
        cj[k] = ok ? __ldg(col + q) : -1;
        av[k] = ok ? __ldg(val + q) : 0.0;
    }
    const bool own = valid && lane < RW;
    const double D0 = own ? __ldg(diag64 + row) : 0.0;
    const float fxown = own ? __ldg(fixf + row) : 0.f;
    pdl_wait();
    float4 sl[kMxSlotsAhead];
    if (b0) {
#pragma unroll
        for (int k = 0; k < kMxSlotsAhead; ++k) {
            const int q = s_beg + k * G;
            sl[k] = q < s_end ? __ldg(slots + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    // the row's own data, on the row's first lane
    const double4 xown = own ? d[row] : d4z();
    const double Down = own ? D0 + (double)__ldg(c + row) : 0.0;
    const float wown = (own && first_sweep) ? __ldg(dinv + row) : 0.f;
    double4 bi = d4z(), bprev = d4z();
    if (b0) {   // uniform over the block: the row's slots split over its G lanes, FP64 sums
        double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
        for (int k = 0; k < kMxSlotsAhead; ++k) {
            if (s_beg + k * G < s_end) {
                sx += sl[k].x;
                sy += sl[k].y;
                sz += sl[k].z;
            }
        }
        for (int q = s_beg + kMxSlotsAhead * G; q < s_end; q += G) {
            const float4 t = __ldg(slots + q);
            sx += t.x;
            sy += t.y;
            sz += t.z;
        }
#pragma unroll
        for (int o = RW; o < 32; o <<= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o);
        }
        if (valid && lane < RW) {
            if (part_end) bprev = b[row];   // the previous iteration's right-hand side, before it is replaced
            bi = b0[row];
            bi.x += sx;
            bi.y += sy;
            bi.z += sz;
            b[row] = bi;
        }
    }
    double ax = 0.0, ay = 0.0, az = 0.0;
#pragma unroll
    for (int k = 0; k < kMxEllAhead; ++k) {
        if (cj[k] >= 0) {
            const double4 xv = d[cj[k]];
            ax = fma(av[k], xv.x, ax);
            ay = fma(av[k], xv.y, ay);
            az = fma(av[k], xv.z, az);
        }
    }
    for (int q = q0 + kMxEllAhead * G * SH; q < end; q += G * SH) {
        const double a = __ldg(val + q);
        const double4 xv = d[__ldg(col + q)];
        ax = fma(a, xv.x, ax);
        ay = fma(a, xv.y, ay);
        az = fma(a, xv.z, az);
    }
#pragma unroll
    for (int o = RW; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    float rr = 0.f, re = 0.f;
    if (own) {
        const double4 x = xown;
        if (!b0) bi = b[row];
        const double D = Down;
        const float rx = (float)(bi.x - fma(D, x.x, ax)), ry = (float)(bi.y - fma(D, x.y, ay)), rz = (float)(bi.z - fma(D, x.z, az));
        if (part_end) {
            const float fx = fxown;
            const float ex = b0 ? fx * (float)(bprev.x - fma(D, x.x, ax)) : fx * rx;
            const float ey = b0 ? fx * (float)(bprev.y - fma(D, x.y, ay)) : fx * ry;
            const float ez = b0 ? fx * (float)(bprev.z - fma(D, x.z, az)) : fx * rz;
            re = ex * ex + ey * ey + ez * ez;
        }
        r32[row] = make_float4(rx, ry, rz, 0.f);
        const float w = wown;
        e[row] = make_float4(w * rx, w * ry, w * rz, 0.f);
        if (ls_r) {
            const float fx = fxown;
            const float4 q = make_float4(fx * rx, fx * ry, fx * rz, 0.f);
            ls_r[row] = q;
            rr = q.x * q.x + q.y * q.y + q.z * q.z;
        }
    }
    if (ls_r) {   // uniform over the block
        const float t = block_sum_f(rr, red);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
    if (part_end) {   // uniform over the block
        __syncthreads();   // red is reused
        const float t = block_sum_f(re, red);
        if (threadIdx.x == 0) part_end[blockIdx.x] = t;
    }
}

// d += e (FP64), FP32 mirror for the local step.
__global__ void k_mx_update(int n, const float4* __restrict__ e, double4* __restrict__ d, float4* __restrict__ d32) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c = __ldg(e + i);
    double4 v = d[i];
    v.x += c.x;
    v.y += c.y;
    v.z += c.z;
    d[i] = v;
    d32[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
}

// x = s + d, v = v_predicted + d/dt (FP64); FP32 mirror; finiteness check.
__global__ void k_mx_finish(int n, const double4* __restrict__ s, const double4* __restrict__ d, double4* __restrict__ x,
                            double4* __restrict__ v, float4* __restrict__ x32, double inv_dt, int32_t* __restrict__ nonfinite) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 sv = s[i], dv = d[i];
    double4 vel = v[i];
    const double4 p = make_double4(sv.x + dv.x, sv.y + dv.y, sv.z + dv.z, 0.0);
    vel.x += dv.x * inv_dt;
    vel.y += dv.y * inv_dt;
    vel.z += dv.z * inv_dt;
    x[i] = p;
    v[i] = vel;
    x32[i] = make_float4((float)p.x, (float)p.y, (float)p.z, 0.f);
    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) atomicOr(nonfinite, 1);
}


}  // namespace mgsb
