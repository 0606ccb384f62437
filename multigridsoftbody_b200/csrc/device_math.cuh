// Device math shared by the solver kernels (sm_100a, FP32).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace mgsb {

// Programmatic dependent launch: allow the next kernel of the stream to be
// scheduled now (its blocks become resident and wait), then wait until the
// previous kernel has completed and its writes are visible.  Every kernel
// that the solver launches with the programmatic-serialization attribute
// calls this before touching global memory; without the attribute both
// instructions return at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// The two halves, for a kernel with a prologue that touches nothing the
// previous kernels write (it runs between them).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, 0.f); }
__device__ __forceinline__ float4 f4sub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, 0.f); }
__device__ __forceinline__ float4 f4scale(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, 0.f); }
__device__ __forceinline__ float4 f4fma(float s, float4 a, float4 b) {
    return make_float4(fmaf(s, a.x, b.x), fmaf(s, a.y, b.y), fmaf(s, a.z, b.z), 0.f);
}

// ---------------------------------------------------------------------------
// Reference polar decomposition (invariant / Cayley-Hamilton form) as used by
// the reference's accelerated local step, getTetFRV2 (PDSolverAc.cu:447-596),
// equivalently GetRotation_D (utils.cu:123-226).  Row-major F, R.  Returns R;
// the failure branches leave R = I exactly like the reference.  The mixed
// float/double promotions of the reference source are reproduced.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ref_rotation(const float F[9], float R[9]) {
    const float F00 = F[0], F01 = F[1], F02 = F[2], F10 = F[3], F11 = F[4], F12 = F[5], F20 = F[6], F21 = F[7],
                F22 = F[8];
    R[0] = 1.f; R[1] = 0.f; R[2] = 0.f;
    R[3] = 0.f; R[4] = 1.f; R[5] = 0.f;
    R[6] = 0.f; R[7] = 0.f; R[8] = 1.f;
    const float det = F00 * F11 * F22 + F01 * F12 * F20 + F10 * F21 * F02 - F02 * F11 * F20 - F01 * F10 * F22 -
                      F00 * F12 * F21;
    const float III_c = det * det;
    float C[9];
    C[0] = F00 * F00 + F10 * F10 + F20 * F20;
    C[1] = F00 * F01 + F10 * F11 + F20 * F21;
    C[2] = F00 * F02 + F10 * F12 + F20 * F22;
    C[3] = F01 * F00 + F11 * F10 + F21 * F20;
    C[4] = F01 * F01 + F11 * F11 + F21 * F21;
    C[5] = F01 * F02 + F11 * F12 + F21 * F22;
    C[6] = F02 * F00 + F12 * F10 + F22 * F20;
    C[7] = F02 * F01 + F12 * F11 + F22 * F21;
    C[8] = F02 * F02 + F12 * F12 + F22 * F22;
    const float I_c = C[0] + C[4] + C[8];
    const float I_c2 = I_c * I_c;
    float CC[9];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) CC[a * 3 + b] = C[a * 3 + 0] * C[b * 3 + 0] + C[a * 3 + 1] * C[b * 3 + 1] + C[a * 3 + 2] * C[b * 3 + 2];
    const float II_c = (float)(0.5 * (double)(I_c2 - CC[0] - CC[4] - CC[8]));
    const float k = I_c2 - 3 * II_c;
    float invU[9];
    if (k < 1e-6f) {
        if ((double)I_c < 1e-6) return;
        const float t = 1 / sqrtf(I_c / 3);
        for (int i = 0; i < 9; ++i) invU[i] = 0.f;
        invU[0] = invU[4] = invU[8] = t;
    } else {
        const float l = I_c * (I_c * I_c - 4.5f * II_c) + 13.5f * III_c;
        const float k_root = sqrtf(k);
        float value = l / (k * k_root);
        value = fminf(1.0f, fmaxf(-1.0f, value));
        const float phi = acosf(value);
        const float lambda2 = (float)((double)(I_c + 2 * k_root * cosf(phi / 3)) / 3.0);
        const float lambda = sqrtf(lambda2);
        const float III_u = det;
        if ((double)fabsf(lambda) < 1e-6) return;
        if ((double)(-lambda2 + I_c + 2 * III_u / lambda) < 1e-6) return;
        const float I_u = lambda + sqrtf(-lambda2 + I_c + 2 * III_u / lambda);
        const float II_u = (float)((double)(I_u * I_u - I_c) * 0.5);
        if ((double)fabsf(I_u * II_u - III_u) < 1e-6) return;
        float inv_rate = 1 / (I_u * II_u - III_u);
        const float t0 = I_u * III_u * inv_rate;
        const float factor0 = (I_u * I_u - II_u) * inv_rate;
        float U[9];
        for (int i = 0; i < 9; ++i) U[i] = factor0 * C[i] - inv_rate * CC[i];
        U[0] += t0; U[4] += t0; U[8] += t0;
        if ((double)fabsf(III_u) < 1e-6) return;
        inv_rate = 1 / III_u;
        const float t1 = II_u * inv_rate;
        const float factor1 = -I_u * inv_rate;
        for (int i = 0; i < 9; ++i) invU[i] = factor1 * U[i] + inv_rate * C[i];
        invU[0] += t1; invU[4] += t1; invU[8] += t1;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i * 3 + j] = F[i * 3 + 0] * invU[0 * 3 + j] + F[i * 3 + 1] * invU[1 * 3 + j] + F[i * 3 + 2] * invU[2 * 3 + j];
}

// ---------------------------------------------------------------------------
// Rotation of the rotation-variant SVD F = U S V^T (U, V proper rotations,
// S with the sign of det F on the smallest entry): R = U V^T, the closest
// rotation to F, defined for inverted tets too.
// Right singular vectors: cyclic Jacobi eigen-iteration on the symmetric
// S = F^T F (fixed sweep count); left vectors: Gram-Schmidt of F v1, F v2 and
// u3 = u1 x u2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void jacobi_rotate(float S[9], float V[9], int p, int q) {
    const float apq = S[p * 3 + q];
    if (fabsf(apq) < 1e-30f) return;
    const float app = S[p * 3 + p], aqq = S[q * 3 + q];
    const float theta = (aqq - app) / (2.f * apq);
    float t;
    if (fabsf(theta) > 1e10f)
        t = 0.5f / theta;
    else
        t = copysignf(1.f, theta) / (fabsf(theta) + sqrtf(fmaf(theta, theta, 1.f)));
    const float c = rsqrtf(fmaf(t, t, 1.f));
    const float s = t * c;
    const int r = 3 - p - q;
    const float arp = S[r * 3 + p], arq = S[r * 3 + q];
    S[p * 3 + p] = app - t * apq;
    S[q * 3 + q] = aqq + t * apq;
    S[p * 3 + q] = S[q * 3 + p] = 0.f;
    const float nrp = c * arp - s * arq, nrq = s * arp + c * arq;
    S[r * 3 + p] = S[p * 3 + r] = nrp;
    S[r * 3 + q] = S[q * 3 + r] = nrq;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float vp = V[i * 3 + p], vq = V[i * 3 + q];
        V[i * 3 + p] = c * vp - s * vq;
        V[i * 3 + q] = s * vp + c * vq;
    }
}

__device__ __forceinline__ void swap_cols_neg(float V[9], float lam[3], int a, int b) {
    const float tl = lam[a];
    lam[a] = lam[b];
    lam[b] = tl;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float t = V[i * 3 + a];
        V[i * 3 + a] = V[i * 3 + b];
        V[i * 3 + b] = -t;  // keep det V = +1
    }
}

__device__ __forceinline__ void svd_rotation(const float F[9], float R[9]) {
    float S[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) S[a * 3 + b] = F[0 * 3 + a] * F[0 * 3 + b] + F[1 * 3 + a] * F[1 * 3 + b] + F[2 * 3 + a] * F[2 * 3 + b];
    float V[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
#pragma unroll 1
    for (int sweep = 0; sweep < 5; ++sweep) {
        jacobi_rotate(S, V, 0, 1);
        jacobi_rotate(S, V, 0, 2);
        jacobi_rotate(S, V, 1, 2);
    }
    float lam[3] = {S[0], S[4], S[8]};
    if (lam[0] < lam[1]) swap_cols_neg(V, lam, 0, 1);
    if (lam[0] < lam[2]) swap_cols_neg(V, lam, 0, 2);
    if (lam[1] < lam[2]) swap_cols_neg(V, lam, 1, 2);
    // b_i = F v_i
    float b1[3], b2[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        b1[i] = F[i * 3 + 0] * V[0] + F[i * 3 + 1] * V[3] + F[i * 3 + 2] * V[6];
        b2[i] = F[i * 3 + 0] * V[1] + F[i * 3 + 1] * V[4] + F[i * 3 + 2] * V[7];
    }
    const float n1 = b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2];
    if (!(n1 > 1e-30f)) {
#pragma unroll
        for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.f : 0.f;
        return;
    }
    const float r1 = rsqrtf(n1);
    float u1[3] = {b1[0] * r1, b1[1] * r1, b1[2] * r1};
    const float d = u1[0] * b2[0] + u1[1] * b2[1] + u1[2] * b2[2];
    float u2[3] = {b2[0] - d * u1[0], b2[1] - d * u1[1], b2[2] - d * u1[2]};
    float n2 = u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2];
    if (!(n2 > 1e-24f * n1)) {
        // F has rank <= 1: any unit vector orthogonal to u1.
        const float ax = fabsf(u1[0]), ay = fabsf(u1[1]), az = fabsf(u1[2]);
        float e[3] = {0.f, 0.f, 0.f};
        if (ax <= ay && ax <= az) e[0] = 1.f; else if (ay <= az) e[1] = 1.f; else e[2] = 1.f;
        const float de = u1[0] * e[0] + u1[1] * e[1] + u1[2] * e[2];
        u2[0] = e[0] - de * u1[0]; u2[1] = e[1] - de * u1[1]; u2[2] = e[2] - de * u1[2];
        n2 = u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2];
    }
    const float r2 = rsqrtf(n2);
    u2[0] *= r2; u2[1] *= r2; u2[2] *= r2;
    const float u3[3] = {u1[1] * u2[2] - u1[2] * u2[1], u1[2] * u2[0] - u1[0] * u2[2], u1[0] * u2[1] - u1[1] * u2[0]};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) R[i * 3 + j] = u1[i] * V[j * 3 + 0] + u2[i] * V[j * 3 + 1] + u3[i] * V[j * 3 + 2];
}

// Orthogonal polar factor of F for det F > 0 by the scaled Newton iteration
// of Higham (1986), "Computing the polar decomposition - with applications":
// X <- (g X + X^-T / g) / 2 from X = F, with g = (|X^-1|_F / |X|_F)^(1/2) and
// X^-T = cof(X) / det X.  For det F > 0 the polar factor is the rotation
// U V^T of the SVD, the same matrix svd_rotation returns.  Stops when
// |X_new - X|_F < 1e-6 (the error of X_new is then ~1e-12 by quadratic
// convergence; 4-6 steps up to condition number 1e4); returns false if det X
// <= 0 or no convergence in 8 steps (the caller falls back to the SVD).
__device__ __forceinline__ bool polar_newton(const float F[9], float R[9]) {
    float X[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) X[q] = F[q];
#pragma unroll 1
    for (int it = 0; it < 8; ++it) {
        const float C[9] = {X[4] * X[8] - X[5] * X[7], X[5] * X[6] - X[3] * X[8], X[3] * X[7] - X[4] * X[6],
                            X[2] * X[7] - X[1] * X[8], X[0] * X[8] - X[2] * X[6], X[1] * X[6] - X[0] * X[7],
                            X[1] * X[5] - X[2] * X[4], X[2] * X[3] - X[0] * X[5], X[0] * X[4] - X[1] * X[3]};
        const float det = X[0] * C[0] + X[1] * C[1] + X[2] * C[2];
        if (!(det > 0.f)) return false;
        float nx = 0.f, nc = 0.f;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            nx = fmaf(X[q], X[q], nx);
            nc = fmaf(C[q], C[q], nc);
        }
        const float g = sqrtf(sqrtf(nc / nx) / det);
        const float a = 0.5f * g, b = 0.5f / (det * g);
        float d = 0.f;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float xn = fmaf(a, X[q], b * C[q]);
            const float t = xn - X[q];
            d = fmaf(t, t, d);
            X[q] = xn;
        }
        if (!(d == d)) return false;   // NaN
        if (d < 1e-12f) {
#pragma unroll
            for (int q = 0; q < 9; ++q) R[q] = X[q];
            return true;
        }
    }
    return false;
}

// Closest point on segment [a, b] to p; returns the segment parameter.
__device__ __forceinline__ float closest_on_segment(const float p[3], const float a[3], const float b[3], float q[3]) {
    const float ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const float l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    float t = 0.f;
    if (l2 > 0.f) {
        t = ((p[0] - a[0]) * ab[0] + (p[1] - a[1]) * ab[1] + (p[2] - a[2]) * ab[2]) / l2;
        t = fminf(1.f, fmaxf(0.f, t));
    }
    q[0] = a[0] + t * ab[0];
    q[1] = a[1] + t * ab[1];
    q[2] = a[2] + t * ab[2];
    return t;
}

}  // namespace mgsb
