// sm_100a kernels of the PD soft-body frame.  Included by solver.cu only.
//
// Layout in HBM (all bodies of a batch concatenated per level):
//   positions / RHS / corrections : float4 per vertex (xyz + pad, 16-B vector access)
//   tets                          : int4 vertex ids + (float4, float4, float2) rest data
//   per-(tet, corner) RHS slots   : float4, ordered by vertex (CSR), so the RHS
//                                   gather is a contiguous segmented sum — no atomics
//   matrices                      : sliced ELL (32-row slices, column-major inside
//                                   a slice), off-diagonal only; diagonal apart
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_math.cuh"

namespace mgsb {

// ---------------------------------------------------------------------------
// Shared structures passed by value to kernels
// ---------------------------------------------------------------------------
struct SphereSet {
    int count;
    float cx[8], cy[8], cz[8], r[8];
    int active[8];
};

// Per-body table, device resident.  Tool pose is rewritten every frame.
struct BodyDev {
    int v0_off, v0_n;        // finest-level vertex range
    int cl_off, cl_n;        // coarsest-level vertex range
    int dense_off;           // offset of the coarsest dense n*n block
    int pad0;
    float gravity[4];
    float damping;
    float cap_r;
    float pad1[2];
    float cap_a[4];
    float cap_b[4];
};

// ===========================================================================
// Reference-faithful Jacobi/Chebyshev frame (PDSolver::Step)
// ===========================================================================

// calculateST (PDSolver.cu:72-116); external force is always zero in the
// reference's frame and is omitted.
__global__ void k_ref_predict(int n, float4* __restrict__ x, float4* __restrict__ v, float4* __restrict__ s,
                              float4* __restrict__ prev, float4* __restrict__ last, const float* __restrict__ fixf,
                              float damping, float dt, float gx, float gy, float gz) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = x[i], vel = v[i];
    last[i] = p;
    const float fix = fixf[i];
    vel.x *= damping * fix; vel.y *= damping * fix; vel.z *= damping * fix;
    vel.x += gx * dt * fix; vel.y += gy * dt * fix; vel.z += gz * dt * fix;
    p.x += vel.x * dt * fix; p.y += vel.y * dt * fix; p.z += vel.z * dt * fix;
    x[i] = p;
    v[i] = vel;
    s[i] = p;
    prev[i] = p;
}

// Local step, one thread per tet: F = Ds Dm^-1, R by the invariant polar
// decomposition, per (i,j): val = sum_k (R-F)_ik Ac_kj, NaN->0, clamp +-10,
// c = val*V*k, |c| < 1e-5 dropped (PDSolverAc.cu:447-662).  The four corner
// contributions go to their RHS slots (float4 each).
__global__ void __launch_bounds__(256) k_ref_local(int T, const int4* __restrict__ tets, const float4* __restrict__ invA,
                                                   const float4* __restrict__ invB, const float2* __restrict__ invC,
                                                   const float4* __restrict__ x, const int4* __restrict__ slot_of,
                                                   float4* __restrict__ slots, float stiffness, int drop_small = 1) {
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int4 id = __ldg(tets + t);
    const float4 a = __ldg(invA + t), b = __ldg(invB + t);
    const float2 c = __ldg(invC + t);
    const float inv[9] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x};
    const float vol = c.y;
    const float4 p0 = __ldg(x + id.x), p1 = __ldg(x + id.y), p2 = __ldg(x + id.z), p3 = __ldg(x + id.w);
    const float D[9] = {p1.x - p0.x, p2.x - p0.x, p3.x - p0.x, p1.y - p0.y, p2.y - p0.y,
                        p3.y - p0.y, p1.z - p0.z, p2.z - p0.z, p3.z - p0.z};
    float F[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) F[r * 3 + q] = D[r * 3 + 0] * inv[q] + D[r * 3 + 1] * inv[3 + q] + D[r * 3 + 2] * inv[6 + q];
    float R[9];
    ref_rotation(F, R);
    float FR[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) FR[q] = R[q] - F[q];
    // Ac (3x4): column 0 = -(sum of inv rows), columns 1..3 = inv rows.
    float Ac[12];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        Ac[r * 4 + 0] = -inv[r] - inv[r + 3] - inv[r + 6];
        Ac[r * 4 + 1] = inv[r];
        Ac[r * 4 + 2] = inv[r + 3];
        Ac[r * 4 + 3] = inv[r + 6];
    }
    const int4 so = __ldg(slot_of + t);
    const int sid[4] = {so.x, so.y, so.z, so.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float out[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float val = FR[i * 3 + 0] * Ac[0 * 4 + j] + FR[i * 3 + 1] * Ac[1 * 4 + j] + FR[i * 3 + 2] * Ac[2 * 4 + j];
            if (isnan(val)) val = 0.f;
            val = fminf(10.0f, fmaxf(-10.0f, val));
            float res = val * vol * stiffness;
            // the single-kernel calculateIF of the two-level schedule (PDSolver.cu:128-183)
            // keeps small contributions; getTetFRV2/calTetIFV1 drop |c| < 1e-5
            if (drop_small && (double)fabsf(res) < 1e-5) res = 0.f;
            out[i] = res;
        }
        slots[sid[j]] = make_float4(out[0], out[1], out[2], 0.f);
    }
}

// Per vertex: gather the elastic force from the slots, sphere DCD
// (DCDByPoint_sphere, PDSolver.cu:277-331), then the under-relaxed Jacobi
// step with Chebyshev acceleration (calculatePOS, PDSolver.cu:192-235).
// On the last iteration also v = (x - last)/dt (calculateV, PDSolver.cu:245).
__global__ void __launch_bounds__(256) k_ref_vertex(
    int n, float4* __restrict__ x, float4* __restrict__ prev, const float4* __restrict__ s, const float4* __restrict__ last,
    float4* __restrict__ v, const float* __restrict__ fixf, const float* __restrict__ mass, const float* __restrict__ vdiag,
    const int32_t* __restrict__ slot_ptr, const float4* __restrict__ slots, const SphereSet* __restrict__ spheres,
    float kc, float dt, float omega, double relax, int last_iter, int32_t* __restrict__ cflag, float* __restrict__ cdepth,
    float* __restrict__ cenergy, int32_t* __restrict__ nonfinite, const int32_t* __restrict__ tri_ptr = nullptr,
    const int32_t* __restrict__ tri_idx = nullptr, const float4* __restrict__ tri_push = nullptr) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    const int e1 = __ldg(slot_ptr + i + 1);
    for (int e = __ldg(slot_ptr + i); e < e1; ++e) {
        const float4 c = __ldg(slots + e);
        fx += c.x; fy += c.y; fz += c.z;
    }
    const float4 p4 = x[i];
    const float p[3] = {p4.x, p4.y, p4.z};
    float cd[3] = {0.f, 0.f, 0.f}, cf[3] = {0.f, 0.f, 0.f};
    int flag = 0;
    float depth = 0.f, ce = 0.f;
    if (tri_push) {
        // collision from the surface triangles around this vertex (the coarse level of
        // the two-level schedule): k_c per contact on every axis, k_c (c - hit) as force
        float cnt = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
        const int t1 = __ldg(tri_ptr + i + 1);
        for (int e = __ldg(tri_ptr + i); e < t1; ++e) {
            const float4 q = tri_push[__ldg(tri_idx + e)];
            mx += q.x;
            my += q.y;
            mz += q.z;
            cnt += q.w;
        }
        cd[0] = cd[1] = cd[2] = kc * cnt;
        cf[0] = kc * mx;
        cf[1] = kc * my;
        cf[2] = kc * mz;
        flag = (int)cnt;
    }
    const int nsph = tri_push ? 0 : spheres->count;
    for (int q = 0; q < nsph; ++q) {
        if (!spheres->active[q]) continue;
        const float cx = spheres->cx[q], cy = spheres->cy[q], cz = spheres->cz[q];
        float radius = spheres->r[q];
        const float cp[3] = {p[0] - cx, p[1] - cy, p[2] - cz};
        const float len = sqrtf(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]);
        const float dir[3] = {cp[0] / len, cp[1] / len, cp[2] / len};
        const float distance = len;
        const float oldRadius = radius;
        radius *= 1.5f;
        if (distance < radius) {
            const float bq = 2 * (cp[0] * dir[0] + cp[1] * dir[1] + cp[2] * dir[2]);
            const float cq = (cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]) - radius * radius;
            float t = (-bq + sqrtf(bq * bq - 4 * 1 * cq)) / (2 * 1);
            if (t > 0.5f * oldRadius) {
                flag = 1;
                depth = t - 0.5f * oldRadius;
            }
            t = t / 2.0f;
            const float colP[3] = {p[0] + dir[0] * t, p[1] + dir[1] * t, p[2] + dir[2] * t};
            const float cc[3] = {colP[0] - cx, colP[1] - cy, colP[2] - cz};
            const float lc = sqrtf(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
            const float nrm[3] = {cc[0] / lc, cc[1] / lc, cc[2] / lc};
            const float ndd = nrm[0] * dir[0] + nrm[1] * dir[1] + nrm[2] * dir[2];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                cd[a] += kc * nrm[a] * nrm[a];
                cf[a] += kc * t * ndd * nrm[a];
            }
            const float pe = (p[0] - colP[0]) * nrm[0] + (p[1] - colP[1]) * nrm[1] + (p[2] - colP[2]) * nrm[2];
            ce += kc * pe * pe;
        }
    }
    const float fix = __ldg(fixf + i);
    const float dc = __ldg(mass + i) / (dt * dt);
    const float vd = __ldg(vdiag + i);
    const float4 s4 = __ldg(s + i), pv4 = prev[i];
    const float sv[3] = {s4.x, s4.y, s4.z}, pv[3] = {pv4.x, pv4.y, pv4.z};
    const float fe[3] = {fx, fy, fz};
    float nx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float el = fe[a] + cf[a];
        float nxt = (dc * (sv[a] - p[a]) + el) / (vd + cd[a] + dc) * fix + p[a];
        nxt = (float)((double)(nxt - p[a]) * relax + (double)p[a]);
        nxt = omega * (nxt - pv[a]) + pv[a];
        nx[a] = nxt;
    }
    prev[i] = p4;
    const float4 xn = make_float4(nx[0], nx[1], nx[2], 0.f);
    x[i] = xn;
    // last_iter: bit 0 = velocity, bit 1 = contact outputs and the finiteness check
    if (last_iter & 1) {
        const float4 l4 = __ldg(last + i);
        v[i] = make_float4((xn.x - l4.x) / dt, (xn.y - l4.y) / dt, (xn.z - l4.z) / dt, 0.f);
    }
    if (last_iter & 2) {
        cflag[i] = flag;
        cdepth[i] = depth;
        cenergy[i] = ce;
        if (!isfinite(xn.x) || !isfinite(xn.y) || !isfinite(xn.z)) atomicOr(nonfinite, 1);
    }
}

// ===========================================================================
// Multigrid frame
// ===========================================================================

// Inertial prediction (same form as calculateST) with per-body gravity and
// damping: last = x; v = v*damp*fix + g*dt*fix; x = s = x + v*dt*fix.
__global__ void k_mg_predict(int n, float4* __restrict__ x, float4* __restrict__ v, float4* __restrict__ s,
                             float4* __restrict__ last, const float* __restrict__ fixf, const int32_t* __restrict__ body_of,
                             const BodyDev* __restrict__ bodies, float dt) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BodyDev& B = bodies[__ldg(body_of + i)];
    float4 p = x[i], vel = v[i];
    last[i] = p;
    const float fix = __ldg(fixf + i);
    vel.x *= B.damping * fix; vel.y *= B.damping * fix; vel.z *= B.damping * fix;
    vel.x += B.gravity[0] * dt * fix; vel.y += B.gravity[1] * dt * fix; vel.z += B.gravity[2] * dt * fix;
    p.x += vel.x * dt * fix; p.y += vel.y * dt * fix; p.z += vel.z * dt * fix;
    p.w = 0.f;
    x[i] = p;
    v[i] = vel;
    s[i] = p;
}

// Capsule contact of one surface vertex against its body's capsule, evaluated
// in FP64 on the predicted position: contact iff dist(s, segment) < r; the
// projection target is the capsule surface point along the capsule normal.
__device__ __forceinline__ void capsule_test(const float4 sp, const BodyDev& B, int& flag, float4& target) {
    flag = 0;
    target = make_float4(0.f, 0.f, 0.f, 0.f);
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
    target = make_float4((float)(q[0] + r * nrm[0]), (float)(q[1] + r * nrm[1]), (float)(q[2] + r * nrm[2]), 0.f);
}

// ---------------------------------------------------------------------------
// Capsule against the surface triangles (FP64).  A triangle is in contact when
// its distance to the capsule's segment is below the radius, so a capsule that
// enters a face between its vertices is found although no vertex lies inside
// it.  The push of a contacting triangle moves it out along the line of the
// closest points: push = (h - q) / |h - q| * (r - |h - q|), h on the triangle,
// q on the segment -- the capsule form of the face / edge half-cylinder /
// vertex cases of the reference's sphere test DCDByTriangle_sphere_V2
// (PDSolver.cu:612-680, response :462-501), whose push centre - hit is the
// same vector for a sphere.  When the segment touches the triangle (|h - q| ~ 0)
// the push is r along the inward normal.  Per vertex, the pushes of its
// contacting triangles are averaged in ascending triangle order (a gather
// instead of the reference's float atomics).
// ---------------------------------------------------------------------------
struct Dv3 {
    double x, y, z;
};
__device__ __forceinline__ Dv3 dv3(double x, double y, double z) { return Dv3{x, y, z}; }
__device__ __forceinline__ Dv3 dsub(Dv3 a, Dv3 b) { return dv3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ Dv3 dadd(Dv3 a, Dv3 b) { return dv3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ Dv3 dscale(Dv3 a, double s) { return dv3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double ddot(Dv3 a, Dv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Dv3 dcross(Dv3 a, Dv3 b) {
    return dv3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// Closest point of triangle abc to p, by the Voronoi regions of its vertices,
// edges and face (Ericson, Real-Time Collision Detection, sec. 5.1.5).
__device__ __forceinline__ Dv3 tri_closest_point(Dv3 p, Dv3 a, Dv3 b, Dv3 c) {
    const Dv3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    const double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return a;
    const Dv3 bp = dsub(p, b);
    const double d3 = ddot(ab, bp), d4 = ddot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return b;
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return dadd(a, dscale(ab, d1 / (d1 - d3)));
    const Dv3 cp = dsub(p, c);
    const double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return c;
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return dadd(a, dscale(ac, d2 / (d2 - d6)));
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0)
        return dadd(b, dscale(dsub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
    const double den = 1.0 / (va + vb + vc);
    return dadd(a, dadd(dscale(ab, vb * den), dscale(ac, vc * den)));
}

// Closest points c1 on segment p1q1 and c2 on segment p2q2 (Ericson sec. 5.1.9,
// clamped parametric form); returns |c1 - c2|^2.
__device__ __forceinline__ double seg_seg_closest(Dv3 p1, Dv3 q1, Dv3 p2, Dv3 q2, Dv3& c1, Dv3& c2) {
    const Dv3 d1 = dsub(q1, p1), d2 = dsub(q2, p2), r = dsub(p1, p2);
    const double a = ddot(d1, d1), e = ddot(d2, d2), f = ddot(d2, r);
    double s = 0.0, t = 0.0;
    if (a <= 1e-300 && e <= 1e-300) {
        s = t = 0.0;
    } else if (a <= 1e-300) {
        t = fmin(fmax(f / e, 0.0), 1.0);
    } else {
        const double c = ddot(d1, r);
        if (e <= 1e-300) {
            s = fmin(fmax(-c / a, 0.0), 1.0);
        } else {
            const double b = ddot(d1, d2), den = a * e - b * b;
            s = den > 0.0 ? fmin(fmax((b * f - c * e) / den, 0.0), 1.0) : 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) {
                t = 0.0;
                s = fmin(fmax(-c / a, 0.0), 1.0);
            } else if (t > 1.0) {
                t = 1.0;
                s = fmin(fmax((b - c) / a, 0.0), 1.0);
            }
        }
    }
    c1 = dadd(p1, dscale(d1, s));
    c2 = dadd(p2, dscale(d2, t));
    const Dv3 w = dsub(c1, c2);
    return ddot(w, w);
}

// Push of triangle (a, b, c) (o: the fourth vertex of its tet, inside the
// body) out of the capsule (segment p0p1, radius r): true and push when the
// triangle is in contact.
__device__ __forceinline__ bool tri_capsule_push(Dv3 a, Dv3 b, Dv3 c, Dv3 o, Dv3 p0, Dv3 p1, double r, Dv3& push) {
    double best = 1e300;
    Dv3 q = p0, h = a;
    {   // segment end points against the triangle
        const Dv3 h0 = tri_closest_point(p0, a, b, c), h1 = tri_closest_point(p1, a, b, c);
        const double e0 = ddot(dsub(p0, h0), dsub(p0, h0)), e1 = ddot(dsub(p1, h1), dsub(p1, h1));
        if (e0 < best) { best = e0; q = p0; h = h0; }
        if (e1 < best) { best = e1; q = p1; h = h1; }
    }
    const Dv3 ev[3][2] = {{a, b}, {b, c}, {c, a}};
#pragma unroll
    for (int k = 0; k < 3; ++k) {   // segment against the edges
        Dv3 cs, ct;
        const double e2 = seg_seg_closest(p0, p1, ev[k][0], ev[k][1], cs, ct);
        if (e2 < best) { best = e2; q = cs; h = ct; }
    }
    const Dv3 n = dcross(dsub(b, a), dsub(c, a));
    {   // segment through the face
        const double s0 = ddot(n, dsub(p0, a)), s1 = ddot(n, dsub(p1, a));
        if ((s0 <= 0.0 && s1 >= 0.0) || (s0 >= 0.0 && s1 <= 0.0)) {
            if (s0 != s1) {
                const Dv3 x = dadd(p0, dscale(dsub(p1, p0), s0 / (s0 - s1)));
                const double u = ddot(dcross(dsub(b, a), dsub(x, a)), n), v = ddot(dcross(dsub(c, b), dsub(x, b)), n),
                             w = ddot(dcross(dsub(a, c), dsub(x, c)), n);
                if (u >= 0.0 && v >= 0.0 && w >= 0.0) { best = 0.0; q = x; h = x; }
            }
        }
    }
    if (!(best < r * r)) return false;
    const double dist = sqrt(best);
    if (dist > 1e-12) {
        push = dscale(dsub(h, q), (r - dist) / dist);
    } else {   // the segment touches the face: push r along the inward normal
        const double nl = sqrt(ddot(n, n));
        const double sgn = ddot(n, dsub(o, a)) > 0.0 ? 1.0 : -1.0;   // towards the inside of the body
        push = nl > 0.0 ? dscale(n, sgn * r / nl) : dv3(0.0, 0.0, 0.0);
    }
    return true;
}

// Per surface triangle: push[f] = (push, 1) when triangle f touches its body's
// capsule, else zero.  tris[f] = (a, b, c, o) global vertex ids, o the inner
// vertex of the triangle's tet.  P = float4 (FP32 kind) or double4 (mixed).
template <typename P>
__global__ void k_tri_capsule(int nf, const int4* __restrict__ tris, const int32_t* __restrict__ body_of,
                              const BodyDev* __restrict__ bodies, const P* __restrict__ s, double4* __restrict__ push) {
    pdl_enter();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int4 t = __ldg(tris + f);
    const BodyDev& B = bodies[__ldg(body_of + t.x)];
    double4 out = make_double4(0.0, 0.0, 0.0, 0.0);
    const double r = B.cap_r;
    if (r > 0.0) {
        auto ld = [&](int i) {
            const P v = s[i];
            return dv3((double)v.x, (double)v.y, (double)v.z);
        };
        Dv3 pu;
        if (tri_capsule_push(ld(t.x), ld(t.y), ld(t.z), ld(t.w), dv3(B.cap_a[0], B.cap_a[1], B.cap_a[2]),
                             dv3(B.cap_b[0], B.cap_b[1], B.cap_b[2]), r, pu))
            out = make_double4(pu.x, pu.y, pu.z, 1.0);
    }
    push[f] = out;
}

// Mean push of vertex i's contacting surface triangles (vt_ptr / vt_idx: its
// triangles, ascending); false when none is in contact.
__device__ __forceinline__ bool tri_contact_gather(int i, const int32_t* __restrict__ vt_ptr,
                                                   const int32_t* __restrict__ vt_idx, const double4* __restrict__ push,
                                                   Dv3& mean) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    int k = 0;
    const int e1 = __ldg(vt_ptr + i + 1);
    for (int e = __ldg(vt_ptr + i); e < e1; ++e) {
        const double4 pu = push[__ldg(vt_idx + e)];
        if (pu.w != 0.0) {
            sx += pu.x;
            sy += pu.y;
            sz += pu.z;
            ++k;
        }
    }
    if (!k) return false;
    mean = dv3(sx / k, sy / k, sz / k);
    return true;
}

// Brute-force narrow phase over all surface vertices (used when the broad
// phase is disabled).
// With vt_ptr set (triangle contact on), a vertex outside the capsule whose
// surface triangles touch it is a contact too, projected to s + their mean push.
__global__ void k_contact_all(int ns, const int32_t* __restrict__ surf, const int32_t* __restrict__ body_of,
                              const BodyDev* __restrict__ bodies, const float4* __restrict__ s,
                              const float* __restrict__ fixf, float kc, int32_t* __restrict__ cflag,
                              float* __restrict__ c0, float4* __restrict__ target,
                              const int32_t* __restrict__ vt_ptr = nullptr, const int32_t* __restrict__ vt_idx = nullptr,
                              const double4* __restrict__ push = nullptr) {
    pdl_enter();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ns) return;
    const int i = __ldg(surf + q);
    int flag;
    float4 tg;
    const float4 sp = __ldg(s + i);
    capsule_test(sp, bodies[__ldg(body_of + i)], flag, tg);
    Dv3 mp;
    if (!flag && vt_ptr && tri_contact_gather(i, vt_ptr, vt_idx, push, mp)) {
        flag = 1;
        tg = make_float4((float)((double)sp.x + mp.x), (float)((double)sp.y + mp.y), (float)((double)sp.z + mp.z), 0.f);
    }
    cflag[i] = flag;
    c0[i] = (flag && __ldg(fixf + i) != 0.f) ? kc : 0.f;
    target[i] = tg;
}

// Per frame, level 0.  The global step is solved for the displacement from
// the prediction, d = x - s, so every right-hand-side term is a small
// difference: b0 = c (p - s), D = L_ii + c, dinv = fixed ? 0 : omega/D, d = 0.
__global__ void k_l0_frame(int n, const float4* __restrict__ s, const float* __restrict__ c0,
                           const float4* __restrict__ target, const float* __restrict__ diag0,
                           const float* __restrict__ fixf, float omega, float4* __restrict__ b0, float* __restrict__ dfull,
                           float* __restrict__ dinv, float4* __restrict__ d) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float c = __ldg(c0 + i);
    const float4 sv = __ldg(s + i), tg = __ldg(target + i);
    b0[i] = c != 0.f ? make_float4(c * (tg.x - sv.x), c * (tg.y - sv.y), c * (tg.z - sv.z), 0.f)
                     : make_float4(0.f, 0.f, 0.f, 0.f);
    const float D = __ldg(diag0 + i) + c;
    dfull[i] = D;
    dinv[i] = (__ldg(fixf + i) != 0.f) ? omega / D : 0.f;
    d[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Positions as packed xyz (3 floats per vertex) for the zero-copy frame
// readback; launched on its own after a frame, outside the frame's graph.
__global__ void k_pack_xyz(int n, const float4* __restrict__ x, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = x[i];
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
}

// End of frame: x = s + d, v = v_predicted + d/dt (= (x - x_prev)/dt), and a
// finiteness check of the new positions.
__global__ void k_mg_finish(int n, const float4* __restrict__ s, const float4* __restrict__ d, float4* __restrict__ x,
                            float4* __restrict__ v, float inv_dt, int32_t* __restrict__ nonfinite) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 sv = __ldg(s + i), dv = __ldg(d + i);
    float4 vel = v[i];
    const float4 p = make_float4(sv.x + dv.x, sv.y + dv.y, sv.z + dv.z, 0.f);
    vel.x = fmaf(dv.x, inv_dt, vel.x);
    vel.y = fmaf(dv.y, inv_dt, vel.y);
    vel.z = fmaf(dv.z, inv_dt, vel.z);
    x[i] = p;
    v[i] = vel;
    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) atomicOr(nonfinite, 1);
}

// Per frame, level l >= 1: lumped contact weight c_l = P^T c_{l-1}, D and dinv.
// The children, their weights and the contact-free diagonal are set-up data:
// the first kCoarseFrameHeld children are loaded before the dependency wait.
constexpr int kCoarseFrameHeld = 8;
__global__ void k_coarse_frame(int n, const int32_t* __restrict__ rptr, const int32_t* __restrict__ rcol,
                               const float* __restrict__ rw, const float* __restrict__ cfine,
                               const float* __restrict__ diag0, float omega, float* __restrict__ c,
                               float* __restrict__ dfull, float* __restrict__ dinv) {
    pdl_trigger();
    const int J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= n) return;
    const int e0 = __ldg(rptr + J), e1 = __ldg(rptr + J + 1);
    int ch[kCoarseFrameHeld];
    float w[kCoarseFrameHeld];
#pragma unroll
    for (int k = 0; k < kCoarseFrameHeld; ++k) {
        ch[k] = e0 + k < e1 ? __ldg(rcol + e0 + k) : -1;
        w[k] = e0 + k < e1 ? __ldg(rw + e0 + k) : 0.f;
    }
    const float d0 = __ldg(diag0 + J);
    pdl_wait();
    float acc = 0.f;   // the children in CSR order, as one loop over them
#pragma unroll
    for (int k = 0; k < kCoarseFrameHeld; ++k)
        if (ch[k] >= 0) acc = fmaf(w[k], __ldg(cfine + ch[k]), acc);
    for (int e = e0 + kCoarseFrameHeld; e < e1; ++e) acc = fmaf(__ldg(rw + e), __ldg(cfine + __ldg(rcol + e)), acc);
    c[J] = acc;
    const float D = d0 + acc;
    dfull[J] = D;
    dinv[J] = d0 > 0.f ? omega / D : 0.f;
}

// Local step, one thread per tet, on x = s + d: F = sum_j x_j g_j^T from the
// edge vectors (s_k - s_0) + (d_k - d_0), R = closest rotation; the RHS of
// the displacement system gets w (R - F(s)) g_j in the four corner slots.
__global__ void __launch_bounds__(256) k_mg_local(int T, const int4* __restrict__ tets, const float4* __restrict__ gA,
                                                  const float4* __restrict__ gB, const float2* __restrict__ gC,
                                                  const float4* __restrict__ s, const float4* __restrict__ d,
                                                  const int4* __restrict__ slot_of, float4* __restrict__ slots) {
    pdl_trigger();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) {
        pdl_wait();
        return;
    }
    // the tet's set-up data (vertices, shape gradients, weight, slots) is written by no kernel:
    // loaded before the dependency wait, while the previous kernel runs
    const int4 id = __ldg(tets + t);
    const float4 a = __ldg(gA + t), b = __ldg(gB + t);
    const float2 c = __ldg(gC + t);
    const int4 so = __ldg(slot_of + t);
    pdl_wait();
    // g1 = (a.x a.y a.z), g2 = (a.w b.x b.y), g3 = (b.z b.w c.x), w = c.y
    const float g1[3] = {a.x, a.y, a.z}, g2[3] = {a.w, b.x, b.y}, g3[3] = {b.z, b.w, c.x};
    const float w = c.y;
    const float4 s0 = __ldg(s + id.x), s1 = __ldg(s + id.y), s2 = __ldg(s + id.z), s3 = __ldg(s + id.w);
    const float4 q0 = __ldg(d + id.x), q1 = __ldg(d + id.y), q2 = __ldg(d + id.z), q3 = __ldg(d + id.w);
    const float e1[3] = {s1.x - s0.x, s1.y - s0.y, s1.z - s0.z};
    const float e2[3] = {s2.x - s0.x, s2.y - s0.y, s2.z - s0.z};
    const float e3[3] = {s3.x - s0.x, s3.y - s0.y, s3.z - s0.z};
    const float f1[3] = {q1.x - q0.x, q1.y - q0.y, q1.z - q0.z};
    const float f2[3] = {q2.x - q0.x, q2.y - q0.y, q2.z - q0.z};
    const float f3[3] = {q3.x - q0.x, q3.y - q0.y, q3.z - q0.z};
    float Fs[9], F[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            Fs[r * 3 + q] = e1[r] * g1[q] + e2[r] * g2[q] + e3[r] * g3[q];
            F[r * 3 + q] = (e1[r] + f1[r]) * g1[q] + (e2[r] + f2[r]) * g2[q] + (e3[r] + f3[r]) * g3[q];
        }
    float R[9];
    if (!polar_newton(F, R)) svd_rotation(F, R);   // the SVD only for inverted / degenerate tets
#pragma unroll
    for (int q = 0; q < 9; ++q) R[q] -= Fs[q];
    float o1[3], o2[3], o3[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        o1[r] = w * (R[r * 3 + 0] * g1[0] + R[r * 3 + 1] * g1[1] + R[r * 3 + 2] * g1[2]);
        o2[r] = w * (R[r * 3 + 0] * g2[0] + R[r * 3 + 1] * g2[1] + R[r * 3 + 2] * g2[2]);
        o3[r] = w * (R[r * 3 + 0] * g3[0] + R[r * 3 + 1] * g3[1] + R[r * 3 + 2] * g3[2]);
    }
    slots[so.x] = make_float4(-(o1[0] + o2[0] + o3[0]), -(o1[1] + o2[1] + o3[1]), -(o1[2] + o2[2] + o3[2]), 0.f);
    slots[so.y] = make_float4(o1[0], o1[1], o1[2], 0.f);
    slots[so.z] = make_float4(o2[0], o2[1], o2[2], 0.f);
    slots[so.w] = make_float4(o3[0], o3[1], o3[2], 0.f);
}

// RHS assembly alone: b = b0 + sum of the vertex's slots.
__global__ void k_gather_rhs(int n, float4* __restrict__ b, const float4* __restrict__ b0,
                             const int32_t* __restrict__ slot_ptr, const float4* __restrict__ slots) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 bi = __ldg(b0 + i);
    const int e1 = __ldg(slot_ptr + i + 1);
    for (int e = __ldg(slot_ptr + i); e < e1; ++e) {
        const float4 c = __ldg(slots + e);
        bi.x += c.x; bi.y += c.y; bi.z += c.z;
    }
    b[i] = bi;
}

// v = (x - last)/dt plus a finiteness check of the new positions.
__global__ void k_velocity(int n, const float4* __restrict__ x, const float4* __restrict__ last, float4* __restrict__ v,
                           float dt, int32_t* __restrict__ nonfinite) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = __ldg(x + i), l = __ldg(last + i);
    v[i] = make_float4((p.x - l.x) / dt, (p.y - l.y) / dt, (p.z - l.z) / dt, 0.f);
    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) atomicOr(nonfinite, 1);
}

}  // namespace mgsb
