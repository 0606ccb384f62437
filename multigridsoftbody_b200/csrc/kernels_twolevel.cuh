// Kernels of the reference's two-level schedule (PDSolver_MG::Step,
// PDSolver_MG.cpp:183-253): the coarse level's sphere-vs-surface-triangle
// collision, and the position transfers between the levels.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace mgsb {

// Sphere vs boundary triangle, per triangle (UpdateTriNormal + DCDByTriangle_sphere_V2,
// PDSolver.cu:394-425 and 612-680): unit normal n of (A, B, C); with every
// active sphere in turn: |n.(c - A)| > r -> no contact; else the centre's
// projection inside the triangle pushes along the face normal, else an edge
// whose outer half-cylinder holds the centre pushes radially, else a vertex
// within r pushes radially.  A contact adds the push c - hit to the
// triangle's sum and counts 1.  The reference scatters k_c and k_c (c - hit)
// into the three vertices with float atomics (PDSolver.cu:462-501); here the
// vertex kernel gathers the per-triangle sums through a vertex->triangle CSR.
__global__ void __launch_bounds__(256) k_ref_tri_dcd(int nf, const int4* __restrict__ tris, const float4* __restrict__ x,
                                                     const SphereSet* __restrict__ spheres, float4* __restrict__ push) {
    pdl_enter();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int4 t = __ldg(tris + f);
    const float4 a4 = x[t.x], b4 = x[t.y], c4 = x[t.z];
    const float V[3][3] = {{a4.x, a4.y, a4.z}, {b4.x, b4.y, b4.z}, {c4.x, c4.y, c4.z}};
    const float* A = V[0];
    float n[3];
    {
        const float ab[3] = {V[1][0] - A[0], V[1][1] - A[1], V[1][2] - A[2]};
        const float ac[3] = {V[2][0] - A[0], V[2][1] - A[1], V[2][2] - A[2]};
        n[0] = ab[1] * ac[2] - ab[2] * ac[1];
        n[1] = ab[2] * ac[0] - ab[0] * ac[2];
        n[2] = ab[0] * ac[1] - ab[1] * ac[0];
        const float l = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        n[0] /= l;
        n[1] /= l;
        n[2] /= l;
    }
    float mx = 0.f, my = 0.f, mz = 0.f, cnt = 0.f;
    const int ns = spheres->count;
    for (int q = 0; q < ns; ++q) {
        if (!spheres->active[q]) continue;
        const float ctr[3] = {spheres->cx[q], spheres->cy[q], spheres->cz[q]};
        const float r = spheres->r[q];
        const float ca[3] = {ctr[0] - A[0], ctr[1] - A[1], ctr[2] - A[2]};
        const float sd = n[0] * ca[0] + n[1] * ca[1] + n[2] * ca[2];
        const float dist = fabsf(sd);
        if (dist > r) continue;
        const float proj[3] = {ctr[0] - n[0] * sd, ctr[1] - n[1] * sd, ctr[2] - n[2] * sd};
        float hit[3];
        bool found = false;
        // projection inside the triangle (barycentric test, pointInTriangle utils.cu:366-383)
        {
            const float v0[3] = {V[2][0] - A[0], V[2][1] - A[1], V[2][2] - A[2]};
            const float v1[3] = {V[1][0] - A[0], V[1][1] - A[1], V[1][2] - A[2]};
            const float v2[3] = {proj[0] - A[0], proj[1] - A[1], proj[2] - A[2]};
            const float d00 = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
            const float d01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
            const float d02 = v0[0] * v2[0] + v0[1] * v2[1] + v0[2] * v2[2];
            const float d11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
            const float d12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
            const float inv = 1.0f / (d00 * d11 - d01 * d01);
            const float u = (d11 * d02 - d01 * d12) * inv;
            const float v = (d00 * d12 - d01 * d02) * inv;
            if (u >= 0 && v >= 0 && u + v <= 1.0f) {
                const float sgn = sd < 0 ? -1.f : 1.f;
                for (int k = 0; k < 3; ++k) hit[k] = ctr[k] + n[k] * (r - dist) * sgn;
                found = true;
            }
        }
        // outer half-cylinder of an edge
        for (int i = 0; i < 3 && !found; ++i) {
            const float* Bg = V[i];
            const float* En = V[(i + 1) % 3];
            float ed[3] = {En[0] - Bg[0], En[1] - Bg[1], En[2] - Bg[2]};
            const float el = sqrtf(ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]);
            ed[0] /= el;
            ed[1] /= el;
            ed[2] /= el;
            const float tt = (ctr[0] - Bg[0]) * ed[0] + (ctr[1] - Bg[1]) * ed[1] + (ctr[2] - Bg[2]) * ed[2];
            if (tt < 0 || tt > el) continue;
            const float cl[3] = {Bg[0] + ed[0] * tt, Bg[1] + ed[1] * tt, Bg[2] + ed[2] * tt};
            float rad[3] = {ctr[0] - cl[0], ctr[1] - cl[1], ctr[2] - cl[2]};
            const float rl = sqrtf(rad[0] * rad[0] + rad[1] * rad[1] + rad[2] * rad[2]);
            if (rl >= r) continue;
            const float* Ot = V[(i + 2) % 3];
            const float bo[3] = {Ot[0] - Bg[0], Ot[1] - Bg[1], Ot[2] - Bg[2]};
            const float bp[3] = {proj[0] - Bg[0], proj[1] - Bg[1], proj[2] - Bg[2]};
            const float c1[3] = {ed[1] * bo[2] - ed[2] * bo[1], ed[2] * bo[0] - ed[0] * bo[2], ed[0] * bo[1] - ed[1] * bo[0]};
            const float c2[3] = {ed[1] * bp[2] - ed[2] * bp[1], ed[2] * bp[0] - ed[0] * bp[2], ed[0] * bp[1] - ed[1] * bp[0]};
            if (c1[0] * c2[0] + c1[1] * c2[1] + c1[2] * c2[2] >= 0) continue;   // inner half-cylinder
            rad[0] /= rl;
            rad[1] /= rl;
            rad[2] /= rl;
            for (int k = 0; k < 3; ++k) hit[k] = cl[k] + rad[k] * r;
            found = true;
        }
        // vertex sphere
        for (int i = 0; i < 3 && !found; ++i) {
            float vo[3] = {ctr[0] - V[i][0], ctr[1] - V[i][1], ctr[2] - V[i][2]};
            const float vl = sqrtf(vo[0] * vo[0] + vo[1] * vo[1] + vo[2] * vo[2]);
            if (vl > r) continue;
            vo[0] /= vl;
            vo[1] /= vl;
            vo[2] /= vl;
            for (int k = 0; k < 3; ++k) hit[k] = V[i][k] + vo[k] * r;
            found = true;
        }
        if (!found) continue;
        mx += ctr[0] - hit[0];
        my += ctr[1] - hit[1];
        mz += ctr[2] - hit[2];
        cnt += 1.f;
    }
    push[f] = make_float4(mx, my, mz, cnt);
}

// x = prev = sum_k w_k src[id_k] (updatePointInTet, PDSolver.cu:724-743): the
// fine level from the coarse one (runInterpolate) and back (runAverage).
__global__ void k_tl_transfer(int n, const int4* __restrict__ ids, const float4* __restrict__ w,
                              const float4* __restrict__ src, float4* __restrict__ x, float4* __restrict__ prev) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 id = __ldg(ids + i);
    const float4 c = __ldg(w + i);
    const float4 p0 = src[id.x], p1 = src[id.y], p2 = src[id.z], p3 = src[id.w];
    const float4 q = make_float4(c.x * p0.x + c.y * p1.x + c.z * p2.x + c.w * p3.x,
                                 c.x * p0.y + c.y * p1.y + c.z * p2.y + c.w * p3.y,
                                 c.x * p0.z + c.y * p1.z + c.z * p2.z + c.w * p3.z, 0.f);
    x[i] = q;
    prev[i] = q;
}

// Fine-vertex weights recomputed from the current positions in the same coarse
// tet (updateMapping, PDSolver.cu:764-793; barycentricCoordinate utils.cu:335-364).
__global__ void k_tl_update_mapping(int n, const float4* __restrict__ xf, const int4* __restrict__ ids,
                                    const float4* __restrict__ xc, float4* __restrict__ w) {
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 id = __ldg(ids + i);
    const float4 P4 = xf[i];
    const float4 v4[4] = {xc[id.x], xc[id.y], xc[id.z], xc[id.w]};
    float v[4][3];
    for (int k = 0; k < 4; ++k) {
        v[k][0] = v4[k].x;
        v[k][1] = v4[k].y;
        v[k][2] = v4[k].z;
    }
    const float e1[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
    const float e2[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
    const float e3[3] = {v[3][0] - v[0][0], v[3][1] - v[0][1], v[3][2] - v[0][2]};
    const float vol = (e1[0] * (e2[1] * e3[2] - e2[2] * e3[1]) + e1[1] * (e2[2] * e3[0] - e2[0] * e3[2]) +
                       e1[2] * (e2[0] * e3[1] - e2[1] * e3[0])) / 6.0f;
    const float ctr[3] = {(v[0][0] + v[1][0] + v[2][0] + v[3][0]) * 0.25f, (v[0][1] + v[1][1] + v[2][1] + v[3][1]) * 0.25f,
                          (v[0][2] + v[1][2] + v[2][2] + v[3][2]) * 0.25f};
    const float pc[3] = {P4.x - ctr[0], P4.y - ctr[1], P4.z - ctr[2]};
    float out[4];
    for (int i4 = 0; i4 < 4; ++i4) {
        const float* q = v[i4];
        const float* f0 = v[(i4 + 1) % 4];
        const float* f1 = v[(i4 + 2) % 4];
        const float* f2 = v[(i4 + 3) % 4];
        const float a[3] = {f1[0] - f0[0], f1[1] - f0[1], f1[2] - f0[2]};
        const float b[3] = {f2[0] - f0[0], f2[1] - f0[1], f2[2] - f0[2]};
        float nrm[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        if (nrm[0] * (q[0] - f0[0]) + nrm[1] * (q[1] - f0[1]) + nrm[2] * (q[2] - f0[2]) > 0) {
            nrm[0] = -nrm[0];
            nrm[1] = -nrm[1];
            nrm[2] = -nrm[2];
        }
        const float l = sqrtf(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        const float area = l * 0.5f;
        out[i4] = 0.25f - (pc[0] * nrm[0] / l + pc[1] * nrm[1] / l + pc[2] * nrm[2] / l) * area / (3.f * vol);
    }
    w[i] = make_float4(out[0], out[1], out[2], out[3]);
}

}  // namespace mgsb
