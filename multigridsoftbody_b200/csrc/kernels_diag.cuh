// Diagnostics read back on demand (not part of a frame): surface vertex
// normals and the energy/convergence reduction.
//
//   normals   UpdateTriNormal + AvgOutsideTetVertNormal (PDSolver.cu:394-460).
//             The reference scatters each triangle normal into its three
//             vertices with float atomics; here the triangle normals go to a
//             scratch array and every surface vertex gathers its triangles
//             through a vertex->triangle CSR (ascending triangle order), so the
//             result does not depend on scheduling.
//   energy    runCalEnergy (PDSolver.cu:816-924): Ek = sum m|x-s|^2/(2h^2),
//             Ep = sum w/2 ||F-R||_F^2, Ec, contact count, and |x-prev| (the
//             reference kind) or the fine-level residual norm of the last
//             global step (multigrid kinds).  The reference copies the state to
//             the host and loops there; here one grid-strided kernel writes FP64
//             per-block partial sums to scratch and one block sums them in a
//             fixed order (deterministic).
#pragma once

#include <cfloat>
#include <cstdint>

#include "device_math.cuh"

namespace mgsb {

// ---------------------------------------------------------------------------
// normals
// ---------------------------------------------------------------------------
// Unit normal of each surface triangle (a, b, c): (b-a) x (c-a) / |.|, as the
// reference's normalize (utils.cu:293) divides without an epsilon test.
__global__ void __launch_bounds__(256) k_tri_normals(int nf, const int4* __restrict__ tris, const float4* __restrict__ x,
                                                     float4* __restrict__ fn) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int4 t = __ldg(tris + f);
    const float4 a = __ldg(x + t.x), b = __ldg(x + t.y), c = __ldg(x + t.z);
    const float ab[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
    const float ac[3] = {c.x - a.x, c.y - a.y, c.z - a.z};
    const float n[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
    const float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    fn[f] = make_float4(n[0] / len, n[1] / len, n[2] / len, 0.f);
}

// Per surface vertex j: sum of its triangles' normals (vertex->triangle CSR,
// triangle ids local to the body), divided by the length when it exceeds
// FLT_EPSILON (AvgOutsideTetVertNormal).
__global__ void __launch_bounds__(256) k_vert_normals(int nsv, const int32_t* __restrict__ ptr,
                                                      const int32_t* __restrict__ fidx, const float4* __restrict__ fn,
                                                      float4* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nsv) return;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    const int e1 = __ldg(ptr + j + 1);
    for (int e = __ldg(ptr + j); e < e1; ++e) {
        const float4 n = fn[__ldg(fidx + e)];
        sx += n.x;
        sy += n.y;
        sz += n.z;
    }
    const float len = sqrtf(sx * sx + sy * sy + sz * sz);
    if (len > FLT_EPSILON) {
        sx /= len;
        sy /= len;
        sz /= len;
    }
    out[j] = make_float4(sx, sy, sz, 0.f);
}

// ---------------------------------------------------------------------------
// energy
// ---------------------------------------------------------------------------
constexpr int kEnergyBlocks = 592;   // 4 x 148 SMs; grid-stride over vertices and tets
constexpr int kEnergyThreads = 256;
constexpr int kEnergyTerms = 5;      // Ek, Ep, Ec, Nc, (dX^2 | r^2)

enum EnergyKind : int { kEnergyReference = 0, kEnergyMultigrid = 1, kEnergyMixed = 2 };

struct EnergyArgs {
    int kind;
    int v0, nv, t0, nt;
    double inv_2h2;
    float kv;                                   // reference kind: volume stiffness
    const float4 *x, *s, *prev;                 // FP32 state (prev: reference kind)
    const double4 *x64, *s64;                   // mixed precision state
    const float *mass, *fixf;
    const int4* tets;
    const float4 *tA, *tB;                      // per tet: gradient rows + weight (multigrid)
    const float2* tC;                           //   or inverse rest matrix + volume (reference)
    const int32_t* cflag;
    const float *c0, *cenergy;
    const float4* target;
    // fine-level residual of the last global step (multigrid kinds; residual = 0
    // before the first frame)
    int residual, S;
    const int32_t *sp, *col;
    const float *val, *dfull;                   // FP32: D includes the contact stiffness
    const float4 *b, *d;
    const double *val64, *diag64;               // mixed: D = diag64 + c0
    const double4 *b64, *d64;
};

__device__ __forceinline__ double4 ld_state(const float4* p32, const double4* p64, int i) {
    if (p64) return p64[i];
    const float4 v = p32[i];
    return make_double4(v.x, v.y, v.z, 0.0);
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;   // valid in thread 0
}

// partial[k * gridDim.x + block] for the five terms.
__global__ void __launch_bounds__(kEnergyThreads) k_energy_partial(EnergyArgs a, double* __restrict__ partial) {
    __shared__ double red[kEnergyThreads / 32];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const bool mg = a.kind != kEnergyReference;
    double ek = 0.0, ep = 0.0, ec = 0.0, nc = 0.0, r2 = 0.0;
    for (int i = tid; i < a.nv; i += stride) {
        const int gi = a.v0 + i;
        const double4 x = ld_state(a.x, a.x64, gi), s = ld_state(a.s, a.s64, gi);
        const double dx = x.x - s.x, dy = x.y - s.y, dz = x.z - s.z;
        ek += (double)a.mass[gi] * (dx * dx + dy * dy + dz * dz);
        if (a.cflag[gi] > 0) nc += 1.0;
        if (!mg) {
            const float4 pv = a.prev[gi];
            const double px = x.x - pv.x, py = x.y - pv.y, pz = x.z - pv.z;
            r2 += px * px + py * py + pz * pz;
            ec += (double)a.cenergy[gi];
            continue;
        }
        const float c = a.c0[gi];
        if (c > 0.f) {
            const float4 tg = a.target[gi];
            const double qx = x.x - tg.x, qy = x.y - tg.y, qz = x.z - tg.z;
            ec += 0.5 * (double)c * (qx * qx + qy * qy + qz * qz);
        }
        if (!a.residual || a.fixf[gi] == 0.f) continue;
        // r = b - (D d + sum_offdiag a_ij d_j), sliced-ELL row walk
        const int slice = gi / a.S;
        const int beg = a.sp[slice], end = a.sp[slice + 1];
        double ax = 0.0, ay = 0.0, az = 0.0;
        double4 di, bi;
        double D;
        if (a.kind == kEnergyMixed) {
            for (int q = beg + (gi - slice * a.S); q < end; q += a.S) {
                const double v = a.val64[q];
                const double4 dj = a.d64[a.col[q]];
                ax += v * dj.x; ay += v * dj.y; az += v * dj.z;
            }
            di = a.d64[gi];
            bi = a.b64[gi];
            D = a.diag64[gi] + (double)c;
        } else {
            for (int q = beg + (gi - slice * a.S); q < end; q += a.S) {
                const double v = a.val[q];
                const float4 dj = a.d[a.col[q]];
                ax += v * dj.x; ay += v * dj.y; az += v * dj.z;
            }
            const float4 d4 = a.d[gi], b4 = a.b[gi];
            di = make_double4(d4.x, d4.y, d4.z, 0.0);
            bi = make_double4(b4.x, b4.y, b4.z, 0.0);
            D = a.dfull[gi];
        }
        const double rx = bi.x - (D * di.x + ax), ry = bi.y - (D * di.y + ay), rz = bi.z - (D * di.z + az);
        r2 += rx * rx + ry * ry + rz * rz;
    }
    for (int t = tid; t < a.nt; t += stride) {
        const int gt = a.t0 + t;
        const int4 id = a.tets[gt];
        const double4 p0 = ld_state(a.x, a.x64, id.x), p1 = ld_state(a.x, a.x64, id.y), p2 = ld_state(a.x, a.x64, id.z),
                      p3 = ld_state(a.x, a.x64, id.w);
        const float4 A = a.tA[gt], B = a.tB[gt];
        const float2 C = a.tC[gt];
        // rows of the inverse rest matrix (the multigrid gradients g1..g3 are
        // the same rows): m = [[A.x A.y A.z] [A.w B.x B.y] [B.z B.w C.x]]
        const double m[9] = {A.x, A.y, A.z, A.w, B.x, B.y, B.z, B.w, C.x};
        const double e[3][3] = {{p1.x - p0.x, p2.x - p0.x, p3.x - p0.x},
                                {p1.y - p0.y, p2.y - p0.y, p3.y - p0.y},
                                {p1.z - p0.z, p2.z - p0.z, p3.z - p0.z}};
        float F[9], R[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) F[r * 3 + q] = (float)(e[r][0] * m[q] + e[r][1] * m[3 + q] + e[r][2] * m[6 + q]);
        if (mg)
            svd_rotation(F, R);
        else
            ref_rotation(F, R);
        double en = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const double df = (double)F[q] - (double)R[q];
            en += df * df;
        }
        ep += mg ? en * (double)C.y * 0.5 : en * (double)C.y * (double)a.kv * 0.5;
    }
    const double terms[kEnergyTerms] = {ek * a.inv_2h2, ep, ec, nc, r2};
#pragma unroll
    for (int k = 0; k < kEnergyTerms; ++k) {
        const double t = block_sum(terms[k], red);
        if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = t;
    }
}

// out[k] = sum over blocks of partial k (fixed order); out[4] = sqrt.
__global__ void __launch_bounds__(kEnergyThreads) k_energy_final(const double* __restrict__ partial, int nblk,
                                                                 double* __restrict__ out) {
    __shared__ double red[kEnergyThreads / 32];
    for (int k = 0; k < kEnergyTerms; ++k) {
        double v = 0.0;
        for (int j = threadIdx.x; j < nblk; j += blockDim.x) v += partial[k * nblk + j];
        const double t = block_sum(v, red);
        if (threadIdx.x == 0) out[k] = k == kEnergyTerms - 1 ? sqrt(t) : t;
    }
}

}  // namespace mgsb
