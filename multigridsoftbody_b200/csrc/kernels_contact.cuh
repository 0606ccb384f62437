// Uniform-grid broad phase for the tool contact of the multigrid kinds
// (sm_100a).  Included by solver.cu only.
//
// Each body has a fixed uniform grid over its rest bounding box (one cell of
// margin).  Every frame the surface vertices are binned by their predicted
// positions with a counting sort (count -> per-body exclusive scan, one CTA
// per body -> scatter); coordinates outside the grid are clamped into the boundary
// cells, and the query clamps the same way, so a vertex inside the query box
// is always found.  Each body's capsule then visits only the cells its
// swept box (segment AABB grown by the radius and a small margin) covers.
// The candidates are recorded (per-vertex flag + list, so the next frame
// resets exactly them); in the FP32 kind the narrow phase (capsule_test, the
// same test the brute-force kernel runs) writes the contact state of every
// candidate, in the mixed kind k_mx_contact_frame tests only the flagged
// vertices in FP64.  Vertices that are never candidates keep the zero state
// the brute-force kernel would write for them.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace mgsb {

struct BpGrid {
    float ox, oy, oz, inv_h;   // origin and 1 / cell size
    int nx, ny, nz, cell_off;  // cells per axis, first cell of this body (counts)
    int start_off;             // first entry of this body's cell starts (cell_off + body: n + 1 entries each)
    int sorted_off;            // first slot of this body's surface vertices in the sorted list
};

constexpr int kBpScanThreads = 1024;

__device__ __forceinline__ int bp_axis(float x, float o, float inv_h, int n) {
    const int i = __float2int_rd((x - o) * inv_h);   // saturating; NaN -> 0
    return min(max(i, 0), n - 1);
}

// Body-local cell index of a point (clamped into the grid).
__device__ __forceinline__ int bp_cell(const BpGrid& g, float x, float y, float z) {
    const int ix = bp_axis(x, g.ox, g.inv_h, g.nx), iy = bp_axis(y, g.oy, g.inv_h, g.ny),
              iz = bp_axis(z, g.oz, g.inv_h, g.nz);
    return (iz * g.ny + iy) * g.nx + ix;
}

// Reset the previous frame's candidates (flag, and in the FP32 kind their
// contact state) and zero the cell counts.
__global__ void k_bp_clear(int ncells, int32_t* __restrict__ counts, const int32_t* __restrict__ list,
                           const int32_t* __restrict__ nlist, uint8_t* __restrict__ cand, int32_t* __restrict__ cflag,
                           float* __restrict__ c0, float4* __restrict__ target) {
    pdl_enter();
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncells; i += stride) counts[i] = 0;
    const int nl = *nlist;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += stride) {
        const int v = list[i];
        cand[v] = 0;
        if (cflag) {
            cflag[v] = 0;
            c0[v] = 0.f;
            target[v] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// Cell and rank of every surface vertex (x: index of its cell's start
// entry); also restarts the candidate list.
__global__ void k_bp_bin(int ns, const int32_t* __restrict__ surf, const int32_t* __restrict__ body_of,
                         const BpGrid* __restrict__ grids, const float4* __restrict__ s, int32_t* __restrict__ counts,
                         int2* __restrict__ cellrank, int32_t* __restrict__ nlist) {
    pdl_enter();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q == 0) *nlist = 0;
    if (q >= ns) return;
    const int v = __ldg(surf + q);
    const float4 p = __ldg(s + v);
    const BpGrid& g = grids[__ldg(body_of + v)];
    const int c = bp_cell(g, p.x, p.y, p.z);
    cellrank[q] = make_int2(g.start_off + c, atomicAdd(counts + g.cell_off + c, 1));
}

// Exclusive scan of one body's cell counts per CTA, in coalesced tiles of
// blockDim cells with a running carry: start[start_off + c] = sorted_off +
// vertices in the body's cells before c; start[start_off + n] = the end.
__global__ void __launch_bounds__(kBpScanThreads) k_bp_scan(const BpGrid* __restrict__ grids,
                                                           const int32_t* __restrict__ counts,
                                                           int32_t* __restrict__ start) {
    pdl_enter();
    __shared__ int warp_tot[kBpScanThreads / 32];
    const BpGrid g = grids[blockIdx.x];
    const int n = g.nx * g.ny * g.nz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int carry = g.sorted_off;
    for (int t0 = 0; t0 < n; t0 += blockDim.x) {
        const int i = t0 + threadIdx.x;
        const int c = i < n ? counts[g.cell_off + i] : 0;
        int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < nw) warp_tot[lane] = t;
        }
        __syncthreads();
        const int incl = x + (warp > 0 ? warp_tot[warp - 1] : 0);
        if (i < n) start[g.start_off + i] = carry + incl - c;
        carry += warp_tot[nw - 1];
        __syncthreads();   // warp_tot is rewritten by the next tile
    }
    if (threadIdx.x == 0) start[g.start_off + n] = carry;
}

__global__ void k_bp_scatter(int ns, const int32_t* __restrict__ surf, const int2* __restrict__ cellrank,
                             const int32_t* __restrict__ start, int32_t* __restrict__ sorted) {
    pdl_enter();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ns) return;
    const int2 cr = cellrank[q];
    sorted[__ldg(start + cr.x) + cr.y] = __ldg(surf + q);
}

// One CTA per body: the cells of the capsule's swept box; every vertex there
// becomes a candidate, and with cflag set (FP32 kind) gets the narrow phase.
__global__ void k_bp_query(const BpGrid* __restrict__ grids, const BodyDev* __restrict__ bodies,
                           const int32_t* __restrict__ start, const int32_t* __restrict__ sorted,
                           const float4* __restrict__ s, const float* __restrict__ fixf, float kc,
                           uint8_t* __restrict__ cand, int32_t* __restrict__ list, int32_t* __restrict__ nlist,
                           int32_t* __restrict__ cflag, float* __restrict__ c0, float4* __restrict__ target) {
    pdl_enter();
    const BpGrid g = grids[blockIdx.x];
    const BodyDev& B = bodies[blockIdx.x];
    const float r = B.cap_r;
    if (!(r > 0.f)) return;
    float lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float m = r + 1e-4f + 1e-6f * fmaxf(fabsf(B.cap_a[k]), fabsf(B.cap_b[k]));
        lo[k] = fminf(B.cap_a[k], B.cap_b[k]) - m;
        hi[k] = fmaxf(B.cap_a[k], B.cap_b[k]) + m;
    }
    const int x0 = bp_axis(lo[0], g.ox, g.inv_h, g.nx), x1 = bp_axis(hi[0], g.ox, g.inv_h, g.nx);
    const int y0 = bp_axis(lo[1], g.oy, g.inv_h, g.ny), y1 = bp_axis(hi[1], g.oy, g.inv_h, g.ny);
    const int z0 = bp_axis(lo[2], g.oz, g.inv_h, g.nz), z1 = bp_axis(hi[2], g.oz, g.inv_h, g.nz);
    const int wx = x1 - x0 + 1, wy = y1 - y0 + 1, ncell = wx * wy * (z1 - z0 + 1);
    for (int k = threadIdx.x; k < ncell; k += blockDim.x) {
        const int ix = x0 + k % wx, iy = y0 + (k / wx) % wy, iz = z0 + k / (wx * wy);
        const int c = g.start_off + (iz * g.ny + iy) * g.nx + ix;
        for (int j = start[c]; j < start[c + 1]; ++j) {
            const int v = sorted[j];
            cand[v] = 1;
            list[atomicAdd(nlist, 1)] = v;
            if (cflag) {
                int flag;
                float4 tg;
                capsule_test(__ldg(s + v), B, flag, tg);
                cflag[v] = flag;
                c0[v] = (flag && __ldg(fixf + v) != 0.f) ? kc : 0.f;
                target[v] = tg;
            }
        }
    }
}

}  // namespace mgsb
