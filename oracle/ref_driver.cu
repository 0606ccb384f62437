// C-ABI driver around the reference's own solver classes, compiled together
// with the reference sources (MultiGridSoftBody/src) by oracle/ref_build.sh
// into oracle/_ref/libmgsb_ref.so.  TEST INFRASTRUCTURE ONLY: it pins the
// oracle against the reference itself (precompute and polar decomposition on
// the CPU; whole frames of PDSolver::Step on a GPU).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "global.h"
#include "PDSolver.h"
#include "PDSolver_MG.h"
#include "SoftObject.h"
#include "Simulator.h"

// Globals the reference's solver translation units reference (global.h).
FILE* timeOutputFile_physical = nullptr;
FILE* energyOutputFile = nullptr;
float g_conEnergy_V2 = 0.f;
int g_stepCnt = 0;
std::chrono::high_resolution_clock::time_point g_systemBeginTime = std::chrono::high_resolution_clock::now();
Simulator* g_simulator = nullptr;

// Simulator.cpp is not compiled (it pulls in GLFW); the singleton accessor is
// the only member the solver path needs.
Simulator& Simulator::GetInstance() {
    static Simulator instance;
    return instance;
}

static void ensure_globals() {
    if (!timeOutputFile_physical) timeOutputFile_physical = std::fopen("/dev/null", "w");
    if (!energyOutputFile) energyOutputFile = std::fopen("/dev/null", "w");
    if (!g_simulator) g_simulator = &Simulator::GetInstance();
}

extern "C" {

// PDSolver::InitVolumeConstraint (PDSolver.cpp:12-132) on the host, FP32.
int ref_precompute(const float* pos, int V, const int32_t* tets, int T, float stiffness, float* inv, float* ac,
                   float* vol, float* mass, float* diag) {
    ensure_globals();
    PDSolver s;
    s.m_tetVertNum = V;
    s.m_tetNum = T;
    s.m_volumnStiffness = stiffness;
    s.m_tetVertPos.assign(pos, pos + 3 * (size_t)V);
    s.m_tetIndex.assign(tets, tets + 4 * (size_t)T);
    s.InitVolumeConstraint();
    for (size_t i = 0; i < s.m_tetInvD3x3.size(); ++i) inv[i] = s.m_tetInvD3x3[i];
    for (size_t i = 0; i < s.m_tetInvD3x4.size(); ++i) ac[i] = s.m_tetInvD3x4[i];
    for (int t = 0; t < T; ++t) vol[t] = s.m_tetVolume[t];
    for (int i = 0; i < V; ++i) {
        mass[i] = s.m_tetVertMass[i];
        diag[i] = s.m_tetVolumeDiag[i];
    }
    return 0;
}

// GetRotation_D (utils.cu:123-226), host build, FP32.
void ref_rotation(const float* F, float* R, float* det) {
    float Fm[3][3], Rm[3][3];
    for (int i = 0; i < 9; ++i) Fm[i / 3][i % 3] = F[i];
    float d = 0.f;
    GetRotation_D(Fm, Rm, d);
    for (int i = 0; i < 9; ++i) R[i] = Rm[i / 3][i % 3];
    if (det) *det = d;
}

// Matrix_Inverse_3 (utils.cu:233-252); callers must not pass |det| < 1e-6.
float ref_inverse3(const float* A, float* R) {
    float a[9];
    for (int i = 0; i < 9; ++i) a[i] = A[i];
    return Matrix_Inverse_3(a, R);
}

// barycentricCoordinate (utils.cu:335-364).
void ref_barycentric(const float* p, const float* a, const float* b, const float* c, const float* d, float* w) {
    Point3D P(p[0], p[1], p[2]), A(a[0], a[1], a[2]), B(b[0], b[1], b[2]), Cc(c[0], c[1], c[2]), D(d[0], d[1], d[2]);
    barycentricCoordinate(P, A, B, Cc, D, w);
}

// SoftObject::ReadFromFile (.msh part) + TetFaceExtraction.  Two calls: the
// first (out == NULL) returns the counts.
static std::unique_ptr<SoftObject> g_obj;
int ref_read_msh(const char* path, int* V, int* T, int* F) {
    ensure_globals();
    g_obj.reset(new SoftObject("ref", "/nonexistent-mgsb.obj", path, "/dev/null"));
    g_obj->ReadFromFile();
    g_obj->TetFaceExtraction();
    *V = (int)(g_obj->m_tetVertPosORIG.size() / 3);
    *T = (int)(g_obj->m_tetIdxORIG.size() / 4);
    *F = (int)(g_obj->m_tetFaceIdx.size() / 3);
    return 0;
}

void ref_read_msh_arrays(float* pos, int32_t* tets, int32_t* tris, int32_t* opp) {
    for (size_t i = 0; i < g_obj->m_tetVertPosORIG.size(); ++i) pos[i] = g_obj->m_tetVertPosORIG[i];
    for (size_t i = 0; i < g_obj->m_tetIdxORIG.size(); ++i) tets[i] = g_obj->m_tetIdxORIG[i];
    for (size_t i = 0; i < g_obj->m_tetFaceIdx.size(); ++i) tris[i] = (int32_t)g_obj->m_tetFaceIdx[i];
    for (size_t i = 0; i < g_obj->m_tetFaceOppositeTetVertIdx.size(); ++i) opp[i] = (int32_t)g_obj->m_tetFaceOppositeTetVertIdx[i];
}

// TetFaceExtraction on given tets (no file read).
int ref_extract_surface(const float* pos, int V, const int32_t* tets, int T, int32_t* tris, int32_t* opp, int cap) {
    ensure_globals();
    SoftObject so("ref", "", "", "/dev/null");
    so.m_tetVertPosORIG.assign(pos, pos + 3 * (size_t)V);
    so.m_tetIdxORIG.assign(tets, tets + 4 * (size_t)T);
    so.TetFaceExtraction();
    const int F = (int)(so.m_tetFaceIdx.size() / 3);
    if (tris && opp && F <= cap) {
        for (int i = 0; i < 3 * F; ++i) tris[i] = (int32_t)so.m_tetFaceIdx[i];
        for (int i = 0; i < F; ++i) opp[i] = (int32_t)so.m_tetFaceOppositeTetVertIdx[i];
    }
    return F;
}

// Run PDSolver::Step (PDSolver.cpp:243-293) for `frames` frames on the GPU.
// fixed: 1 = fixed.  sphere: per frame (cx, cy, cz, r); r <= 0 = inactive.
// Outputs per frame: positions (3V floats) and contact flags (V ints);
// ms[f] = wall time of Step() (it synchronises internally).  Returns 0 or a
// CUDA error code.
int ref_run(const float* pos, int V, const int32_t* tets, int T, const uint8_t* fixed, int iters, int frames,
            const float* sphere, float* out_pos, int32_t* out_flags, float* ms) {
    ensure_globals();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return -1;
    Simulator* sim = g_simulator;
    sim->m_sphereFixers.clear();
    sim->m_sphereColliders.clear();
    sim->m_sphereColliders.push_back(std::shared_ptr<SphereCollider>(new SphereCollider({0.f, 0.f, 0.f}, 1.f)));
    SoftObject so("ref", "", "", "/dev/null");
    so.m_tetVertPosORIG.assign(pos, pos + 3 * (size_t)V);
    so.m_tetIdxORIG.assign(tets, tets + 4 * (size_t)T);
    so.TetFaceExtraction();
    const int F = (int)(so.m_tetFaceIdx.size() / 3);
    sim->m_tetVertPos = so.m_tetVertPosORIG;
    sim->m_tetFaceIdx = so.m_tetFaceIdx;
    sim->m_normal.assign(3 * (size_t)V, 0.f);
    sim->m_tetVertIsCollide.assign(V, 0);
    sim->m_tetVertCollisionDepth.assign(V, 0.f);
    sim->m_triIsCollide.assign(F, 0);
    sim->m_triMoveVec.assign(3 * (size_t)F, 0.f);
    PDSolver* s = new PDSolver();
    s->Init(so.m_tetVertPosORIG, so.m_tetIdxORIG, so.m_tetFaceIdx, so.m_tetFaceOppositeTetVertIdx);
    s->m_iterNum = iters;
    std::vector<float> fixf(V);
    for (int i = 0; i < V; ++i) fixf[i] = fixed && fixed[i] ? 0.0f : 1.0f;
    s->m_tetVertFixed = fixf;
    cudaMemcpy(s->pdSolverData->tetVertFixed_d, fixf.data(), V * sizeof(float), cudaMemcpyHostToDevice);
    cudaDeviceSynchronize();
    for (int f = 0; f < frames; ++f) {
        SphereCollider& sp = *sim->m_sphereColliders[0];
        sp.m_position = Point3D(sphere[4 * f], sphere[4 * f + 1], sphere[4 * f + 2]);
        sp.m_radius = sphere[4 * f + 3] > 0 ? sphere[4 * f + 3] : 1.f;
        sp.m_active = sphere[4 * f + 3] > 0;
        auto t0 = std::chrono::high_resolution_clock::now();
        s->Step();
        cudaDeviceSynchronize();
        auto t1 = std::chrono::high_resolution_clock::now();
        if (ms) ms[f] = std::chrono::duration<float, std::milli>(t1 - t0).count();
        if (out_pos)
            for (int i = 0; i < 3 * V; ++i) out_pos[(size_t)f * 3 * V + i] = sim->m_tetVertPos[i];
        if (out_flags)
            for (int i = 0; i < V; ++i) out_flags[(size_t)f * V + i] = sim->m_tetVertIsCollide[i];
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

// PDSolver_MG (the two-level schedule) on a coarse and a fine mesh of one body:
// per frame the sphere pose, one Step, then the fine and coarse positions.
int ref_mg2_run(const float* cpos, int cV, const int32_t* ctets, int cT, const float* fpos, int fV,
                const int32_t* ftets, int fT, const uint8_t* cfixed, const uint8_t* ffixed, int frames,
                const float* sphere, float* out_fine, float* out_coarse, float* ms) {
    ensure_globals();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return -1;
    Simulator* sim = g_simulator;
    sim->m_sphereFixers.clear();
    sim->m_sphereColliders.clear();
    sim->m_sphereColliders.push_back(std::shared_ptr<SphereCollider>(new SphereCollider({0.f, 0.f, 0.f}, 1.f)));
    SoftObject co("coarse", "", "", "/dev/null"), fo("fine", "", "", "/dev/null");
    co.m_tetVertPosORIG.assign(cpos, cpos + 3 * (size_t)cV);
    co.m_tetIdxORIG.assign(ctets, ctets + 4 * (size_t)cT);
    co.TetFaceExtraction();
    fo.m_tetVertPosORIG.assign(fpos, fpos + 3 * (size_t)fV);
    fo.m_tetIdxORIG.assign(ftets, ftets + 4 * (size_t)fT);
    fo.TetFaceExtraction();
    const int F = (int)(fo.m_tetFaceIdx.size() / 3);
    sim->m_tetVertPos = fo.m_tetVertPosORIG;
    sim->m_tetFaceIdx = fo.m_tetFaceIdx;
    sim->m_normal.assign(3 * (size_t)fV, 0.f);
    sim->m_tetVertIsCollide.assign(fV, 0);
    sim->m_tetVertCollisionDepth.assign(fV, 0.f);
    sim->m_triIsCollide.assign(F, 0);
    sim->m_triMoveVec.assign(3 * (size_t)F, 0.f);
    // PDSolver_MG::Step ends with runCalEnergy(..., true), which fills these per fine vertex
    sim->m_tetVertEpDensity.assign(fV, 0.f);
    sim->m_tetVertEpSum.assign(fV, 0.f);
    sim->m_tetVertVSum.assign(fV, 0.f);
    PDSolver_MG* mg = new PDSolver_MG();
    mg->Init(co.m_tetVertPosORIG, co.m_tetIdxORIG, co.m_tetFaceIdx, co.m_tetFaceOppositeTetVertIdx, fo.m_tetVertPosORIG,
             fo.m_tetIdxORIG, fo.m_tetFaceIdx, fo.m_tetFaceOppositeTetVertIdx);
    auto set_fixed = [](PDSolver* s, const uint8_t* mask, int V) {
        std::vector<float> fixf(V);
        for (int i = 0; i < V; ++i) fixf[i] = mask && mask[i] ? 0.0f : 1.0f;
        s->m_tetVertFixed = fixf;
        cudaMemcpy(s->pdSolverData->tetVertFixed_d, fixf.data(), V * sizeof(float), cudaMemcpyHostToDevice);
    };
    set_fixed(mg->m_pdSolverCoarse, cfixed, cV);
    set_fixed(mg->m_pdSolverFine, ffixed, fV);
    cudaDeviceSynchronize();
    for (int f = 0; f < frames; ++f) {
        SphereCollider& sp = *sim->m_sphereColliders[0];
        sp.m_position = Point3D(sphere[4 * f], sphere[4 * f + 1], sphere[4 * f + 2]);
        sp.m_radius = sphere[4 * f + 3] > 0 ? sphere[4 * f + 3] : 1.f;
        sp.m_active = sphere[4 * f + 3] > 0;
        auto t0 = std::chrono::high_resolution_clock::now();
        mg->Step();
        cudaDeviceSynchronize();
        auto t1 = std::chrono::high_resolution_clock::now();
        if (ms) ms[f] = std::chrono::duration<float, std::milli>(t1 - t0).count();
        if (out_fine)
            cudaMemcpy(out_fine + (size_t)f * 3 * fV, mg->m_pdSolverFine->pdSolverData->tetVertPos_d,
                       3 * (size_t)fV * sizeof(float), cudaMemcpyDeviceToHost);
        if (out_coarse)
            cudaMemcpy(out_coarse + (size_t)f * 3 * cV, mg->m_pdSolverCoarse->pdSolverData->tetVertPos_d,
                       3 * (size_t)cV * sizeof(float), cudaMemcpyDeviceToHost);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
