// Stand-in for the reference's MultiGridSoftBody/src/global.h when its solver
// sources are compiled headless (no GUI, renderer, glog or CSV set-up).
// Written for this build; declares only what the solver translation units use.
#pragma once
#define PRINT_CUDA_ERROR_AFTER(func)
#define BLOCK_SIZE(eleNum, threadNum) (((eleNum) + (threadNum) - 1) / (threadNum))

#include <cassert>
#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "simpleMath.h"
#include "Simulator.h"

namespace mgsb_ref_shim {
struct NullLog {
    template <typename T>
    NullLog& operator<<(const T&) { return *this; }
};
}  // namespace mgsb_ref_shim
#define LOG(severity) (mgsb_ref_shim::NullLog())

using namespace std;
extern FILE* timeOutputFile_physical;
extern FILE* energyOutputFile;
extern float g_conEnergy_V2;
extern double duration_physical;
extern double duration_physicalInner;
extern int g_stepCnt;
extern std::chrono::high_resolution_clock::time_point g_systemBeginTime;
extern Simulator* g_simulator;
void printCudaError(const char* funcName);
void OutputPosNormIndex(string filepath, vector<float> pos, vector<float> norm, vector<unsigned int> index);
