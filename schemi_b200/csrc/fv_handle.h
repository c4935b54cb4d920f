// fv_handle.h -- private layout of the C-ABI handle (shared by fv_capi.cu and fv_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/fvstep.h"
#include "fv_chem_launch.h"
#include "fv_diffusion_launch.h"
#include "fv_launch.cuh"

using namespace fv;

extern "C" fv_status fv_set_march_shape(fv_handle* h, int bx, int by, int rows);

// Frees the recorded trajectory of a handle (fv_adjoint.cu); called by fv_destroy.
void releaseTrajectory(fv_handle* h);

struct fv_handle {
    fv_config cfg;
    StepParams P;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double* U[2] = {nullptr, nullptr};
    double* Ustage = nullptr;      // SecondOrderRK: state after the second stage
    double* conc = nullptr;        // SecondOrderRK / ThirdOrder: averaged concentrations c_0..c_N
    double* concStage = nullptr;   // ThirdOrder: concentrations of the 0.25 average
    int cur = 0;
    double* prim0 = nullptr;
    DevClock* ck = nullptr;        // device clock
    DevClock* ckHost = nullptr;    // pinned mirror
    double* blockMax = nullptr;
    long long blockMaxCap = 0;
    double* pc[2] = {nullptr, nullptr};  // FP64 warp strip: primitive cache of U[0] / U[1]
    double* geo = nullptr;         // all geometry tables
    void* Pc = nullptr;            // generic scratch
    void* FS = nullptr;
    void* FL = nullptr;
    GenericLayout L{};
    double* outBuf = nullptr;      // download staging
    int path = PATH_GENERIC;
    chem::ChemParams chem{};       // chemistry pass (cfg.chemistry != FV_CHEM_NONE)
    diff::DiffParams diff{};       // diffusion stage (cfg.diffusion): its buffers and coefficients
    MarchShape shape{128, 1, 32};
    int nConserved = 0;
    // graphs of step chunks, one per start buffer
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graphSteps = 0;
    // recorded trajectory of fv_record (checkpoints, per-step records, adjoint buffers)
    struct Trajectory* traj = nullptr;
    std::string err;
};
