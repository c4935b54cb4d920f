// fv_launch.cuh -- host-side launchers of the step kernels, instantiated once per arithmetic
// (fv_f64.cu: FP64 without FMA contraction, fv_f32.cu: FP32 flux arithmetic).
#pragma once

#include "fv_generic.cuh"
#include "fv_warp2d.cuh"
#include "fv_warp2d64.cuh"

namespace fv {

// Tile shape of the fused march (chosen by the autotuner in fv_tune.cpp).
struct MarchShape {
    int bx;      // threads along x (incl. the 2 halo columns)
    int by;      // threads along y in 3D (incl. halo), 1 in 2D
    int rows;    // cells per CTA along the marching axis
    int warp;    // ensembles: every case runs the warp-strip march (FP32-flux 2D): 1, rows through
                 // registers; 2, rows through the shared-memory ring
};

struct StepBuffers {
    const double* U;
    double* Un;
    const double* prim0;
    DevClock* ck;
    double* blockMax;
    long long blockMaxCap;
    void* Pc;            // generic path: primitives (T)
    void* FS;            // generic path: face states (T)
    void* FL;            // generic path: face fluxes (T)
    GenericLayout L;
    const double* pcIn;  // FP64 warp strip: primitive cache of U (null: none)
    double* pcOut;       // FP64 warp strip: primitive cache of Un, written by a fused step
};

enum StepPath { PATH_MARCH = 0, PATH_GENERIC = 1 };

// Number of CTAs (= blockMax entries) one step writes.
long long marchBlocks(const StepParams& P, const MarchShape& s);
long long genericBlocks(const StepParams& P);

// Enqueue one step (without the finalize kernel).  Returns cudaSuccess or the launch error.
cudaError_t launchStepF64(const StepParams& P, const StepBuffers& B, int path, const MarchShape& s, cudaStream_t st);
cudaError_t launchStepF32(const StepParams& P, const StepBuffers& B, int path, const MarchShape& s, cudaStream_t st);

// Enqueue one ensemble step kernel over the case table (without the per-case finalize).
// With casesDev == nullptr and st == nullptr it only configures the kernel and returns, in
// *gridBlocks, the persistent grid size (SMs x resident CTAs).
cudaError_t launchBatchF64(int ns, int eos, int dims, const BatchCase* casesDev, int nCases, long long totalTiles,
                           const MarchShape& s, int* gridBlocks, cudaStream_t st);
cudaError_t launchBatchF32(int ns, int eos, int dims, const BatchCase* casesDev, int nCases, long long totalTiles,
                           const MarchShape& s, int* gridBlocks, cudaStream_t st);

// Shared memory of the fused march for a shape (bytes), per precision.
size_t marchSmemF64(int ns, int dims, const MarchShape& s);
size_t marchSmemF32(int ns, int dims, const MarchShape& s);

// Supported fused-march shapes.
bool marchShapeSupported(int dims, const MarchShape& s);

}  // namespace fv
