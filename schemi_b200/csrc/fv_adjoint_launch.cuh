// fv_adjoint_launch.cuh -- launchers of the adjoint step kernel, one per arithmetic
// (fv_adjoint_f64.cu: FP64; fv_adjoint_f32.cu: FP32 face arithmetic with FP64 adjoint
// accumulation, the reverse of the FP32-flux step).
#pragma once

#include "fv_adjoint.cuh"

namespace fv {

// Enqueues one adjoint step.  With A.U == nullptr and st == nullptr it only opts the kernel in
// to its dynamic shared memory (call once, outside any stream capture).
cudaError_t launchAdjointF64(int ns, int dims, const StepParams& P, const adj::AdjParams& A, cudaStream_t st);
cudaError_t launchAdjointF32(int ns, int dims, const StepParams& P, const adj::AdjParams& A, cudaStream_t st);

}  // namespace fv
