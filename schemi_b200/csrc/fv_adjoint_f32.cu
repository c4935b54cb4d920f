// Adjoint step kernels of the FP32-flux step: face-state and flux reverse arithmetic in FP32,
// the adjoint state accumulated in FP64 (1..4 species, 2D and 3D).
#define FV_T float
#define FV_ADJ_LAUNCH_NAME launchAdjointF32
#include "fv_adjoint_inst.inc"
