// FP64 adjoint step kernels (1..4 species, 2D and 3D).
#define FV_T double
#define FV_ADJ_LAUNCH_NAME launchAdjointF64
#include "fv_adjoint_inst.inc"
