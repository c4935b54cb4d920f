// FP32-flux instantiation of the step kernels: reconstruction, closures and fluxes in FP32
// (with FMA), conserved variables read, accumulated and stored in FP64.
#define FV_T float
#define FV_LAUNCH_NAME launchStepF32
#define FV_SMEM_NAME marchSmemF32
#include "fv_inst.inc"
