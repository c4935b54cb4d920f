// FP64 instantiation of the step kernels.  Built with --fmad=false so that every expression
// rounds like the reference's x86-64 build (no fused multiply-add), which makes the FP64 path
// reproduce the reference bit for bit.
#define FV_T double
#define FV_LAUNCH_NAME launchStepF64
#define FV_SMEM_NAME marchSmemF64
#include "fv_inst.inc"
