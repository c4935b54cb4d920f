// FP64 step kernels for 1 species, ideal-gas mixtures.  Built with --fmad=false so that every expression rounds
// like the reference's x86-64 build (no fused multiply-add): the FP64 path is bit-exact.
#define FV_T double
#define FV_NS 1
#define FV_EOS 0
#define FV_LAUNCH_NAME launchStepF64
#define FV_BATCH_NAME launchBatchF64
#define FV_SMEM_NAME marchSmemF64
#include "fv_inst.inc"
