// FP32-flux step kernels for 4 species, ideal-gas mixtures: reconstruction, closures and fluxes in FP32 (fast
// math), conserved variables read, accumulated and stored in FP64.
#define FV_T float
#define FV_NS 4
#define FV_EOS 0
#define FV_LAUNCH_NAME launchStepF32
#define FV_BATCH_NAME launchBatchF32
#define FV_SMEM_NAME marchSmemF32
#include "fv_inst.inc"
