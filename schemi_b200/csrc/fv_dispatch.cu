// fv_dispatch.cu -- selects the instantiation unit of a species count and an equation of state
// (fv_<prec>_ns<N>_<eos>.cu).
#include "fv_launch.cuh"

namespace fv {

// Entry points of one unit: species count N, equation of state E (0 ideal, 1 van der Waals, 9 the
// real-gas mixtures on the generic path).
#define FV_DECLARE_UNIT(P, N, E)                                                                                \
    cudaError_t launchStep##P##_ns##N##_e##E(const StepParams&, const StepBuffers&, int, const MarchShape&,      \
                                             cudaStream_t);                                                      \
    cudaError_t launchBatch##P##_ns##N##_e##E(int, const BatchCase*, int, long long, const MarchShape&, int*,    \
                                              cudaStream_t);
#define FV_DECLARE_REAL(P, N)                                                                                   \
    cudaError_t launchStep##P##_ns##N##_e9(const StepParams&, const StepBuffers&, int, const MarchShape&,        \
                                           cudaStream_t);
#define FV_DECLARE(P)                                                                                           \
    FV_DECLARE_UNIT(P, 1, 0) FV_DECLARE_UNIT(P, 1, 1) FV_DECLARE_UNIT(P, 2, 0) FV_DECLARE_UNIT(P, 2, 1)           \
    FV_DECLARE_UNIT(P, 3, 0) FV_DECLARE_UNIT(P, 3, 1) FV_DECLARE_UNIT(P, 4, 0) FV_DECLARE_UNIT(P, 4, 1)           \
    FV_DECLARE_REAL(P, 1) FV_DECLARE_REAL(P, 2) FV_DECLARE_REAL(P, 3) FV_DECLARE_REAL(P, 4)                       \
    size_t marchSmem##P##_ns1_e0(int, const MarchShape&);                                                       \
    size_t marchSmem##P##_ns2_e0(int, const MarchShape&);                                                       \
    size_t marchSmem##P##_ns3_e0(int, const MarchShape&);                                                       \
    size_t marchSmem##P##_ns4_e0(int, const MarchShape&);

FV_DECLARE(F64)
FV_DECLARE(F32)

#define FV_STEP_CASE(P, N)                                                                                      \
    case N:                                                                                                     \
        if (real) return launchStep##P##_ns##N##_e9(p, b, path, s, st);                                         \
        return vdw ? launchStep##P##_ns##N##_e1(p, b, path, s, st) : launchStep##P##_ns##N##_e0(p, b, path, s, st);
#define FV_BATCH_CASE(P, N)                                                                                     \
    case N:                                                                                                     \
        return vdw ? launchBatch##P##_ns##N##_e1(dims, c, n, tt, s, g, st)                                      \
                   : launchBatch##P##_ns##N##_e0(dims, c, n, tt, s, g, st);

#define FV_DEFINE(P)                                                                                           \
    cudaError_t launchStep##P(const StepParams& p, const StepBuffers& b, int path, const MarchShape& s,          \
                              cudaStream_t st) {                                                               \
        const bool vdw = p.mix.eos_kind == FV_EOS_VAN_DER_WAALS;                                               \
        const bool real = p.mix.eos_kind != FV_EOS_IDEAL && !vdw;                                              \
        switch (p.mix.ns) {                                                                                    \
            FV_STEP_CASE(P, 1)                                                                                 \
            FV_STEP_CASE(P, 2)                                                                                 \
            FV_STEP_CASE(P, 3)                                                                                 \
            FV_STEP_CASE(P, 4)                                                                                 \
        }                                                                                                      \
        return cudaErrorInvalidConfiguration;                                                                  \
    }                                                                                                          \
    cudaError_t launchBatch##P(int ns, int eos, int dims, const BatchCase* c, int n, long long tt,              \
                               const MarchShape& s, int* g, cudaStream_t st) {                                 \
        const bool vdw = eos == FV_EOS_VAN_DER_WAALS;                                                          \
        if (eos != FV_EOS_IDEAL && !vdw) return cudaErrorInvalidConfiguration; /* ensembles: ideal / vdW */    \
        switch (ns) {                                                                                          \
            FV_BATCH_CASE(P, 1)                                                                                \
            FV_BATCH_CASE(P, 2)                                                                                \
            FV_BATCH_CASE(P, 3)                                                                                \
            FV_BATCH_CASE(P, 4)                                                                                \
        }                                                                                                      \
        return cudaErrorInvalidConfiguration;                                                                  \
    }                                                                                                          \
    size_t marchSmem##P(int ns, int dims, const MarchShape& s) {                                               \
        switch (ns) {                                                                                          \
        case 1: return marchSmem##P##_ns1_e0(dims, s);                                                          \
        case 2: return marchSmem##P##_ns2_e0(dims, s);                                                          \
        case 3: return marchSmem##P##_ns3_e0(dims, s);                                                          \
        case 4: return marchSmem##P##_ns4_e0(dims, s);                                                          \
        }                                                                                                      \
        return 0;                                                                                              \
    }

FV_DEFINE(F64)
FV_DEFINE(F32)

}  // namespace fv
