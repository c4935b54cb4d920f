// fv_dispatch.cu -- selects the per-species-count instantiation units (fv_<prec>_ns<N>.cu).
#include "fv_launch.cuh"

namespace fv {

#define FV_DECLARE(P)                                                                                         \
    cudaError_t launchStep##P##_ns1(const StepParams&, const StepBuffers&, int, const MarchShape&, cudaStream_t); \
    cudaError_t launchStep##P##_ns2(const StepParams&, const StepBuffers&, int, const MarchShape&, cudaStream_t); \
    cudaError_t launchStep##P##_ns3(const StepParams&, const StepBuffers&, int, const MarchShape&, cudaStream_t); \
    cudaError_t launchStep##P##_ns4(const StepParams&, const StepBuffers&, int, const MarchShape&, cudaStream_t); \
    cudaError_t launchBatch##P##_ns1(int, int, const BatchCase*, int, long long, const MarchShape&, int*, cudaStream_t); \
    cudaError_t launchBatch##P##_ns2(int, int, const BatchCase*, int, long long, const MarchShape&, int*, cudaStream_t); \
    cudaError_t launchBatch##P##_ns3(int, int, const BatchCase*, int, long long, const MarchShape&, int*, cudaStream_t); \
    cudaError_t launchBatch##P##_ns4(int, int, const BatchCase*, int, long long, const MarchShape&, int*, cudaStream_t); \
    size_t marchSmem##P##_ns1(int, const MarchShape&);                                                       \
    size_t marchSmem##P##_ns2(int, const MarchShape&);                                                       \
    size_t marchSmem##P##_ns3(int, const MarchShape&);                                                       \
    size_t marchSmem##P##_ns4(int, const MarchShape&);

FV_DECLARE(F64)
FV_DECLARE(F32)

#define FV_DEFINE(P)                                                                                           \
    cudaError_t launchStep##P(const StepParams& p, const StepBuffers& b, int path, const MarchShape& s,          \
                              cudaStream_t st) {                                                               \
        switch (p.mix.ns) {                                                                                    \
        case 1: return launchStep##P##_ns1(p, b, path, s, st);                                                  \
        case 2: return launchStep##P##_ns2(p, b, path, s, st);                                                  \
        case 3: return launchStep##P##_ns3(p, b, path, s, st);                                                  \
        case 4: return launchStep##P##_ns4(p, b, path, s, st);                                                  \
        }                                                                                                      \
        return cudaErrorInvalidConfiguration;                                                                  \
    }                                                                                                          \
    cudaError_t launchBatch##P(int ns, int eos, int dims, const BatchCase* c, int n, long long tt,              \
                               const MarchShape& s, int* g, cudaStream_t st) {                                 \
        switch (ns) {                                                                                          \
        case 1: return launchBatch##P##_ns1(eos, dims, c, n, tt, s, g, st);                                     \
        case 2: return launchBatch##P##_ns2(eos, dims, c, n, tt, s, g, st);                                     \
        case 3: return launchBatch##P##_ns3(eos, dims, c, n, tt, s, g, st);                                     \
        case 4: return launchBatch##P##_ns4(eos, dims, c, n, tt, s, g, st);                                     \
        }                                                                                                      \
        return cudaErrorInvalidConfiguration;                                                                  \
    }                                                                                                          \
    size_t marchSmem##P(int ns, int dims, const MarchShape& s) {                                               \
        switch (ns) {                                                                                          \
        case 1: return marchSmem##P##_ns1(dims, s);                                                             \
        case 2: return marchSmem##P##_ns2(dims, s);                                                             \
        case 3: return marchSmem##P##_ns3(dims, s);                                                             \
        case 4: return marchSmem##P##_ns4(dims, s);                                                             \
        }                                                                                                      \
        return 0;                                                                                              \
    }

FV_DEFINE(F64)
FV_DEFINE(F32)

}  // namespace fv
