// fv_diffusion.cu -- instantiations and launcher of the diffusion stage (fv_diffusion.cuh), FP64
// with --fmad=false like the reference's arithmetic.
#include "fv_diffusion.cuh"
#include "fv_diffusion_gs.cuh"
#include "fv_diffusion_launch.h"

namespace fv {

namespace {
constexpr int kDiffThreads = 256;

template <int NS, int EOS, int D>
cudaError_t launchT(const StepParams& P, const GenericLayout& L, const diff::DiffParams& X, double* U, DevClock* ck,
                    double* blockMax, cudaStream_t st) {
    const unsigned gc = (unsigned)((P.ncell + kDiffThreads - 1) / kDiffThreads);
    const unsigned gf = (unsigned)((L.nfaces + kDiffThreads - 1) / kDiffThreads);
    diff::k_diff_prim<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, X, U, ck);
    diff::k_diff_faces<NS, EOS, D><<<gf, kDiffThreads, 0, st>>>(P, L, X, ck);
    if (!X.gs) {
        diff::k_diff_cells<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, L, X, U, ck, blockMax);
    } else {
        // the implicit solver: mass-fraction matrices and solves, new concentrations, the
        // averaged enthalpy flow, velocity and temperature matrices and solves, the phase
        const long long s = P.stride;
        diff::k_gs_wmat<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, L, X, U, ck);
        for (int k = 0; k < NS; ++k)
            diff::k_gs_solve<D><<<1, diff::kGsThreads, 0, st>>>(P, X.wDiag + k * s, X.wFree + k * s, X.wOff + k * 6 * s,
                                                               X.sol + k * s, X.work, X.maxIter, ck);
        diff::k_gs_post1<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, X, U, ck);
        if (X.enthalpy) diff::k_gs_afdif<NS, EOS, D><<<gf, kDiffThreads, 0, st>>>(P, L, X, ck);
        diff::k_gs_vtmat<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, L, X, U, ck);
        for (int d = 0; d < P.nmom; ++d)
            diff::k_gs_solve<D><<<1, diff::kGsThreads, 0, st>>>(P, X.vDiag, X.vFree + d * s, X.vOff,
                                                               X.sol + (NS + d) * s, X.work, X.maxIter, ck);
        diff::k_gs_solve<D><<<1, diff::kGsThreads, 0, st>>>(P, X.tDiag, X.tFree, X.tOff, X.sol + (NS + 3) * s,
                                                           X.work, X.maxIter, ck);
        diff::k_gs_final<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, L, X, U, ck, blockMax);
    }
    diff::k_diff_source<<<1, 1024, 0, st>>>(X, ck, (int)gc);
    return cudaGetLastError();
}

template <int NS, int EOS>
cudaError_t byDims(int dims, const StepParams& P, const GenericLayout& L, const diff::DiffParams& X, double* U,
                   DevClock* ck, double* blockMax, cudaStream_t st) {
    if (dims == 1) return launchT<NS, EOS, 1>(P, L, X, U, ck, blockMax, st);
    if (dims == 2) return launchT<NS, EOS, 2>(P, L, X, U, ck, blockMax, st);
    return launchT<NS, EOS, 3>(P, L, X, U, ck, blockMax, st);
}

template <int NS>
cudaError_t byEos(int eos, int dims, const StepParams& P, const GenericLayout& L, const diff::DiffParams& X, double* U,
                  DevClock* ck, double* blockMax, cudaStream_t st) {
    if (eos == FV_EOS_IDEAL) return byDims<NS, FV_EOS_IDEAL>(dims, P, L, X, U, ck, blockMax, st);
    return byDims<NS, FV_EOS_VAN_DER_WAALS>(dims, P, L, X, U, ck, blockMax, st);
}
}  // namespace

int diffusionBlocks(const StepParams& P) { return (int)((P.ncell + kDiffThreads - 1) / kDiffThreads); }

cudaError_t launchDiffusion(int ns, int eos, int dims, const StepParams& P, const GenericLayout& L,
                            const diff::DiffParams& X, double* U, DevClock* ck, double* blockMax, cudaStream_t st) {
    switch (ns) {
    case 1: return byEos<1>(eos, dims, P, L, X, U, ck, blockMax, st);
    case 2: return byEos<2>(eos, dims, P, L, X, U, ck, blockMax, st);
    case 3: return byEos<3>(eos, dims, P, L, X, U, ck, blockMax, st);
    default: return byEos<4>(eos, dims, P, L, X, U, ck, blockMax, st);
    }
}

}  // namespace fv
