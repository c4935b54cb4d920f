// fv_chem.cu -- instantiation and launcher of the chemistry pass (FP64, no FMA contraction so
// that every expression rounds as the CPU does).
#include "fv_chem.cuh"
#include "fv_chem_launch.h"

namespace fv {
namespace {

template <int N, int EOS, int D>
cudaError_t launchT(const StepParams& P, const chem::ChemParams& C, double* U, DevClock* ck, double* blockMax,
                    int blocks, cudaStream_t st) {
    if (C.conc) chem::k_chemistry<N, EOS, D, true><<<blocks, 256, 0, st>>>(P, C, U, ck, blockMax);
    else chem::k_chemistry<N, EOS, D, false><<<blocks, 256, 0, st>>>(P, C, U, ck, blockMax);
    return cudaGetLastError();
}

template <int N, int EOS>
cudaError_t launchD(int dims, const StepParams& P, const chem::ChemParams& C, double* U, DevClock* ck,
                    double* blockMax, int blocks, cudaStream_t st) {
    switch (dims) {
    case 1: return launchT<N, EOS, 1>(P, C, U, ck, blockMax, blocks, st);
    case 2: return launchT<N, EOS, 2>(P, C, U, ck, blockMax, blocks, st);
    case 3: return launchT<N, EOS, 3>(P, C, U, ck, blockMax, blocks, st);
    }
    return cudaErrorInvalidValue;
}

template <int N>
cudaError_t launchE(int eos, int dims, const StepParams& P, const chem::ChemParams& C, double* U, DevClock* ck,
                    double* blockMax, int blocks, cudaStream_t st) {
    return eos == FV_EOS_IDEAL ? launchD<N, FV_EOS_IDEAL>(dims, P, C, U, ck, blockMax, blocks, st)
                               : launchD<N, FV_EOS_VAN_DER_WAALS>(dims, P, C, U, ck, blockMax, blocks, st);
}

}  // namespace

int chemistryBlocks(const StepParams& P) {
    const long long b = (P.ncell + 255) / 256;
    return (int)(b < 148 * 8 ? b : 148 * 8);
}

cudaError_t launchChemistry(int ns, int eos, int dims, const StepParams& P, const chem::ChemParams& C, double* U,
                            DevClock* ck, double* blockMax, cudaStream_t st) {
    const int blocks = chemistryBlocks(P);
    if (C.mech == FV_CHEM_CL2 && ns == 2) return launchE<2>(eos, dims, P, C, U, ck, blockMax, blocks, st);
    if (C.mech == FV_CHEM_A_B_2C && ns == 3) return launchE<3>(eos, dims, P, C, U, ck, blockMax, blocks, st);
    return cudaErrorInvalidValue;
}

}  // namespace fv
