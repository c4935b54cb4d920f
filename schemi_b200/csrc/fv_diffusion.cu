// fv_diffusion.cu -- instantiations and launcher of the diffusion stage (fv_diffusion.cuh), FP64
// with --fmad=false like the reference's arithmetic.
#include "fv_diffusion.cuh"
#include "fv_diffusion_gs.cuh"
#include "fv_diffusion_launch.h"

namespace fv {

namespace {
constexpr int kDiffThreads = 256;

// Launch shape of the Gauss-Seidel solve (k_gs_solve): up to 512 columns (2D / 3D) the split
// mode, two threads per column rounded to warps; else one per column (whole warps) or the CTA's
// maximum.  Its dynamic shared memory: the split mode's slots, then both iterates when they fit
// (itersInSmem), else the iterates live in the work buffer.  The Jacobi solve's: the iterates
// alone when they fit.
struct GsShape {
    int threads, smem, itersInSmem;
};
GsShape gsShape(const StepParams& P, int D) {
    const long long ncol = D == 1 ? 1 : (D == 2 ? (long long)P.n[0] : (long long)P.n[0] * P.n[1]);
    const long long W = (ncol + 31) / 32 * 32;
    const bool split = D >= 2 && ncol <= 512;
    GsShape g;
    g.threads = split ? (int)(2 * W) : (ncol >= diff::kGsThreads ? diff::kGsThreads : (int)W);
    const long long role = split ? diff::kGsRoleDoubles * W * (long long)sizeof(double) : 0;
    const long long iters = 2 * P.ncell * (long long)sizeof(double);
    g.itersInSmem = role + iters <= diff::kGsSmemBytes;
    g.smem = (int)(role + (g.itersInSmem ? iters : 0));
    return g;
}
int jacobiSmemBytes(const StepParams& P) {
    const long long b = 2 * P.ncell * (long long)sizeof(double);
    return b <= diff::kGsSmemBytes ? (int)b : 0;
}

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
        const GsShape gs = gsShape(P, D);
        const int sm = jacobiSmemBytes(P);
        // one solve of diag x + off x = free (x: the start in, the solution out) by the deck's solver
        auto solve = [&](const double* dg, const double* fr, const double* of, double* xs) {
            if (X.sle == FV_SLE_JACOBI)
                diff::k_jacobi_solve<D><<<1, diff::kGsThreads, sm, st>>>(P, dg, fr, of, xs, X.work, X.maxIter, sm > 0, ck);
            else if (X.sle == FV_SLE_THOMAS)
                diff::k_thomas_solve<<<1, 32, 0, st>>>(P, dg, fr, of, xs, X.work, ck);
            else if (X.sle == FV_SLE_NO_SOLVER)
                return;  // noMatrixSolver::solve: the start field is the solution
            else if (X.sle == FV_SLE_CG)
                diff::k_cg_solve<D, 0><<<1, diff::kGsThreads, 0, st>>>(P, dg, fr, of, xs, X.work, X.maxIter, ck);
            else if (X.sle == FV_SLE_JACOBI_CG)
                diff::k_cg_solve<D, 1><<<1, diff::kGsThreads, 0, st>>>(P, dg, fr, of, xs, X.work, X.maxIter, ck);
            else if (X.sle == FV_SLE_BICG)
                diff::k_cg_solve<D, 2><<<1, diff::kGsThreads, 0, st>>>(P, dg, fr, of, xs, X.work, X.maxIter, ck);
            else
                diff::k_gs_solve<D><<<1, gs.threads, gs.smem, st>>>(P, dg, fr, of, xs, X.work, X.maxIter, gs.itersInSmem,
                                                                    ck);
        };
        diff::k_gs_wmat<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, L, X, U, ck);
        for (int k = 0; k < NS; ++k) solve(X.wDiag + k * s, X.wFree + k * s, X.wOff + k * 6 * s, X.sol + k * s);
        diff::k_gs_post1<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, X, U, ck);
        if (X.enthalpy) diff::k_gs_afdif<NS, EOS, D><<<gf, kDiffThreads, 0, st>>>(P, L, X, ck);
        diff::k_gs_vtmat<NS, EOS, D><<<gc, kDiffThreads, 0, st>>>(P, L, X, U, ck);
        for (int d = 0; d < P.nmom; ++d) solve(X.vDiag, X.vFree + d * s, X.vOff, X.sol + (NS + d) * s);
        solve(X.tDiag, X.tFree, X.tOff, X.sol + (NS + 3) * s);
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

cudaError_t configureDiffusion(int dims, const StepParams& P) {
    const int sg = gsShape(P, dims).smem, sj = jacobiSmemBytes(P);
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaSuccess;
    if (dims == 1) {
        if (sg > 48 * 1024) e = cudaFuncSetAttribute(diff::k_gs_solve<1>, a, sg);
        if (e == cudaSuccess && sj > 48 * 1024) e = cudaFuncSetAttribute(diff::k_jacobi_solve<1>, a, sj);
    } else if (dims == 2) {
        if (sg > 48 * 1024) e = cudaFuncSetAttribute(diff::k_gs_solve<2>, a, sg);
        if (e == cudaSuccess && sj > 48 * 1024) e = cudaFuncSetAttribute(diff::k_jacobi_solve<2>, a, sj);
    } else {
        if (sg > 48 * 1024) e = cudaFuncSetAttribute(diff::k_gs_solve<3>, a, sg);
        if (e == cudaSuccess && sj > 48 * 1024) e = cudaFuncSetAttribute(diff::k_jacobi_solve<3>, a, sj);
    }
    return e;
}

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
