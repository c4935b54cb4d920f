// fv_capi.cu -- the C-ABI of include/fvstep.h: handle management, geometry tables, upload /
// download, the device-resident time loop (CUDA graphs of step chunks) and error reporting.
//
// Built with --fmad=false: the upload kernel restates phaseInitialization.cpp:1827-1885 and the
// finalize kernel the CFL block of Schemi.cpp:807-835 with the reference's rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "../../include/fvstep.h"
#include "fv_diffusion_launch.h"
#include "fv_launch.cuh"
#include "fv_validate.h"

using namespace fv;

// ============================================================================ device kernels
namespace {

// phaseInitialization.cpp:1827-1885 for one cell
template <int NS, int EOS>
__global__ void k_upload(const StepParams P, const double* __restrict__ prim, double* __restrict__ U) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long s = P.stride;
    double c[NS + 1], rho[NS + 1];
    c[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = prim[(k - 1) * s + i];
        c[0] += c[k];
    }
#pragma unroll
    for (int k = 1; k <= NS; ++k) rho[k] = c[k] * P.mix.M[k - 1];
    rho[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) rho[0] += rho[k];
    const double v[3] = {prim[NS * s + i], prim[(NS + 1) * s + i], prim[(NS + 2) * s + i]};
    const double p = prim[(NS + 3) * s + i];
    const double Uv = Mixture<double, NS, EOS>::UvFromp(P.mix, c, p);
    double v2 = 0;
    v2 += v[0] * v[0];
    v2 += v[1] * v[1];
    v2 += v[2] * v[2];
    const double E = Uv + rho[0] * v2 * 0.5 + 0.0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) U[(k - 1) * s + i] = rho[k];
    U[NS * s + i] = rho[0];
    for (int d = 0; d < 3; ++d) U[(NS + 1 + d) * s + i] = v[d] * rho[0];
    U[(NS + 4) * s + i] = E;
}

// output set (fv_field order) of one cell; primitives from the restart set before step 1
template <int NS, int EOS>
__global__ void k_download(const StepParams P, const double* __restrict__ U, const double* __restrict__ prim0,
                           const DevClock* __restrict__ ck, double* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long n = P.ncell, s = P.stride;
    double c[NS + 1], v[3], p, rho0, rho[NS + 1], m[3], E;
    // the restart set before the first step; after a diffusion stage the primitives, energy and
    // temperature it set (Diffusion.cpp:965-1025: the phase's T is the stage's, not TFromUv)
    const bool stage = !ck->first && ck->stagePrim;
    const double* prim = ck->first ? prim0 : (stage ? P.stagePrim : nullptr);
    switch (P.dims) {
    case 1: cellPrimitive<double, NS, EOS, 1>(P, U, prim, i, c, v, p, rho0, rho, m, E); break;
    case 2: cellPrimitive<double, NS, EOS, 2>(P, U, prim, i, c, v, p, rho0, rho, m, E); break;
    default: cellPrimitive<double, NS, EOS, 3>(P, U, prim, i, c, v, p, rho0, rho, m, E); break;
    }
    double Uv;
    if (stage) {
        Uv = P.stagePrim[(NS + 4) * s + i];
    } else if (prim) {
        Uv = Mixture<double, NS, EOS>::UvFromp(P.mix, c, p);
    } else {
        double v2 = 0;
        v2 += v[0] * v[0];
        v2 += v[1] * v[1];
        v2 += v[2] * v[2];
        Uv = E - rho0 * v2 * 0.5 - 0.0;
    }
    for (int k = 0; k < NS; ++k) out[(FV_F_CONC + k) * n + i] = c[k + 1];
    out[FV_F_VX * n + i] = v[0];
    out[FV_F_VY * n + i] = v[1];
    out[FV_F_VZ * n + i] = v[2];
    out[FV_F_P * n + i] = p;
    for (int k = 0; k < NS; ++k) out[(FV_F_RHO_K + k) * n + i] = rho[k + 1];
    out[FV_F_RHO * n + i] = rho0;
    out[FV_F_MX * n + i] = m[0];
    out[FV_F_MY * n + i] = m[1];
    out[FV_F_MZ * n + i] = m[2];
    out[FV_F_E * n + i] = E;
    out[FV_F_UV * n + i] = Uv;
    out[FV_F_T * n + i] = stage ? P.stagePrim[(NS + 5) * s + i] : Mixture<double, NS, EOS>::TFromUv(P.mix, c, Uv);
    out[FV_F_SONIC * n + i] = sqrt(Mixture<double, NS, EOS>::sqSonic(P.mix, c, rho0, Uv, p));
    out[FV_F_CONC0 * n + i] = c[0];
}

// flag |= (any transverse velocity component of the restart set is non-zero)
__global__ void k_transverse(const StepParams P, const double* __restrict__ prim, int* flag) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    bool nz = false;
    for (int d = P.dims; d < 3; ++d) nz |= prim[(P.mix.ns + d) * P.stride + i] != 0.0;
    if (nz) atomicOr(flag, 1);
}

// SecondOrderRK: Un2.average(Un, 0.5) + copyFrom (secondOrderStepSolverRK.cpp:64-66,
// bunchOfFields.hpp:166-237) of the state after the second stage U2 with the step's start state
// U0, then main's CFL signal of the averaged state.  Concentrations are averaged as fields: c of
// U2 is rho_k / M_k with c_0 their sum (Advection2dOrder.cpp:578-585), c of U0 the stored ones
// (or the restart set before step 1).  Writes the averaged state to Un and conc.
// ThirdOrder uses the same kernel with the weights 0.25 and 2/3 (thirdOrderStepSolver.cpp:64-82),
// reading the start state's concentrations from concIn and writing the averaged ones to concOut.
template <int NS, int EOS, int D>
__global__ void k_rk_average(const StepParams P, const double* __restrict__ U2, const double* __restrict__ U0,
                             const double* __restrict__ prim0, DevClock* __restrict__ ck, double* __restrict__ Un,
                             const double* concIn, double* concOut, double ownWeight, double* __restrict__ blockMax) {
    __shared__ double red[32];
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double localMax = -1;
    if (i < P.ncell) {
        const long long s = P.stride;
        const double own = ownWeight, in = 1 - ownWeight;
        double c2[NS + 1], c0[NS + 1], c[NS + 1];
        c2[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            c2[k] = U2[(k - 1) * s + i] / P.mix.M[k - 1];
            c2[0] += c2[k];
        }
        if (ck->first) {
            c0[0] = 0;
#pragma unroll
            for (int k = 1; k <= NS; ++k) {
                c0[k] = prim0[(k - 1) * s + i];
                c0[0] += c0[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k <= NS; ++k) c0[k] = concIn[k * s + i];
        }
#pragma unroll
        for (int k = 0; k <= NS; ++k) {
            c[k] = own * c2[k] + in * c0[k];
            concOut[k * s + i] = c[k];
        }
        double rho[NS + 1];
#pragma unroll
        for (int k = 0; k <= NS; ++k) {
            const int f = k == 0 ? NS : k - 1;
            rho[k] = own * U2[f * s + i] + in * U0[f * s + i];
            Un[f * s + i] = rho[k];
        }
        double m[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d < P.nmom) {
                m[d] = U2[(NS + 1 + d) * s + i] * own + U0[(NS + 1 + d) * s + i] * in;
                Un[(NS + 1 + d) * s + i] = m[d];
            }
        const double E = own * U2[(NS + 4) * s + i] + in * U0[(NS + 4) * s + i];
        Un[(NS + 4) * s + i] = E;
        // copyFrom: v = m / rho, Uv = E - k - 0.5 rho (v & v), p = pFromUv(c, Uv); CFL signal
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = d < P.nmom ? m[d] / rho[0] : 0.0;
        double vv = 0;
        vv += v[0] * v[0];
        vv += v[1] * v[1];
        vv += v[2] * v[2];
        const double Uv = (E - 0.0) - 0.5 * rho[0] * vv;
        const double p = Mixture<double, NS, EOS>::pFromUv(P.mix, c, Uv);
        const double sonic = sqrt(Mixture<double, NS, EOS>::sqSonic(P.mix, c, rho[0], Uv, p));
        int ijk[3];
        ijk[0] = (int)(i % P.n[0]);
        ijk[1] = D >= 2 ? (int)((i / P.n[0]) % P.n[1]) : 0;
        ijk[2] = D >= 3 ? (int)(i / ((long long)P.n[0] * P.n[1])) : 0;
        const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
        const double minLS = 1.0 / smin(smin(ex, ey), ez);
        double sg = (P.nmom == 3 ? mag3<double>(v[0], v[1], v[2]) : mag2z<double>(v[0], v[1])) + sonic;
        sg *= minLS;
        localMax = sg;
    }
    const double bm = blockMaxReduce<double>(localMax, red);
    if (threadIdx.x == 0) blockMax[blockIdx.x] = bm;
}

}  // namespace

namespace fv {
// CFL block of Schemi.cpp:802-835 and the last-step clamp of :933-935.
__global__ void k_finalize(const StepParams P, DevClock* ck, const double* __restrict__ blockMax, int nblocks) {
    finalizeCase(P, ck, blockMax, nblocks);
}
__global__ void k_finalize_batch(const BatchCase* __restrict__ cases, int nCases) {
    const BatchCase& C = cases[blockIdx.x];
    finalizeCase(C.P, C.ck, C.blockMax, C.nPartials);
}
}  // namespace fv

// ============================================================================ host side
#include "fv_handle.h"

namespace {

const char* kNoHandle = "invalid handle";

fv_status fail(fv_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

fv_status cudaFail(fv_handle* h, cudaError_t e, const char* what) {
    return fail(h, FV_ERR_SYSTEM, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FV_CUDA(h, call)                                      \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cudaFail((h), e_, #call); \
    } while (0)

// scaled hypot of one non-zero component (|x| exactly)
double edge(double a, double b) { return std::fabs(b - a); }

// Per-axis geometry tables with the mesh generator's arithmetic (mesh.cpp:296-1900):
// node coordinates 0 + d*i, cell centres as the 8-corner average, face centres as the
// 4-corner average in the corner order of each face type.
void buildGeometry(const fv_config& c, std::vector<double>& host, size_t off[3][5], int nAxis[3]) {
    host.clear();
    for (int a = 0; a < 3; ++a) {
        const bool used = a < c.dims;
        const int n = used ? c.n[a] : 1;
        nAxis[a] = n;
        const double L = c.L[a];
        const double d = L / n;
        auto node = [&](int i) -> double {
            if (used) return 0.0 + d * (double)(size_t)i;
            return i == 0 ? 0.0 : L;
        };
        // h
        off[a][0] = host.size();
        for (int i = 0; i < n; ++i) host.push_back(edge(node(i), node(i + 1)));
        // cell centre: pattern x: a b a b a b a b ; y: a a b b a a b b ; z: a a a a b b b b
        off[a][1] = host.size();
        for (int i = 0; i < n; ++i) {
            const double A = node(i), B = node(i + 1);
            double seq[8];
            for (int q = 0; q < 8; ++q) {
                const int bit = a == 0 ? (q & 1) : (a == 1 ? ((q >> 1) & 1) : ((q >> 2) & 1));
                seq[q] = bit ? B : A;
            }
            double s = seq[0] + seq[1];
            for (int q = 2; q < 8; ++q) s = s + seq[q];
            host.push_back(s / 8.);
        }
        // own-axis face centre: X at all four corners; X = 0 + 0., 0 + d*i, 0 + L
        off[a][2] = host.size();
        for (int i = 0; i <= n; ++i) {
            double X;
            if (i == 0) X = 0.0 + 0.;
            else if (i == n) X = 0.0 + L;
            else X = node(i);
            double s = X + X;
            s = s + X;
            s = s + X;
            host.push_back(s / 4.);
        }
        // transverse face-centre coordinates
        off[a][3] = host.size();
        for (int i = 0; i < n; ++i) {
            const double A = node(i), B = node(i + 1);
            double s = A + A;
            s = s + B;
            s = s + B;
            host.push_back(s / 4.);
        }
        off[a][4] = host.size();
        for (int i = 0; i < n; ++i) {
            const double A = node(i), B = node(i + 1);
            double s = A + B;
            s = s + A;
            s = s + B;
            host.push_back(s / 4.);
        }
    }
}

template <int NS, int EOS>
void launchUpload(fv_handle* h, const double* primDev) {
    const int tpb = 256;
    const unsigned g = (unsigned)((h->P.ncell + tpb - 1) / tpb);
    k_upload<NS, EOS><<<g, tpb, 0, h->stream>>>(h->P, primDev, h->U[h->cur]);
}
template <int NS, int EOS>
void launchDownload(fv_handle* h) {
    const int tpb = 256;
    const unsigned g = (unsigned)((h->P.ncell + tpb - 1) / tpb);
    k_download<NS, EOS><<<g, tpb, 0, h->stream>>>(h->P, h->U[h->cur], h->prim0, h->ck, h->outBuf);
}
template <template <int, int> class F> struct Dispatch;

void upload(fv_handle* h, const double* primDev) {
    const int ns = h->cfg.n_species;
    const int e = fvEosTemplate(h->cfg.eos);
    switch (ns) {
    case 1: e == 0 ? launchUpload<1, 0>(h, primDev) : e == 1 ? launchUpload<1, 1>(h, primDev) : launchUpload<1, kEosGeneral>(h, primDev); break;
    case 2: e == 0 ? launchUpload<2, 0>(h, primDev) : e == 1 ? launchUpload<2, 1>(h, primDev) : launchUpload<2, kEosGeneral>(h, primDev); break;
    case 3: e == 0 ? launchUpload<3, 0>(h, primDev) : e == 1 ? launchUpload<3, 1>(h, primDev) : launchUpload<3, kEosGeneral>(h, primDev); break;
    default: e == 0 ? launchUpload<4, 0>(h, primDev) : e == 1 ? launchUpload<4, 1>(h, primDev) : launchUpload<4, kEosGeneral>(h, primDev); break;
    }
}
void download(fv_handle* h) {
    const int ns = h->cfg.n_species;
    const int e = fvEosTemplate(h->cfg.eos);
    switch (ns) {
    case 1: e == 0 ? launchDownload<1, 0>(h) : e == 1 ? launchDownload<1, 1>(h) : launchDownload<1, kEosGeneral>(h); break;
    case 2: e == 0 ? launchDownload<2, 0>(h) : e == 1 ? launchDownload<2, 1>(h) : launchDownload<2, kEosGeneral>(h); break;
    case 3: e == 0 ? launchDownload<3, 0>(h) : e == 1 ? launchDownload<3, 1>(h) : launchDownload<3, kEosGeneral>(h); break;
    default: e == 0 ? launchDownload<4, 0>(h) : e == 1 ? launchDownload<4, 1>(h) : launchDownload<4, kEosGeneral>(h); break;
    }
}

void destroyGraphs(fv_handle* h) {
    for (auto& g : h->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    h->graphSteps = 0;
}

StepBuffers buffersFor(fv_handle* h, int from) {
    StepBuffers B;
    B.U = h->U[from];
    B.Un = h->U[from ^ 1];
    B.prim0 = h->prim0;
    B.ck = h->ck;
    B.blockMax = h->blockMax;
    B.blockMaxCap = h->blockMaxCap;
    B.Pc = h->Pc;
    B.FS = h->FS;
    B.FL = h->FL;
    B.L = h->L;
    B.pcIn = h->pc[from];
    B.pcOut = h->pc[from ^ 1];
    return B;
}

long long stepBlocks(fv_handle* h) {
    return h->path == PATH_MARCH ? marchBlocks(h->P, h->shape) : genericBlocks(h->P);
}

// enqueue step [+ chemistry] + finalize reading U[from]
// (Ustage, U[from]) averaged into U[from ^ 1]
template <int NS, int EOS>
void launchAverage(fv_handle* h, int from, const double* concIn, double* concOut, double ownWeight) {
    const int tpb = 128;
    const unsigned g = (unsigned)genericBlocks(h->P);
    switch (h->cfg.dims) {
    case 1: k_rk_average<NS, EOS, 1><<<g, tpb, 0, h->stream>>>(h->P, h->Ustage, h->U[from], h->prim0, h->ck, h->U[from ^ 1], concIn, concOut, ownWeight, h->blockMax); break;
    case 2: k_rk_average<NS, EOS, 2><<<g, tpb, 0, h->stream>>>(h->P, h->Ustage, h->U[from], h->prim0, h->ck, h->U[from ^ 1], concIn, concOut, ownWeight, h->blockMax); break;
    default: k_rk_average<NS, EOS, 3><<<g, tpb, 0, h->stream>>>(h->P, h->Ustage, h->U[from], h->prim0, h->ck, h->U[from ^ 1], concIn, concOut, ownWeight, h->blockMax); break;
    }
}

void average(fv_handle* h, int from, const double* concIn, double* concOut, double ownWeight) {
    const int ns = h->cfg.n_species;
    const int e = fvEosTemplate(h->cfg.eos);
#define FV_AVG(N)                                                                                           \
    (e == 0 ? launchAverage<N, 0>(h, from, concIn, concOut, ownWeight)                                      \
            : e == 1 ? launchAverage<N, 1>(h, from, concIn, concOut, ownWeight)                             \
                     : launchAverage<N, kEosGeneral>(h, from, concIn, concOut, ownWeight))
    switch (ns) {
    case 1: FV_AVG(1); break;
    case 2: FV_AVG(2); break;
    case 3: FV_AVG(3); break;
    default: FV_AVG(4); break;
    }
#undef FV_AVG
}

// The chemistry pass after a multi-stage average (secondOrderStepSolverRK.cpp:114-118,
// thirdOrderStepSolver.cpp:125-129) on U[from ^ 1] and the stored concentrations, then the CFL
// finalize over its partials; without chemistry the finalize over the average's partials.
cudaError_t chemistryAndFinalize(fv_handle* h, int from) {
    int blocks = (int)genericBlocks(h->P);
    if (h->cfg.chemistry != FV_CHEM_NONE) {
        chem::ChemParams C = h->chem;
        C.conc = h->conc;
        cudaError_t e = launchChemistry(h->cfg.n_species, h->cfg.eos, h->cfg.dims, h->P, C, h->U[from ^ 1], h->ck,
                                        h->blockMax, h->stream);
        if (e != cudaSuccess) return e;
        blocks = chemistryBlocks(h->P);
    }
    k_finalize<<<1, 1024, 0, h->stream>>>(h->P, h->ck, h->blockMax, blocks);
    return cudaGetLastError();
}

// SecondOrderRK: stage 1 U[from] -> U[from ^ 1] (concentrations of the start state), stage 2
// U[from ^ 1] -> Ustage, average (Ustage, U[from]) -> U[from ^ 1] with the CFL partials.
cudaError_t enqueueRk2(fv_handle* h, int from) {
    StepBuffers B1 = buffersFor(h, from);
    B1.pcIn = nullptr;  // the stages do not use the primitive cache
    B1.pcOut = nullptr;
    StepParams P2 = h->P;
    P2.conc = nullptr;  // stage 2 reads the first stage's own rho_k / M_k
    StepBuffers B2 = B1;
    B2.U = h->U[from ^ 1];
    B2.Un = h->Ustage;
    B2.prim0 = nullptr;
    const bool f64 = h->cfg.precision == FV_PREC_F64;
    cudaError_t e = f64 ? launchStepF64(h->P, B1, h->path, h->shape, h->stream)
                        : launchStepF32(h->P, B1, h->path, h->shape, h->stream);
    if (e != cudaSuccess) return e;
    e = f64 ? launchStepF64(P2, B2, h->path, h->shape, h->stream) : launchStepF32(P2, B2, h->path, h->shape, h->stream);
    if (e != cudaSuccess) return e;
    average(h, from, h->conc, h->conc, 0.5);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return chemistryAndFinalize(h, from);
}

// ThirdOrder (SSP-RK3): stage 1 U[from] -> U[from ^ 1]; stage 2 U[from ^ 1] -> Ustage;
// average 0.25 (Ustage, U[from]) -> U[from ^ 1] with its concentrations in concStage; stage 3
// U[from ^ 1] (concentrations concStage) -> Ustage; average 2/3 (Ustage, U[from]) -> U[from ^ 1]
// with the CFL partials; finalize.
cudaError_t enqueueRk3(fv_handle* h, int from) {
    const bool f64 = h->cfg.precision == FV_PREC_F64;
    auto stage = [&](const StepParams& Ps, const double* in, double* out, const double* prim) {
        StepBuffers B = buffersFor(h, from);
        B.pcIn = nullptr;  // the stages do not use the primitive cache
        B.pcOut = nullptr;
        B.U = in;
        B.Un = out;
        B.prim0 = prim;
        return f64 ? launchStepF64(Ps, B, h->path, h->shape, h->stream) : launchStepF32(Ps, B, h->path, h->shape, h->stream);
    };
    StepParams P2 = h->P, P3 = h->P;
    P2.conc = nullptr;         // the first stage's own rho_k / M_k
    P3.conc = h->concStage;    // the 0.25 average's concentrations
    cudaError_t e = stage(h->P, h->U[from], h->U[from ^ 1], h->prim0);
    if (e != cudaSuccess) return e;
    if ((e = stage(P2, h->U[from ^ 1], h->Ustage, nullptr)) != cudaSuccess) return e;
    average(h, from, h->conc, h->concStage, 0.25);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = stage(P3, h->U[from ^ 1], h->Ustage, nullptr)) != cudaSuccess) return e;
    average(h, from, h->conc, h->conc, 2. / 3.);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return chemistryAndFinalize(h, from);
}

cudaError_t enqueueStep(fv_handle* h, int from) {
    if (h->cfg.order == FV_ORDER_SECOND_RK) return enqueueRk2(h, from);
    if (h->cfg.order == FV_ORDER_THIRD || h->cfg.order == FV_ORDER_THIRD_CADA) return enqueueRk3(h, from);
    const StepBuffers B = buffersFor(h, from);
    if (h->cfg.diffusion) {
        // secondOrderStepSolver::calculateStep: the advection, then the diffusion stage of the
        // advected state with the same dt; main's CFL block reads the state after the stage
        cudaError_t e = launchStepF64(h->P, B, h->path, h->shape, h->stream);
        if (e != cudaSuccess) return e;
        e = launchDiffusion(h->cfg.n_species, h->cfg.eos, h->cfg.dims, h->P, h->L, h->diff, h->U[from ^ 1], h->ck,
                            h->blockMax, h->stream);
        if (e != cudaSuccess) return e;
        int blocks = diffusionBlocks(h->P);
        if (h->cfg.chemistry != FV_CHEM_NONE) {
            // then the chemistry of the phase the stage left (secondOrderStepSolver.cpp:87-91)
            chem::ChemParams C = h->chem;
            C.stage = h->diff.stagePrim;
            e = launchChemistry(h->cfg.n_species, h->cfg.eos, h->cfg.dims, h->P, C, h->U[from ^ 1], h->ck,
                                h->blockMax, h->stream);
            if (e != cudaSuccess) return e;
            blocks = chemistryBlocks(h->P);
        }
        k_finalize<<<1, 1024, 0, h->stream>>>(h->P, h->ck, h->blockMax, blocks);
        return cudaGetLastError();
    }
    if (h->cfg.chemistry == FV_CHEM_NONE) {
        // the step kernel's last CTA reduces the CFL partials and advances the clock
        StepParams Pf = h->P;
        Pf.fuseFinalize = 1;
        cudaError_t e = h->cfg.precision == FV_PREC_F64 ? launchStepF64(Pf, B, h->path, h->shape, h->stream)
                                                         : launchStepF32(Pf, B, h->path, h->shape, h->stream);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    cudaError_t e = h->cfg.precision == FV_PREC_F64 ? launchStepF64(h->P, B, h->path, h->shape, h->stream)
                                                     : launchStepF32(h->P, B, h->path, h->shape, h->stream);
    if (e != cudaSuccess) return e;
    int blocks = (int)stepBlocks(h);
    if (h->cfg.chemistry != FV_CHEM_NONE) {
        // secondOrderStepSolver::calculateStep: the chemistry of the advected state with the same
        // dt; main's CFL block then reads the state after the chemistry
        e = launchChemistry(h->cfg.n_species, h->cfg.eos, h->cfg.dims, h->P, h->chem, h->U[from ^ 1], h->ck,
                            h->blockMax, h->stream);
        if (e != cudaSuccess) return e;
        blocks = chemistryBlocks(h->P);
    }
    k_finalize<<<1, 1024, 0, h->stream>>>(h->P, h->ck, h->blockMax, blocks);
    return cudaGetLastError();
}

// Opt the chosen fused-march instantiation in to its dynamic shared memory; runs outside any
// stream capture (a launch with null buffers and the legacy stream only configures).
fv_status configureKernels(fv_handle* h) {
    if (h->path != PATH_MARCH) return FV_OK;
    StepBuffers B{};
    cudaError_t e = h->cfg.precision == FV_PREC_F64 ? launchStepF64(h->P, B, PATH_MARCH, h->shape, nullptr)
                                                     : launchStepF32(h->P, B, PATH_MARCH, h->shape, nullptr);
    if (e != cudaSuccess) return cudaFail(h, e, "kernel configuration");
    return FV_OK;
}

fv_status ensureScratch(fv_handle* h) {
    long long nb = std::max(marchBlocks(h->P, h->shape), genericBlocks(h->P));
    if (h->cfg.chemistry != FV_CHEM_NONE) nb = std::max<long long>(nb, chemistryBlocks(h->P));
    if (h->cfg.diffusion) nb = std::max<long long>(nb, diffusionBlocks(h->P));
    if (nb > h->blockMaxCap) {
        if (h->blockMax) cudaFree(h->blockMax);
        FV_CUDA(h, cudaMalloc(&h->blockMax, sizeof(double) * nb));
        h->blockMaxCap = nb;
    }
    if (configureKernels(h) != FV_OK) return FV_ERR_SYSTEM;
    if (h->cfg.precision == FV_PREC_F64 && h->path == PATH_MARCH && warpStripMarch(h->P) && !h->pc[0]) {
        // the FP64 warp strip's primitive cache: c_1..c_N, v_x, v_y, p and the 4 mixture
        // coefficients of each cell, one array per state buffer
        const size_t bytes = sizeof(double) * (size_t)(h->cfg.n_species + 7) * (size_t)h->P.ncell;
        FV_CUDA(h, cudaMalloc(&h->pc[0], bytes));
        FV_CUDA(h, cudaMalloc(&h->pc[1], bytes));
    }
    if (h->cfg.diffusion && !h->diff.face) {
        // the stage's buffers: star velocities and face quantities per face, the advected
        // primitives, the stage's primitives and the partial minima of its limits
        const int ns = h->cfg.n_species;
        const size_t nf = (size_t)h->L.nfaces, st = (size_t)h->P.stride;
        diff::DiffParams& X = h->diff;
        FV_CUDA(h, cudaMalloc(&X.starV, sizeof(double) * 3 * nf));
        FV_CUDA(h, cudaMalloc(&X.starP, sizeof(double) * nf));
        FV_CUDA(h, cudaMalloc(&X.face, sizeof(double) * diff::faceSlotCount(ns) * nf));
        FV_CUDA(h, cudaMalloc(&X.cellPrim, sizeof(double) * (2 * ns + 5) * st));
        FV_CUDA(h, cudaMalloc(&X.stagePrim, sizeof(double) * (ns + 6) * st));
        FV_CUDA(h, cudaMalloc(&X.partMin, sizeof(double) * 2 * (size_t)diffusionBlocks(h->P)));
        if (X.gs) {
            FV_CUDA(h, cudaMalloc(&X.wDiag, sizeof(double) * ns * st));
            FV_CUDA(h, cudaMalloc(&X.wFree, sizeof(double) * ns * st));
            FV_CUDA(h, cudaMalloc(&X.wOff, sizeof(double) * ns * 6 * st));
            FV_CUDA(h, cudaMalloc(&X.vDiag, sizeof(double) * st));
            FV_CUDA(h, cudaMalloc(&X.vFree, sizeof(double) * 3 * st));
            FV_CUDA(h, cudaMalloc(&X.vOff, sizeof(double) * 6 * st));
            FV_CUDA(h, cudaMalloc(&X.tDiag, sizeof(double) * st));
            FV_CUDA(h, cudaMalloc(&X.tFree, sizeof(double) * st));
            FV_CUDA(h, cudaMalloc(&X.tOff, sizeof(double) * 6 * st));
            FV_CUDA(h, cudaMalloc(&X.sol, sizeof(double) * (ns + 4) * st));
            FV_CUDA(h, cudaMalloc(&X.work, sizeof(double) * 7 * st));
            FV_CUDA(h, cudaMalloc(&X.cNew, sizeof(double) * (ns + 3) * st));
        }
        h->P.starV = X.starV;
        h->P.starP = X.starP;
        h->P.stagePrim = X.stagePrim;
        if (X.gs) FV_CUDA(h, configureDiffusion(h->cfg.dims, h->P));
    }
    if (h->path == PATH_GENERIC && !h->FS) {
        const size_t tsz = h->cfg.precision == FV_PREC_F64 ? sizeof(double) : sizeof(float);
        const int ns = h->cfg.n_species;
        const int nff = 2 * (ns + 1) + 10;
        const int nfl = ns + 1 + 3 + 1;
        FV_CUDA(h, cudaMalloc(&h->Pc, tsz * (ns + 4) * h->P.ncell));
        FV_CUDA(h, cudaMalloc(&h->FS, tsz * 2 * nff * h->L.nfaces));
        FV_CUDA(h, cudaMalloc(&h->FL, tsz * nfl * h->L.nfaces));
    }
    return FV_OK;
}

int choosePath(const fv_config& c) {
    if (c.dims < 2) return PATH_GENERIC;
    if (c.diffusion) return PATH_GENERIC;  // the stage reads the generic path's Riemann star velocities
    if (c.eos != FV_EOS_IDEAL && c.eos != FV_EOS_VAN_DER_WAALS) return PATH_GENERIC;  // real-gas mixtures
    if (c.order == FV_ORDER_THIRD || c.order == FV_ORDER_THIRD_CADA) return PATH_GENERIC;  // directional slopes: k_faces3
    for (int a = 0; a < c.dims; ++a)
        if (c.n[a] < 2) return PATH_GENERIC;
    return limiterZeroForNonPositiveR(c.limiter) ? PATH_MARCH : PATH_GENERIC;
}

MarchShape defaultShape(const fv_config& c) {
    if (c.dims == 2) return MarchShape{128, 1, 32};
    return MarchShape{32, 8, 32};
}

fv_status readClock(fv_handle* h) {
    FV_CUDA(h, cudaMemcpyAsync(h->ckHost, h->ck, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status clockError(fv_handle* h) {
    const int e = h->ckHost->err;
    if (!e) return FV_OK;
    switch (e) {
    case FV_ERR_RIEMANN: return fail(h, e, "Fatal error in Riemann solver.");
    case FV_ERR_BOUNDARY: return fail(h, e, "fixedValueSurface is not a valid cell boundary value");
    default: return fail(h, e, "device error");
    }
}

}  // namespace

// ============================================================================ C ABI
extern "C" {

int fv_abi_version(void) { return FV_ABI_VERSION; }

const char* fv_last_error(const fv_handle* h) { return h ? h->err.c_str() : kNoHandle; }

fv_status fv_create(const fv_config* cfg, fv_handle** out) {
    if (!cfg || !out) return FV_ERR_INIT;
    *out = nullptr;
    std::string e;
    if (!fvValidateConfig(*cfg, e)) {
        fprintf(stderr, "fv_create: %s\n", e.c_str());
        return FV_ERR_INIT;
    }
    fv_handle* h = new (std::nothrow) fv_handle();
    if (!h) return FV_ERR_SYSTEM;
    h->cfg = *cfg;
    cudaError_t ce = cudaGetDevice(&h->device);
    if (ce != cudaSuccess) {
        delete h;
        fprintf(stderr, "fv_create: no CUDA device: %s\n", cudaGetErrorString(ce));
        return FV_ERR_SYSTEM;
    }
    StepParams& P = h->P;
    memset(&P, 0, sizeof(P));
    P.dims = cfg->dims;
    for (int a = 0; a < 3; ++a) {
        P.n[a] = a < cfg->dims ? cfg->n[a] : 1;
        P.ext[a] = cfg->L[a];
    }
    P.periodic[0] = cfg->bc_vel[FV_PATCH_TAIL] == FV_BC_PERIODIC;
    P.periodic[1] = cfg->dims >= 2 && cfg->bc_vel[FV_PATCH_RIGHT] == FV_BC_PERIODIC;
    P.periodic[2] = cfg->dims >= 3 && cfg->bc_vel[FV_PATCH_BOTTOM] == FV_BC_PERIODIC;
    P.ncell = (long long)P.n[0] * P.n[1] * P.n[2];
    P.stride = P.ncell;
    P.limiter = cfg->limiter;
    P.flux = cfg->flux;
    P.gravity = cfg->gravity;
    P.courant_only = cfg->courant_only;
    P.courant = cfg->courant;
    P.min_dt = cfg->min_timestep;
    P.const_dt = cfg->const_timestep;
    fvMixParams(*cfg, P.mix);
    for (int p = 0; p < 6; ++p) {
        for (int k = 0; k < FV_MAX_SPECIES; ++k) {
            P.bc.conc[p][k] = cfg->bc_conc[p][k];
            P.bc.conc_value[p][k] = cfg->bc_conc_value[p][k];
        }
        P.bc.vel[p] = cfg->bc_vel[p];
        for (int d = 0; d < 3; ++d) P.bc.vel_value[p][d] = cfg->bc_vel_value[p][d];
        P.bc.p[p] = cfg->bc_p[p];
        P.bc.p_value[p] = cfg->bc_p_value[p];
    }
    h->nConserved = cfg->n_species + 5;
    P.nmom = cfg->dims;
    // rows are staged with 16-byte aligned bulk copies: field and row pitches must be even
    P.tma = (P.n[0] % 2 == 0) ? 1 : 0;
    // 2D steps of the fused march run the warp-strip layout (FP32 flux: fv_warp2d.cuh, whose
    // fields are addressed with 32-bit offsets; FP64: fv_warp2d64.cuh); the FP32 one stages rows
    // by 8-byte copies, so its staging needs no even row length
    P.warp2d = (cfg->dims == 2 && (cfg->precision == FV_PREC_F64 || P.ncell * (cfg->n_species + 5) < (1LL << 31)))
                   ? 1 : 0;
    if (P.warp2d && cfg->precision == FV_PREC_F32_FLUX) P.tma = 1;
    P.hancock = cfg->order == FV_ORDER_SECOND ? 1 : 0;
    P.third = (cfg->order == FV_ORDER_THIRD || cfg->order == FV_ORDER_THIRD_CADA) ? 1 : 0;
    P.cada = cfg->order == FV_ORDER_THIRD_CADA ? 1 : 0;
    h->path = choosePath(*cfg);
    h->chem.mech = cfg->chemistry;
    h->chem.solver = cfg->chem_solver;
    h->chem.maxIter = cfg->chem_max_iter;
    h->chem.Af = cfg->chem_forward.A;
    h->chem.nf = cfg->chem_forward.n;
    h->chem.Ef = cfg->chem_forward.E;
    h->chem.Ab = cfg->chem_backward.A;
    h->chem.nb = cfg->chem_backward.n;
    h->chem.Eb = cfg->chem_backward.E;
    h->chem.q = cfg->chem_q;
    h->chem.conc = nullptr;  // the multi-stage enqueues pass the stored concentrations
    h->chem.stage = nullptr;  // the diffusion enqueue passes the stage's primitives
    if (cfg->diffusion) {
        diff::DiffParams& X = h->diff;
        X.mu = cfg->mu_const;
        X.D = cfg->D_const;
        X.kappa = cfg->kappa_const;
        X.transport = cfg->transport;
        for (int k = 0; k < FV_MAX_SPECIES; ++k) {
            X.diam[k] = cfg->transport_diameter[k];
            X.ljEps[k] = cfg->transport_lj_eps[k];
            X.ljSig[k] = cfg->transport_lj_sigma[k];
        }
        X.enthalpy = cfg->enthalpy_flow != FV_ENTHALPY_NO;
        X.enthImplicit = cfg->enthalpy_flow == FV_ENTHALPY_IMPLICIT;
        X.molmass = cfg->molmass_diffusion != 0;
        // gravity invalidates the star velocities (secondOrderStepSolver.cpp:71-73); the
        // "linear" reconstruction takes the cell velocities' gradient (Diffusion.cpp:178-184)
        X.interpV = cfg->gravity || cfg->linear_reconstruction;
        X.dtDiff = cfg->diffusion_timestep != 0;
        X.gs = cfg->sle_solver != FV_SLE_EXPLICIT;
        X.sle = cfg->sle_solver;
        X.maxIter = cfg->sle_max_iter;
        X.coeffSource = cfg->dt_coeff_source;
        X.coeffDiff = cfg->dt_coeff_diffusion;
    }
    h->shape = defaultShape(*cfg);

    // generic face layout
    long long base = 0;
    for (int a = 0; a < 3; ++a) {
        h->L.faceBase[a] = base;
        if (a < cfg->dims) {
            long long cnt = P.n[a] + 1;
            for (int b = 0; b < 3; ++b)
                if (b != a) cnt *= P.n[b];
            base += cnt;
        }
    }
    h->L.nfaces = base;

    std::vector<double> geo;
    size_t off[3][5];
    int nAxis[3];
    buildGeometry(*cfg, geo, off, nAxis);

    auto bail = [&](cudaError_t e2, const char* what) {
        fprintf(stderr, "fv_create: %s: %s\n", what, cudaGetErrorString(e2));
        fv_destroy(h);
        return FV_ERR_SYSTEM;
    };
    if ((ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(ce, "stream");
    if ((ce = cudaEventCreate(&h->ev0)) != cudaSuccess) return bail(ce, "event");
    if ((ce = cudaEventCreate(&h->ev1)) != cudaSuccess) return bail(ce, "event");
    const size_t stateBytes = sizeof(double) * h->nConserved * P.ncell;
    for (int b = 0; b < 2; ++b)
        if ((ce = cudaMalloc(&h->U[b], stateBytes)) != cudaSuccess) return bail(ce, "state");
    if (cfg->order != FV_ORDER_SECOND) {
        // the last stage's state and the averaged concentrations c_0..c_N (ThirdOrder: also those
        // of its intermediate average)
        const size_t concBytes = sizeof(double) * (cfg->n_species + 1) * P.ncell;
        if ((ce = cudaMalloc(&h->Ustage, stateBytes)) != cudaSuccess) return bail(ce, "stage state");
        if ((ce = cudaMalloc(&h->conc, concBytes)) != cudaSuccess) return bail(ce, "concentrations");
        if ((cfg->order == FV_ORDER_THIRD || cfg->order == FV_ORDER_THIRD_CADA) &&
            (ce = cudaMalloc(&h->concStage, concBytes)) != cudaSuccess)
            return bail(ce, "stage concentrations");
        P.conc = h->conc;
    }
    if ((ce = cudaMalloc(&h->prim0, sizeof(double) * (cfg->n_species + 4) * P.ncell)) != cudaSuccess)
        return bail(ce, "restart set");
    if ((ce = cudaMalloc(&h->ck, sizeof(DevClock))) != cudaSuccess) return bail(ce, "clock");
    if ((ce = cudaMallocHost(&h->ckHost, sizeof(DevClock))) != cudaSuccess) return bail(ce, "clock mirror");
    if ((ce = cudaMalloc(&h->geo, sizeof(double) * geo.size())) != cudaSuccess) return bail(ce, "geometry");
    if ((ce = cudaMemcpy(h->geo, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(ce, "geometry copy");
    for (int a = 0; a < 3; ++a) {
        P.geo.h[a] = h->geo + off[a][0];
        P.geo.cc[a] = h->geo + off[a][1];
        P.geo.fpos[a] = h->geo + off[a][2];
        P.geo.aabb[a] = h->geo + off[a][3];
        P.geo.abab[a] = h->geo + off[a][4];
    }
    memset(h->ckHost, 0, sizeof(DevClock));
    h->ckHost->dt = cfg->min_timestep;
    h->ckHost->dt_free = cfg->min_timestep;
    h->ckHost->t_end = std::numeric_limits<double>::infinity();
    h->ckHost->first = 1;
    for (int d = 0; d < 3; ++d) {
        h->ckHost->g[d] = cfg->g[d];
        h->ckHost->g_delta[d] = cfg->g_delta[d];
    }
    if ((ce = cudaMemcpy(h->ck, h->ckHost, sizeof(DevClock), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(ce, "clock copy");
    if (ensureScratch(h) != FV_OK) {
        fprintf(stderr, "fv_create: %s\n", h->err.c_str());
        fv_destroy(h);
        return FV_ERR_SYSTEM;
    }
    *out = h;
    return FV_OK;
}

void fv_destroy(fv_handle* h) {
    if (!h) return;
    destroyGraphs(h);
    if (h->stream) cudaStreamSynchronize(h->stream);
    releaseTrajectory(h);
    for (auto& u : h->U)
        if (u) cudaFree(u);
    if (h->prim0) cudaFree(h->prim0);
    if (h->Ustage) cudaFree(h->Ustage);
    if (h->conc) cudaFree(h->conc);
    if (h->concStage) cudaFree(h->concStage);
    if (h->ck) cudaFree(h->ck);
    if (h->ckHost) cudaFreeHost(h->ckHost);
    if (h->blockMax) cudaFree(h->blockMax);
    for (double* q : h->pc)
        if (q) cudaFree(q);
    if (h->geo) cudaFree(h->geo);
    if (h->Pc) cudaFree(h->Pc);
    if (h->FS) cudaFree(h->FS);
    if (h->FL) cudaFree(h->FL);
    if (h->outBuf) cudaFree(h->outBuf);
    for (double* q : {h->diff.starV, h->diff.starP, h->diff.face, h->diff.cellPrim, h->diff.stagePrim, h->diff.partMin, h->diff.wDiag,
                      h->diff.wFree, h->diff.wOff, h->diff.vDiag, h->diff.vFree, h->diff.vOff, h->diff.tDiag,
                      h->diff.tFree, h->diff.tOff, h->diff.sol, h->diff.work, h->diff.cNew})
        if (q) cudaFree(q);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

// Carry all three momentum components when the restart set has a transverse velocity.
static fv_status setMomentumComponents(fv_handle* h) {
    int nmom = h->cfg.dims;
    if (h->cfg.dims < 3) {
        FV_CUDA(h, cudaMemsetAsync(&h->ck->flag, 0, sizeof(int), h->stream));
        const unsigned g = (unsigned)((h->P.ncell + 255) / 256);
        k_transverse<<<g, 256, 0, h->stream>>>(h->P, h->prim0, &h->ck->flag);
        FV_CUDA(h, cudaGetLastError());
        int flag = 0;
        FV_CUDA(h, cudaMemcpyAsync(&flag, &h->ck->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        FV_CUDA(h, cudaStreamSynchronize(h->stream));
        if (flag) nmom = 3;
        // a fixed-value patch velocity with a transverse component feeds the transverse momentum
        for (int p = 0; p < 6; ++p) {
            const int t = h->cfg.bc_vel[p];
            if (t != FV_BC_FIXED_CELL && t != FV_BC_FIXED_SURFACE) continue;
            for (int d = h->cfg.dims; d < 3; ++d)
                if (h->cfg.bc_vel_value[p][d] != 0.0) nmom = 3;
        }
    }
    if (nmom != h->P.nmom) {
        h->P.nmom = nmom;
        destroyGraphs(h);
        // the kernel choice depends on the carried momenta (warp strip with two): configure it
        return ensureScratch(h);
    }
    return FV_OK;
}

static fv_status resetClock(fv_handle* h) {
    DevClock& c = *h->ckHost;
    memset(&c, 0, sizeof(DevClock));
    // Schemi.cpp:664-668: the first step is the minimal time step, or the constant step
    c.dt = h->cfg.const_timestep > 0 ? h->cfg.const_timestep : h->cfg.min_timestep;
    c.dt_free = c.dt;
    c.t_end = std::numeric_limits<double>::infinity();
    c.first = 1;
    for (int d = 0; d < 3; ++d) {
        c.g[d] = h->cfg.g[d];
        c.g_delta[d] = h->cfg.g_delta[d];
    }
    FV_CUDA(h, cudaMemcpyAsync(h->ck, h->ckHost, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
    return FV_OK;
}

fv_status fv_upload_device(fv_handle* h, const double* const* prim_dev) {
    if (!h || !prim_dev) return FV_ERR_INIT;
    const int nf = h->cfg.n_species + 4;
    const long long n = h->P.ncell;
    for (int f = 0; f < nf; ++f)
        FV_CUDA(h, cudaMemcpyAsync(h->prim0 + f * n, prim_dev[f], sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                   h->stream));
    h->cur = 0;
    fv_status st = setMomentumComponents(h);
    if (st != FV_OK) return st;
    upload(h, h->prim0);
    FV_CUDA(h, cudaGetLastError());
    st = resetClock(h);
    if (st != FV_OK) return st;
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status fv_upload(fv_handle* h, const double* const* prim) {
    if (!h || !prim) return FV_ERR_INIT;
    const int nf = h->cfg.n_species + 4;
    const long long n = h->P.ncell;
    for (int f = 0; f < nf; ++f)
        FV_CUDA(h, cudaMemcpyAsync(h->prim0 + f * n, prim[f], sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    h->cur = 0;
    fv_status st = setMomentumComponents(h);
    if (st != FV_OK) return st;
    upload(h, h->prim0);
    FV_CUDA(h, cudaGetLastError());
    st = resetClock(h);
    if (st != FV_OK) return st;
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status fv_step(fv_handle* h, double* dt_used, double* dt_next) {
    if (!h) return FV_ERR_INIT;
    // single steps are never clamped to an end time
    h->ckHost->t_end = std::numeric_limits<double>::infinity();
    FV_CUDA(h, cudaMemcpyAsync(&h->ck->t_end, &h->ckHost->t_end, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    FV_CUDA(h, cudaMemsetAsync(&h->ck->done, 0, sizeof(int), h->stream));
    FV_CUDA(h, enqueueStep(h, h->cur));
    h->cur ^= 1;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    if (dt_used) *dt_used = h->ckHost->dt_used;
    if (dt_next) *dt_next = h->ckHost->dt;
    return clockError(h);
}

fv_status fv_run(fv_handle* h, double t_end, long long max_steps, fv_run_stats* stats) {
    if (!h) return FV_ERR_INIT;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    const long long steps0 = h->ckHost->steps;
    // main: mesh_.setTimestep(std::min(mesh_.timestep(), timeOfCalculation)) before the loop; in
    // the loop's own form (Schemi.cpp:933-935) so that a run resumed with the same end time takes
    // the step the device clamp already chose
    DevClock& c = *h->ckHost;
    c.t_end = t_end;
    c.done = !(c.time < t_end);
    c.dt = (c.time + c.dt_free) > t_end ? t_end - c.time : c.dt_free;
    FV_CUDA(h, cudaMemcpyAsync(h->ck, h->ckHost, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
    const int chunk = 32;  // steps per graph
    if (h->graphSteps != chunk) {
        destroyGraphs(h);
        for (int start = 0; start < 2; ++start) {
            cudaGraph_t g;
            FV_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            int from = start;
            for (int s = 0; s < chunk; ++s) {
                cudaError_t e = enqueueStep(h, from);
                if (e != cudaSuccess) {
                    cudaStreamEndCapture(h->stream, &g);
                    return cudaFail(h, e, "step capture");
                }
                from ^= 1;
            }
            FV_CUDA(h, cudaStreamEndCapture(h->stream, &g));
            FV_CUDA(h, cudaGraphInstantiate(&h->graph[start], g, 0));
            cudaGraphDestroy(g);
        }
        h->graphSteps = chunk;
    }
    FV_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    long long done = 0;
    while (!c.done && done < max_steps) {
        const long long left = max_steps - done;
        if (left >= chunk) {
            // a graph of `chunk` steps; steps after the end time are no-ops that leave the
            // state in place, so the current buffer follows the executed step count
            FV_CUDA(h, cudaGraphLaunch(h->graph[h->cur], h->stream));
        } else {
            int from = h->cur;
            for (long long s = 0; s < left; ++s) {
                FV_CUDA(h, enqueueStep(h, from));
                from ^= 1;
            }
        }
        const long long before = c.steps;
        st = readClock(h);
        if (st != FV_OK) return st;
        const long long executed = c.steps - before;
        if (executed & 1) h->cur ^= 1;
        done += (left >= chunk) ? chunk : left;
        if (c.err) break;
    }
    FV_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    FV_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    if (stats) {
        stats->time = c.time;
        stats->dt_next = c.dt;
        stats->steps = c.steps - steps0;
        stats->device_ms = ms;
    }
    return clockError(h);
}

fv_status fv_download(fv_handle* h, double* const* out) {
    if (!h || !out) return FV_ERR_INIT;
    const long long n = h->P.ncell;
    if (!h->outBuf) FV_CUDA(h, cudaMalloc(&h->outBuf, sizeof(double) * FV_F_COUNT * n));
    download(h);
    FV_CUDA(h, cudaGetLastError());
    for (int f = 0; f < FV_F_COUNT; ++f) {
        if (!out[f]) continue;
        const bool species = (f >= FV_F_CONC && f < FV_F_CONC + FV_MAX_SPECIES) ||
                             (f >= FV_F_RHO_K && f < FV_F_RHO_K + FV_MAX_SPECIES);
        if (species) {
            const int k = f >= FV_F_RHO_K ? f - FV_F_RHO_K : f - FV_F_CONC;
            if (k >= h->cfg.n_species) continue;
        }
        FV_CUDA(h, cudaMemcpyAsync(out[f], h->outBuf + f * n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    }
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status fv_get_time(const fv_handle* hc, double* time, double* dt) {
    fv_handle* h = const_cast<fv_handle*>(hc);
    if (!h) return FV_ERR_INIT;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    if (time) *time = h->ckHost->time;
    if (dt) *dt = h->ckHost->dt;
    return FV_OK;
}

fv_status fv_get_source_timestep(const fv_handle* hc, double* dt_source) {
    fv_handle* h = const_cast<fv_handle*>(hc);
    if (!h) return FV_ERR_INIT;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    if (dt_source) *dt_source = h->ckHost->dtSourceLast > 0 ? h->ckHost->dtSourceLast : kVeryBigD();
    return FV_OK;
}

fv_status fv_set_time(fv_handle* h, double time, double dt) {
    if (!h) return FV_ERR_INIT;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    h->ckHost->time = time;
    h->ckHost->dt = dt;
    h->ckHost->dt_free = dt;
    FV_CUDA(h, cudaMemcpyAsync(h->ck, h->ckHost, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status fv_state_device(fv_handle* h, double** fields, int* n_fields, long long* n_cells) {
    if (!h) return FV_ERR_INIT;
    if (n_fields) *n_fields = h->nConserved;
    if (n_cells) *n_cells = h->P.ncell;
    if (fields)
        for (int f = 0; f < h->nConserved; ++f) fields[f] = h->U[h->cur] + f * h->P.stride;
    return FV_OK;
}

fv_status fv_sync(fv_handle* h) {
    if (!h) return FV_ERR_INIT;
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status fv_begin_steps(fv_handle* h) {
    if (!h) return FV_ERR_INIT;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    h->ckHost->t_end = std::numeric_limits<double>::infinity();
    h->ckHost->done = 0;
    FV_CUDA(h, cudaMemcpyAsync(h->ck, h->ckHost, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
    FV_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status fv_step_async(fv_handle* h) {
    if (!h) return FV_ERR_INIT;
    FV_CUDA(h, enqueueStep(h, h->cur));
    h->cur ^= 1;
    return FV_OK;
}

void* fv_stream(fv_handle* h) { return h ? (void*)h->stream : nullptr; }

fv_status fv_check(fv_handle* h) {
    if (!h) return FV_ERR_INIT;
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    return clockError(h);
}

long long fv_kernels_per_step(const fv_handle* h) {
    if (!h) return 0;
    const int stage = h->path == PATH_MARCH ? 1 : 4;
    const int chem = h->cfg.chemistry != FV_CHEM_NONE ? 1 : 0;
    if (h->cfg.diffusion && h->diff.gs)
        // prim, faces, the mass-fraction matrices and N solves, concentrations, the averaged
        // enthalpy flow, velocity / temperature matrices and nmom + 1 solves, phase, source, finalize
        return stage + 2 + 1 + (h->diff.sle == FV_SLE_NO_SOLVER ? 0 : h->cfg.n_species + h->P.nmom + 1) + 1 +
               (h->diff.enthalpy ? 1 : 0) + 1 + 1 + 1 + 1 + chem;
    if (h->cfg.diffusion) return stage + 5 + chem;  // the stage's 4 kernels, [chemistry,] finalize
    if (h->cfg.order == FV_ORDER_SECOND_RK) return 2 * stage + 2 + chem;  // two stages, average, finalize
    if (h->cfg.order == FV_ORDER_THIRD || h->cfg.order == FV_ORDER_THIRD_CADA)
        return 3 * stage + 3 + chem;  // three stages, two averages, finalize
    return chem ? stage + 2 : stage;  // without chemistry the step kernel finalizes itself
}

// ---- introspection used by the tests and the bench (no reference counterpart)
int fv_step_path(const fv_handle* h) { return h ? h->path : -1; }

fv_status fv_set_march_shape(fv_handle* h, int bx, int by, int rows) {
    if (!h) return FV_ERR_INIT;
    MarchShape s{bx, by, rows};
    if (!marchShapeSupported(h->cfg.dims, s) || rows < 1) return fail(h, FV_ERR_INIT, "unsupported march shape");
    h->shape = s;
    destroyGraphs(h);
    return ensureScratch(h);
}

// Row staging through shared memory with bulk async copies (1) or direct global loads (0);
// staging needs an even number of cells along x.
fv_status fv_set_staging(fv_handle* h, int on) {
    if (!h) return FV_ERR_INIT;
    // the CTA march stages rows by 16-byte bulk copies (nx even); the warp-strip march copies
    // 8 bytes per lane
    const int want = (on && (h->P.n[0] % 2 == 0 || (h->P.warp2d && h->cfg.precision == FV_PREC_F32_FLUX))) ? 1 : 0;
    if (want != h->P.tma) {
        h->P.tma = want;
        destroyGraphs(h);
    }
    return FV_OK;
}

int fv_get_staging(const fv_handle* h) { return h ? h->P.tma : -1; }

fv_status fv_force_generic(fv_handle* h) {
    if (!h) return FV_ERR_INIT;
    h->path = PATH_GENERIC;
    destroyGraphs(h);
    return ensureScratch(h);
}

// Time `iters` launches of one step kernel (no finalize, state untouched) for the shape.
fv_status fv_time_step_kernel(fv_handle* h, int iters, float* ms_per_step) {
    if (!h || iters < 1) return FV_ERR_INIT;
    const StepBuffers B = buffersFor(h, h->cur);
    // use the second buffer as the output; U[cur] is unchanged
    FV_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    for (int i = 0; i < iters; ++i) {
        cudaError_t e = h->cfg.precision == FV_PREC_F64 ? launchStepF64(h->P, B, h->path, h->shape, h->stream)
                                                         : launchStepF32(h->P, B, h->path, h->shape, h->stream);
        if (e != cudaSuccess) return cudaFail(h, e, "step launch");
    }
    FV_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    FV_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    *ms_per_step = ms / iters;
    return FV_OK;
}

}  // extern "C"

// ============================================================================ shapes
namespace fv {
long long marchBlocks(const StepParams& P, const MarchShape& s) {
    if (P.dims < 2) return 0;
    const int cols = marchTileColumns(P, s.bx);
    const long long gx = (P.n[0] + cols - 1) / cols;
    if (P.dims == 2) return gx * ((P.n[1] + s.rows - 1) / s.rows) * marchPartialsPerTile(P, s.bx);
    const long long gy = (P.n[1] + s.by - 3) / (s.by - 2);
    return gx * gy * ((P.n[2] + s.rows - 1) / s.rows);
}
long long genericBlocks(const StepParams& P) { return (P.ncell + 127) / 128; }
bool marchShapeSupported(int dims, const MarchShape& s) {
    if (dims == 2) return s.by == 1 && (s.bx == 64 || s.bx == 128 || s.bx == 256);
    if (dims == 3) return (s.bx == 32 && (s.by == 8 || s.by == 16)) || (s.bx == 64 && s.by == 8);
    return false;
}
}  // namespace fv
