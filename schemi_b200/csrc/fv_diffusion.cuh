// fv_diffusion.cuh -- the diffusion stage of secondOrderStepSolver::calculateStep
// (secondOrderStepSolver.cpp:69-80, Diffusion.cpp:20-1061) on the generic path, FP64 in the
// reference's operation order.
//
// Scope: molecular transport with the constant, hard-sphere or Lennard-Jones coefficients, no
// turbulence, the explicit solver (each field advances as (explOldTime + freeTerm dt) /
// centralDiagonale; this file) or the implicit matrices and their solvers
// (fv_diffusion_gs.cuh), ideal and van der Waals mixtures, the enthalpy flow off, explicit or
// implicit, the molar-mass (Maxwell-Stefan) correction on or off.  With turbulence off the
// stage's non-linearity loop stops after one pass (its convergence measure is the change of
// epsilon, 0), and its non-ideality term is multiplied by the turbulent tLambda, 0: that term
// (Diffusion.cpp:424-428, 608-617) adds signed zeros to the temperature's free term, which
// leave it unchanged, and is not evaluated.
//
// On this axis-aligned mesh a face normal is +-e_a, so a divergence reads only the axis
// component of a face vector: sum over the cell's faces of (F_a n_a) S in the cell's face order,
// exactly the reference's ((F & n) S) sums, whose other terms add zeros.  The kernels keep that
// component of the scalar gradients, the Maxwell-Stefan fluxes and the enthalpy flow.  The
// velocity's face tensor (dv / |d|^2) d (inner) or (dv / |dR|) dR / |dR| (patch) enters through
// its column a (the Laplacian flow) and through its transpose's column a (the deviatoric
// stress); the latter holds the transverse parts of the direction, which a patch whose centre
// sits off the cell's axis line has, and is kept whole.
//
//   k_diff_prim   cell primitives of the advected state (Advection.cpp:455-479): c_k, v, p, T,
//                 mass fractions (diffusiveFields.cpp:24-46)
//   k_diff_faces  per face: interpolated concentrations, density and temperature; surface
//                 gradients of the mass fractions, molar fractions, velocity and temperature with
//                 the calculated* boundary values of boundaryConditionValue.hpp; the fluxes of
//                 the explicit Laplacians (SLEMatrix.cpp:2054-2110), the molar-mass correction
//                 (transportCoefficients.hpp:256-325,413-456), the explicit enthalpy flow, the
//                 deviatoric viscous stress (Diffusion.cpp:178-229,503-506)
//   k_diff_cells  per cell: divergences, source distribution (SLEMatrix.cpp:2166-2175), new mass
//                 fractions, concentrations, velocity and temperature, the recomputed phase
//                 (Diffusion.cpp:965-1025), the CFL signal of main's next block and the partial
//                 minima of the enthalpy and diffusion time-step limits
//   k_diff_source the stage's source time step (Diffusion.cpp:688-706,1036-1049)
#pragma once

#include "fv_diffusion_launch.h"
#include "fv_generic.cuh"

namespace fv {
namespace diff {


// face quantity slots: flowW_k, corr_k (k < N), enthalpy flow, velocity Laplacian flow (3),
// deviatoric stress (3), temperature Laplacian flow, maximal coefficient; for the implicit
// solver also the interpolated density and temperature and the face's transport coefficients
// mu, kappa and D_k
template <int NS> __host__ __device__ constexpr int faceSlots() { return faceSlotCount(NS); }
template <int NS> __device__ __forceinline__ int slotW(int k) { return k; }
template <int NS> __device__ __forceinline__ int slotCorr(int k) { return NS + k; }
template <int NS> __device__ __forceinline__ int slotEnt() { return 2 * NS; }
template <int NS> __device__ __forceinline__ int slotV(int d) { return 2 * NS + 1 + d; }
template <int NS> __device__ __forceinline__ int slotDev(int d) { return 2 * NS + 4 + d; }
template <int NS> __device__ __forceinline__ int slotT() { return 2 * NS + 7; }
template <int NS> __device__ __forceinline__ int slotMax() { return 2 * NS + 8; }
template <int NS> __device__ __forceinline__ int slotRho() { return 2 * NS + 9; }
template <int NS> __device__ __forceinline__ int slotTs() { return 2 * NS + 10; }
template <int NS> __device__ __forceinline__ int slotMu() { return 2 * NS + 11; }
template <int NS> __device__ __forceinline__ int slotKappa() { return 2 * NS + 12; }
template <int NS> __device__ __forceinline__ int slotDs(int k) { return 2 * NS + 13 + k; }
static_assert(faceSlotCount(1) == 3 * 1 + 13 && faceSlotCount(4) == 3 * 4 + 13, "slots 0 .. 3N + 12");

// ----------------------------------------------------------------------------- mixture functions
// mixtureIdeal.cpp / mixtureVanDerWaals.cpp with idealFluid.cpp / vanDerWaalsFluid.cpp
template <int NS, int EOS>
__device__ __forceinline__ void cvA(const MixParams& mp, const double* c, double& Cvm, double& am) {
    double X[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) X[k] = c[k + 1] / c[0];
    Cvm = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) Cvm += X[k] * mp.Cv[k];
    am = 0;
    if (EOS == FV_EOS_VAN_DER_WAALS) {
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int l = 0; l < NS; ++l) am += X[k] * X[l] * mp.a[k][l];
    }
}
template <int NS, int EOS>
__device__ __forceinline__ double mixCv(const MixParams& mp, const double* c) {
    double Cvm, am;
    cvA<NS, FV_EOS_IDEAL>(mp, c, Cvm, am);
    return Cvm;
}
template <int NS, int EOS>
__device__ __forceinline__ double nonIdeality(const MixParams& mp, const double* c) {
    if (EOS == FV_EOS_IDEAL) return 0;
    double Cvm, am;
    cvA<NS, EOS>(mp, c, Cvm, am);
    return -am * (c[0] * c[0]);
}
template <int NS, int EOS>
__device__ __forceinline__ double UvcFromT(const MixParams& mp, const double* c, double T) {
    double Cvm, am;
    cvA<NS, EOS>(mp, c, Cvm, am);
    if (EOS == FV_EOS_IDEAL) return Cvm * T;
    return Cvm * T - am * c[0];
}
// (UvcFromTk + pcFromTk) / T of species k alone at concentration ck (mixtureIdeal.cpp:291-298,
// mixtureVanDerWaals.cpp:452-459)
template <int EOS>
__device__ __forceinline__ double hkT(const MixParams& mp, double ck, double T, int k) {
    if (EOS == FV_EOS_IDEAL) return (mp.Cv[k] * T + mp.R * T) / T;
    const double a = mp.a[k][k], b = mp.b[k][k];
    return ((mp.Cv[k] * T - a * ck) + (mp.R * T / (1 - ck * b) - a * ck)) / T;
}

// ----------------------------------------------------------------------------- transport models
// transportCoefficients::calculateCoefficients (transportCoefficients.hpp:124-133) of one point
// from its temperature T, pressure p and concentrations c[0..N]: the constants
// (abstractTransportModel.cpp:82-187), the hard-sphere kinetic theory
// (hardSpheresTransportModel.cpp) or the Lennard-Jones collision integrals
// (LennardJonesTransportModel.cpp), each species' value added to the constant, mixed by Wilke's
// rule.  The hard-sphere forms use only sqrt and division (correctly rounded here as in the
// reference); the Lennard-Jones integrals call pow and exp, whose last bit may differ from the
// host library's.
__device__ __forceinline__ double ljOmegaMuKappa(double Ts) {
    return 1.16145 * pow(Ts, -0.14874) + 0.52487 * exp(-0.77320 * Ts) + 2.16178 * exp(-2.4378 * Ts);
}
__device__ __forceinline__ double ljOmegaD(double Ts) {
    return 1.06036 * pow(Ts, -0.1561) + 0.19300 * exp(-0.47635 * Ts) + 1.03587 * exp(-1.52996 * Ts) +
           1.76474 * exp(-3.89411 * Ts);
}
// a species' viscosity and conductivity (hardSpheresTransportModel.cpp:11-38,
// LennardJonesTransportModel.cpp:31-60)
__device__ __forceinline__ void speciesMuKappa(const DiffParams& X, double M, double T, int k, double& mu,
                                               double& kappa) {
    if (X.transport == FV_TRANSPORT_LENNARD_JONES) {
        const double Om = ljOmegaMuKappa(T / X.ljEps[k]);
        const double s = X.ljSig[k];
        mu = X.mu + 2.6693E-6 * sqrt(1E3) * sqrt(M * T) / Om / (s * s);
        kappa = X.kappa + 4.184 * 1.9891E-2 / sqrt(1E3) * sqrt(T / M) / Om / (s * s);
    } else {
        const double s = X.diam[k];
        mu = X.mu + 2.6693E-6 * sqrt(1E3) * sqrt(M * T) / (s * s);
        kappa = X.kappa + 4.184 * 1.9891E-2 / sqrt(1E3) * sqrt(T / M) / (s * s);
    }
}
// binary coefficient of the pair (k1, k2) (calculateDm)
__device__ __forceinline__ double binaryD(const DiffParams& X, const double* M, int k1, int k2, double T, double p) {
    const double M12 = 2 * M[k1] * M[k2] / (M[k1] + M[k2]);
    if (X.transport == FV_TRANSPORT_LENNARD_JONES) {
        const double Om = ljOmegaD(T / sqrt(X.ljEps[k1] * X.ljEps[k2]));
        const double s = 0.5 * (X.ljSig[k1] + X.ljSig[k2]);
        return X.D + 2.6280E-7 / sqrt(1E3) / Om * sqrt(T * T * T / M12) / (p / 101325. * (s * s));
    }
    const double s = 0.5 * (X.diam[k1] + X.diam[k2]);
    return X.D + 2.6280E-7 / sqrt(1E3) * sqrt(T * T * T / M12) / (p / 101325. * (s * s));
}
// Wilke's mixing rule (hardSpheresTransportModel.cpp:55-77; kappa: 0.85 on Phi, :189-210)
template <int NS>
__device__ __forceinline__ double wilke(const double* x, const double* q, const double* M, bool kappa) {
    double mix = 0;
#pragma unroll
    for (int k1 = 0; k1 < NS; ++k1) {
        double Phi_k1 = 0;
#pragma unroll
        for (int k2 = 0; k2 < NS; ++k2) {
            const double num = 1 + sqrt(q[k1] / q[k2]) * sqrt(sqrt(M[k2] / M[k1]));
            const double dem = 8 * (1 + M[k1] / M[k2]);
            const double Phi = kappa ? 0.85 * num * num / sqrt(dem) : num * num / sqrt(dem);
            Phi_k1 += x[k2] * Phi;
        }
        mix += x[k1] * q[k1] / Phi_k1;
    }
    return mix;
}
// the viscosity and conductivity of a point
template <int NS>
__device__ __forceinline__ void pointMuKappa(const DiffParams& X, const double* M, double T, const double* c,
                                             double& mu, double& kappa) {
    if (X.transport == FV_TRANSPORT_CONSTANT) {
        mu = X.mu;
        kappa = X.kappa;
        return;
    }
    double x[NS], muk[NS], kk[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        x[k] = c[k + 1] / c[0];
        speciesMuKappa(X, M[k], T, k, muk[k], kk[k]);
    }
    mu = wilke<NS>(x, muk, M, false);
    kappa = wilke<NS>(x, kk, M, true);
}
// the binary matrix of a point (the diagonal unused)
template <int NS>
__device__ __forceinline__ void pointDm(const DiffParams& X, const double* M, double T, double p, double (*Dm)[NS]) {
#pragma unroll
    for (int k1 = 0; k1 < NS; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < NS; ++k2)
            Dm[k1][k2] = (k1 == k2) ? 0.0 : (X.transport == FV_TRANSPORT_CONSTANT ? X.D : binaryD(X, M, k1, k2, T, p));
}
// a face's coefficient of each species in the mixture (calculateDs, surface variant,
// hardSpheresTransportModel.cpp:360-388: the inverse sum guarded by the stabilizator)
template <int NS>
__device__ __forceinline__ void faceDs(const DiffParams& X, const double* c, const double (*Dm)[NS], double* Ds) {
    if (X.transport == FV_TRANSPORT_CONSTANT) {
#pragma unroll
        for (int k = 0; k < NS; ++k) Ds[k] = X.D;
        return;
    }
    double x[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) x[k] = c[k + 1] / c[0];
#pragma unroll
    for (int k1 = 0; k1 < NS; ++k1) {
        double rDk = 0;
#pragma unroll
        for (int k2 = 0; k2 < NS; ++k2)
            if (k1 != k2) rDk += x[k2] / Dm[k1][k2];
        if (rDk >= Num<double>::stab()) {
            rDk *= 1.0 / (1.0 - x[k1] + Num<double>::stab());
            Ds[k1] = 1 / rDk;
        } else {
            Ds[k1] = Num<double>::stab();
        }
    }
}

// calculatedTemperature (boundaryConditionValue.hpp:89-108, 326-345): the temperature of the
// patch's concentrations and pressure, surface or cell variant
template <int NS, int EOS>
__device__ __forceinline__ double boundaryT(const StepParams& P, int patch, const double* cO, double pO, bool cell,
                                            bool& bad) {
    double cB[NS + 1];
    cB[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        cB[k] = cell ? cellGhostScalar<double, NS>(P, patch, k - 1, cO[k], bad)
                     : surfaceScalar<double, NS>(P, patch, k - 1, cO[k]);
        cB[0] += cB[k];
    }
    const double pB = cell ? cellGhostScalar<double, NS>(P, patch, NS + 3, pO, bad)
                           : surfaceScalar<double, NS>(P, patch, NS + 3, pO);
    return Mixture<double, NS, EOS>::TFromUv(P.mix, cB, Mixture<double, NS, EOS>::UvFromp(P.mix, cB, pB));
}

// Maxwell-Stefan fluxes of one face direction (effectiveTransportCoefficients::caclulateDFluxes
// without turbulence, transportCoefficients.hpp:256-325, and its pivoting Gauss elimination,
// :413-456, with normalize, :544-550): the row of the least concentration replaced by
// sum N_k M_k J_k = 0, the result scaled by M_k c_k.
template <int NS>
__device__ __forceinline__ void maxwellStefan(const double* Nc, const double* M, const double (*Dm)[NS],
                                              const double* gX, double* out) {
    double c[NS];
#pragma unroll
    for (int k = 1; k <= NS; ++k) c[k - 1] = Nc[k];
    double cmin = c[0];
#pragma unroll
    for (int k = 1; k < NS; ++k) cmin = smin(cmin, c[k]);
    int replaceIndex = 0;
    for (int k = NS - 1; k >= 0; --k)
        if (cmin == c[k]) replaceIndex = k + 1;  // the first index holding the minimum
    double A[NS][NS], b[NS];
#pragma unroll
    for (int r = 0; r < NS; ++r) {
        b[r] = -gX[r];
#pragma unroll
        for (int q = 0; q < NS; ++q) A[r][q] = 0.0;
    }
#pragma unroll
    for (int k1 = 1; k1 <= NS; ++k1) {
        if (k1 != replaceIndex) {
#pragma unroll
            for (int k2 = 1; k2 <= NS; ++k2) {
                if (k1 == k2) continue;
                const double Aij = Nc[k1] * Nc[k2] / (Nc[0] * Nc[0] * Dm[k1 - 1][k2 - 1]);
                A[k1 - 1][k2 - 1] = -Aij;
                A[k1 - 1][k1 - 1] += Aij;
            }
        } else {
            b[k1 - 1] = 0;
#pragma unroll
            for (int k2 = 1; k2 <= NS; ++k2) A[k1 - 1][k2 - 1] = Nc[k2] * M[k2 - 1];
        }
    }
#pragma unroll
    for (int k = 0; k < NS - 1; ++k) {
        double mv = A[k][k];
        int mi = k;
#pragma unroll
        for (int r = k + 1; r < NS; ++r)
            if (A[r][k] > mv) { mv = A[r][k]; mi = r; }
        if (mi != k) {
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                const double t = A[mi][q];
                A[mi][q] = A[k][q];
                A[k][q] = t;
            }
            const double t = b[mi];
            b[mi] = b[k];
            b[k] = t;
        }
    }
#pragma unroll
    for (int k = 0; k < NS - 1; ++k)
#pragma unroll
        for (int i = k + 1; i < NS; ++i) {
            const double ratio = A[i][k] / (A[k][k] + Num<double>::stab());
#pragma unroll
            for (int j = k + 1; j < NS; ++j) A[i][j] = A[i][j] - ratio * A[k][j];
            b[i] = b[i] - ratio * b[k];
        }
    double phi[NS];
    phi[NS - 1] = b[NS - 1] / (A[NS - 1][NS - 1] + Num<double>::stab());
#pragma unroll
    for (int i = NS - 2; i >= 0; --i) {
        double term = 0.0;
#pragma unroll
        for (int j = i + 1; j < NS; ++j) term += A[i][j] * phi[j];
        phi[i] = (b[i] - term) / (A[i][i] + Num<double>::stab());
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        if (fabs(phi[k]) < 2.220446049250313e-16) phi[k] = 0;
        out[k] = phi[k] * M[k] * c[k];
    }
}

__device__ __forceinline__ int cellAxisCoords(const StepParams& P, long long i, int D, int* ijk) {
    ijk[0] = (int)(i % P.n[0]);
    ijk[1] = D >= 2 ? (int)((i / P.n[0]) % P.n[1]) : 0;
    ijk[2] = D >= 3 ? (int)(i / ((long long)P.n[0] * P.n[1])) : 0;
    return 0;
}

// minimum over the CTA (all threads pass a value; +inf pads the missing warps); valid in thread 0
__device__ __forceinline__ double blockMinReduce(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nw ? red[lane] : 1.0 / 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// ----------------------------------------------------------------------------- k_diff_prim
template <int NS, int EOS, int D>
__global__ void k_diff_prim(const StepParams P, const DiffParams X, const double* __restrict__ U,
                            DevClock* __restrict__ ck) {
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long st = P.stride;
    double c[NS + 1], v[3], p, rho0, rho[NS + 1], m[3], E;
    cellPrimitive<double, NS, EOS, D>(P, U, nullptr, i, c, v, p, rho0, rho, m, E);
    double v2 = 0;
    v2 += v[0] * v[0];
    v2 += v[1] * v[1];
    v2 += v[2] * v[2];
    const double Uv = E - rho0 * v2 * 0.5 - 0.0;
    const double T = Mixture<double, NS, EOS>::TFromUv(P.mix, c, Uv);
    double w[NS], sum = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        w[k] = rho[k + 1] / rho0;
        sum += w[k];
    }
    double* cp = X.cellPrim;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        cp[k * st + i] = c[k + 1];
        cp[(NS + 5 + k) * st + i] = w[k] / sum;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) cp[(NS + d) * st + i] = v[d];
    cp[(NS + 3) * st + i] = p;
    cp[(NS + 4) * st + i] = T;
}

// ----------------------------------------------------------------------------- k_diff_faces
template <int NS, int EOS, int D>
__global__ void k_diff_faces(const StepParams P, const GenericLayout L, const DiffParams X, DevClock* __restrict__ ck) {
    if (ck->done) return;
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= L.nfaces) return;
    int a = 0;
    while (a + 1 < D && f >= L.faceBase[a + 1]) ++a;
    const long long local = f - L.faceBase[a];
    const int n = P.n[a];
    const int fi = (int)(local % (n + 1));
    if (P.periodic[a] && fi == 0) return;  // unused slot
    const long long tr = local / (n + 1);
    int ijk[3];
    if (a == 0) { ijk[1] = D >= 2 ? (int)(tr % P.n[1]) : 0; ijk[2] = D >= 3 ? (int)(tr / P.n[1]) : 0; }
    else if (a == 1) { ijk[0] = (int)(tr % P.n[0]); ijk[2] = D >= 3 ? (int)(tr / P.n[0]) : 0; }
    else { ijk[0] = (int)(tr % P.n[0]); ijk[1] = (int)(tr / P.n[0]); }
    const bool boundary = !P.periodic[a] && (fi == 0 || fi == n);
    // owner: the cell below the face, or the patch's cell
    ijk[a] = fi == 0 ? 0 : fi - 1;
    const int hi = (boundary && fi == 0) ? 0 : 1;
    const FaceGeo g = faceOf(P, L, ijk, a, hi);
    const long long o = cellIndex(P, ijk[0], ijk[1], ijk[2]);
    const long long st = P.stride, nf = L.nfaces;
    const double* cp = X.cellPrim;
    bool bad = false;

    auto prim = [&](int q, long long j) { return cp[q * st + j]; };
    double cO[NS + 1], vO[3];
    cO[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        cO[k] = prim(k - 1, o);
        cO[0] += cO[k];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) vO[d] = prim(NS + d, o);
    const double pO = prim(NS + 3, o), TO = prim(NS + 4, o);
    const double rO[3] = {P.geo.cc[0][ijk[0]], P.geo.cc[1][ijk[1]], P.geo.cc[2][ijk[2]]};

    // geometry of the gradient: inner d = r_N - r_O and |d|; patch dR = 2 (r_f - r_O), |dR|, dR / |dR|
    long long nb = -1;
    double dA = 0, m2 = 0, dmag = 0, dnA = 0, wOwn = 0, wNei = 0;
    double dir[3];  // d (inner) or dR / |dR| (patch): the gradient's direction
    double cN[NS + 1], vN[3], pN = 0, TN = 0;
    if (!boundary) {
        int nbc[3];
        double sh;
        neighbourOf(P, ijk, a, 1, nbc, sh);
        nb = cellIndex(P, nbc[0], nbc[1], nbc[2]);
        double dv[3], dOwn[3], dNei[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double cnb = P.geo.cc[d][nbc[d]];
            const double neiP = d == a ? cnb + sh : cnb;
            dv[d] = neiP - rO[d];
            dOwn[d] = g.rc[d] - rO[d];
            dNei[d] = g.rc[d] - neiP;
        }
        const double mg = mag3<double>(dv[0], dv[1], dv[2]);
        m2 = mg * mg;
        dA = dv[a];
#pragma unroll
        for (int d = 0; d < 3; ++d) dir[d] = dv[d];
        const double ownR = mag3<double>(dOwn[0], dOwn[1], dOwn[2]);
        const double neiR = mag3<double>(dNei[0], dNei[1], dNei[2]);
        const double sumR = ownR + neiR;
        wOwn = neiR / sumR;
        wNei = ownR / sumR;
        cN[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            cN[k] = prim(k - 1, nb);
            cN[0] += cN[k];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) vN[d] = prim(NS + d, nb);
        pN = prim(NS + 3, nb);
        TN = prim(NS + 4, nb);
    } else {
        double dR[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) dR[d] = (g.rc[d] - rO[d]) * 2.;
        dmag = mag3<double>(dR[0], dR[1], dR[2]);
#pragma unroll
        for (int d = 0; d < 3; ++d) dir[d] = dR[d] / dmag;
        dnA = dir[a];
    }
    (void)pN;
    // axis component of surfGrad (gradient.hpp:96-168) given the owner value and the
    // neighbour's (inner) or the ghost's (patch)
    auto sgrad = [&](double phiO, double other) {
        if (!boundary) {
            const double q = (other - phiO) / m2;
            return q * dA;
        }
        const double q = (other - phiO) / dmag;
        return q * dnA;
    };

    // interpolated concentrations, density and temperature (linearInterpolate.hpp:43-80)
    double sc[NS + 1], sRho = 0.0;
    sc[0] = 0.0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        sc[k] = boundary ? surfaceScalar<double, NS>(P, g.patch, k - 1, cO[k]) : cO[k] * wOwn + cN[k] * wNei;
        sc[0] += sc[k];
        sRho += sc[k] * P.mix.M[k - 1];
    }
    const double sT = boundary ? boundaryT<NS, EOS>(P, g.patch, cO, pO, false, bad) : TO * wOwn + TN * wNei;

    // the patch's concentrations as cell values (ghosts of the calculated* fields)
    double cB[NS + 1];
    if (boundary) {
        cB[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            cB[k] = cellGhostScalar<double, NS>(P, g.patch, k - 1, cO[k], bad);
            cB[0] += cB[k];
        }
    }

    // the face's transport coefficients: its interpolated temperature and concentrations and the
    // Riemann star pressure (Diffusion.cpp:238-240)
    double muF, kappaF, DmF[NS][NS], DsF[NS];
    pointMuKappa<NS>(X, P.mix.M, sT, sc, muF, kappaF);
    pointDm<NS>(X, P.mix.M, sT, X.starP[f], DmF);
    faceDs<NS>(X, sc, DmF, DsF);
    double* F = X.face;
    double flowW[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        // mass fraction k: calculatedMassFraction ghost (boundaryConditionValue.hpp:346-361)
        const double wO = prim(NS + 5 + k, o);
        double other;
        if (boundary) {
            const double dens = cB[k + 1] * P.mix.M[k];
            double sum = 0;
#pragma unroll
            for (int q = 1; q <= NS; ++q) sum += cB[q] * P.mix.M[q - 1];
            other = dens / sum;
        } else {
            other = prim(NS + 5 + k, nb);
        }
        const double gW = sgrad(wO, other);
        const double rhoD = sRho * DsF[k];  // effectiveTransportCoefficients::rhoD (:228-230)
        flowW[k] = gW * (-1 * rhoD);
        F[slotW<NS>(k) * nf + f] = flowW[k];
    }
    double corr[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) corr[k] = 0;
    if (X.molmass) {
        double gX[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            // molar fraction k: calculatedMolarFraction ghost (boundaryConditionValue.hpp:362-377)
            const double xO = cO[k + 1] / cO[0];
            double other;
            if (boundary) {
                double sum = 0;
#pragma unroll
                for (int q = 1; q <= NS; ++q) sum += cB[q];
                other = cB[k + 1] / sum;
            } else {
                other = cN[k + 1] / cN[0];
            }
            gX[k] = sgrad(xO, other);
        }
        double DF[NS];
        if (NS > 1) {
            maxwellStefan<NS>(sc, P.mix.M, DmF, gX, DF);
        } else {
#pragma unroll
            for (int k = 0; k < NS; ++k) DF[k] = 0;
        }
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            corr[k] = DF[k] - flowW[k];
            F[slotCorr<NS>(k) * nf + f] = corr[k];
        }
    }
    if (X.enthalpy) {
        double ent = 0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const double h = hkT<EOS>(P.mix, sc[k + 1], sT, k);
            ent = ent + (corr[k] + flowW[k]) * h / P.mix.M[k];
        }
        // the implicit solver averages the flow with the one of the new concentrations before the
        // product with T (Diffusion.cpp:618-690)
        F[slotEnt<NS>() * nf + f] = X.gs ? ent : ent * sT;
    }
    // velocity: surfGrad column a (dv_i / |d|^2) d_a, surfDivergence, the Laplacian flow and the
    // deviatoric stress (gradient transposed, 2/3 div off the diagonal) of the face
    double vOther[3];
    if (boundary) {
        if (P.bc.vel[g.patch] == FV_BC_FIXED_SURFACE) bad = true;
        ghostVelocity<double>(P.bc.vel[g.patch], P.bc.vel_value[g.patch], a, g.sign, vO, vOther);
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) vOther[d] = vN[d];
    }
    // q = dv / |d|^2 (inner) or dv / |dR| (patch); the face tensor is q dir (outer product)
    double qv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        qv[d] = (vOther[d] - vO[d]) / (boundary ? dmag : m2);
        // row d of (grad_s v mu (-1)) & n: column a
        F[slotV<NS>(d) * nf + f] = qv[d] * dir[a] * muF * -1.;
    }
    double divVs = 0;  // q & dir
    divVs += qv[0] * dir[0];
    divVs += qv[1] * dir[1];
    divVs += qv[2] * dir[2];
    const double lam = (2. / 3.) * divVs;
    // row d of ((grad_s v)^T - 2/3 div I) mu & n: element [d][a] = q_a dir_d (minus 2/3 div on
    // the diagonal); on a patch whose centre is off the cell's axis line dir has transverse parts
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double e = qv[a] * dir[d];
        if (d == a) e -= lam;
        F[slotDev<NS>(d) * nf + f] = e * muF;
    }
    // temperature: calculatedTemperature ghost
    const double Tother = boundary ? boundaryT<NS, EOS>(P, g.patch, cO, pO, true, bad) : TN;
    F[slotT<NS>() * nf + f] = sgrad(TO, Tother) * kappaF * -1.;
    if (X.dtDiff) {
        // effectiveTransportCoefficients::maxValue (transportCoefficients.hpp:172-184)
        double Dmax = DsF[0];
#pragma unroll
        for (int k = 1; k < NS; ++k) Dmax = smax(Dmax, DsF[k]);
        F[slotMax<NS>() * nf + f] = smax(smax(kappaF, sRho * Dmax), muF);
    }
    if (X.gs) {
        F[slotRho<NS>() * nf + f] = sRho;
        F[slotTs<NS>() * nf + f] = sT;
        F[slotMu<NS>() * nf + f] = muF;
        F[slotKappa<NS>() * nf + f] = kappaF;
#pragma unroll
        for (int k = 0; k < NS; ++k) F[slotDs<NS>(k) * nf + f] = DsF[k];
    }
    if (X.interpV) {
        // star.v = linearInterpolate(velocity) (secondOrderStepSolver.cpp:71-73, or the
        // "linear" reconstruction's grad(velocity), Diffusion.cpp:178-184)
        double sv[3];
        if (boundary) {
            surfaceVelocity<double>(P, g.patch, a, g.sign, vO, sv);
        } else {
#pragma unroll
            for (int d = 0; d < 3; ++d) sv[d] = vO[d] * wOwn + vN[d] * wNei;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) X.starV[d * nf + f] = sv[d];
    }
    if (bad) raise(ck, FV_ERR_BOUNDARY);
}

// ----------------------------------------------------------------------------- k_diff_cells
template <int NS, int EOS, int D>
__global__ void k_diff_cells(const StepParams P, const GenericLayout L, const DiffParams X, double* __restrict__ U,
                             DevClock* __restrict__ ck, double* __restrict__ blockMax) {
    __shared__ double red[32];
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double localMax = -1, minE = 1.0 / 0.0, minD = 1.0 / 0.0;
    if (i < P.ncell) {
        const long long st = P.stride, nf = L.nfaces;
        const double dt = ck->dt;
        int ijk[3];
        cellAxisCoords(P, i, D, ijk);
        const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
        const double V = ex * ey * ez;
        const double minLS = 1.0 / smin(smin(ex, ey), ez);
        const double rc[3] = {P.geo.cc[0][ijk[0]], P.geo.cc[1][ijk[1]], P.geo.cc[2][ijk[2]]};
        constexpr int NFC = 2 * D;
        int fa[NFC], fh[NFC];
        {
            int q = 0;
            fa[q] = 0; fh[q++] = 0;
            fa[q] = 0; fh[q++] = 1;
            if (D >= 2) { fa[q] = 1; fh[q++] = 1; fa[q] = 1; fh[q++] = 0; }
            if (D >= 3) { fa[q] = 2; fh[q++] = 0; fa[q] = 2; fh[q++] = 1; }
        }
        const double* F = X.face;
        // divergences: sum over the cell's faces of (F_a n_a) S, then / V
        double divW[NS], divC[NS], divE = 0, divFV[3] = {0, 0, 0}, divDev[3] = {0, 0, 0}, divT = 0;
        double gradV[9], divV = 0;  // Gauss gradient and divergence of the star velocities
        double dist[NFC], sumDist = 0, maxv[NFC];
#pragma unroll
        for (int k = 0; k < NS; ++k) divW[k] = divC[k] = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) gradV[q] = 0;
#pragma unroll
        for (int s = 0; s < NFC; ++s) {
            const FaceGeo g = faceOf(P, L, ijk, fa[s], fh[s]);
            const int a = fa[s];
            const double nsg = g.own ? double(g.sign) : double(-g.sign);
            const double S = g.S;
            const long long f = g.f;
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                divW[k] += F[slotW<NS>(k) * nf + f] * nsg * S;
                if (X.molmass) divC[k] += F[slotCorr<NS>(k) * nf + f] * nsg * S;
            }
            if (X.enthalpy && !X.enthImplicit) divE += F[slotEnt<NS>() * nf + f] * nsg * S;
#pragma unroll
            for (int d = 0; d < 3; ++d) divFV[d] += F[slotV<NS>(d) * nf + f] * nsg * S;
#pragma unroll
            for (int d = 0; d < 3; ++d) divDev[d] += F[slotDev<NS>(d) * nf + f] * nsg * S;
            divT += F[slotT<NS>() * nf + f] * nsg * S;
            // (starV * n) S: column a of the tensor; (starV & n) S
            double sv[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) sv[d] = X.starV[d * nf + f];
#pragma unroll
            for (int d = 0; d < 3; ++d) gradV[3 * d + a] += sv[d] * nsg * S;
            divV += sv[a] * nsg * S;
            if (X.dtDiff) {
                // distance |r_f - r_C| (mesh.cpp:88-112); across a periodic wrap face the face
                // sits one period further along the axis for the neighbour-side cell
                double dr[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double fc = g.rc[d];
                    if (d == a && !g.own && !g.boundary && ijk[a] == 0) fc -= P.ext[a];
                    dr[d] = fc - rc[d];
                }
                dist[s] = mag3<double>(dr[0], dr[1], dr[2]);
                sumDist += dist[s];
                maxv[s] = F[slotMax<NS>() * nf + f];
            }
        }
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            divW[k] /= V;
            divC[k] /= V;
        }
        divE /= V;
        divT /= V;
        divV /= V;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            divFV[d] /= V;
            divDev[d] /= V;
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) gradV[q] /= V;

        const double* cp = X.cellPrim;
        double c[NS + 1], v[3];
        c[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            c[k] = cp[(k - 1) * st + i];
            c[0] += c[k];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = cp[(NS + d) * st + i];
        const double T = cp[(NS + 4) * st + i];
        const double rho0 = U[NS * st + i];

        // mass fractions (Diffusion.cpp:321-339,396-412,430-460)
        double cNew[NS + 1];
        {
            double wNew[NS], sum = 0.;
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                const double w = cp[(NS + 5 + k) * st + i];
                double diag = rho0, freeW = 0.0 - divW[k];
                const double oldW = w * rho0;
                if (X.molmass) {
                    const double s = divC[k] * (-1.0);
                    if (s >= 0.) freeW += s;
                    else diag -= s / (w + Num<double>::stab());
                }
                double x = (oldW + freeW * dt) / diag;
                if (x < 0.) x = 0.0;
                wNew[k] = x;
                sum += x;
            }
            cNew[0] = 0;
#pragma unroll
            for (int k = 1; k <= NS; ++k) {
                cNew[k] = wNew[k - 1] / sum * rho0 / P.mix.M[k - 1];
                cNew[0] += cNew[k];
            }
        }
        const double CCVOld = c[0] * mixCv<NS, EOS>(P.mix, c);
        const double CCVNew = mixCv<NS, EOS>(P.mix, cNew) * cNew[0];
        const double oldEnergy = CCVOld * T + nonIdeality<NS, EOS>(P.mix, c) - nonIdeality<NS, EOS>(P.mix, cNew);
        // velocity (Diffusion.cpp:480-489,600-605,787-797)
        double freeV[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            freeV[d] = 0.0 - divFV[d];
            freeV[d] += divDev[d];
        }
        // temperature (Diffusion.cpp:491-500,688-709,818-825)
        double freeT = 0.0 - divT, diagT = CCVNew;
        if (X.enthalpy && !X.enthImplicit) {
            minE = CCVOld * T / fabs(divE + Num<double>::stab());
            const double s = divE * -1;
            if (s >= 0.) freeT += s;
            else diagT -= s / (T + Num<double>::stab());
        }
        {
            // devPhysVisc && gradV with devPhysVisc = (gradV + gradV^T - 2/3 div I) mu, mu the
            // cell's (Diffusion.cpp:130-132,506)
            double muC, kappaC;
            pointMuKappa<NS>(X, P.mix.M, T, c, muC, kappaC);
            const double l = (2. / 3.) * divV;
            double dd = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    double sv = gradV[3 * q + r] + gradV[3 * r + q];
                    if (r == q) sv -= l;
                    dd += sv * muC * gradV[3 * r + q];
                }
            freeT += dd;
        }
        double vNew[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) vNew[d] = (rho0 * v[d] + freeV[d] * dt) / rho0;
        // (with the implicit enthalpy flow this solver's temperature is the factory's second
        // solver's, a noMatrixSolver: it stays, Diffusion.cpp:820-826)
        const double Tn = X.enthImplicit ? T : (oldEnergy + freeT * dt) / diagT;
        if (Tn < 0.) raise(ck, FV_ERR_NEGATIVE_T);
        // the recomputed phase (Diffusion.cpp:965-1025)
        const double Uv = UvcFromT<NS, EOS>(P.mix, cNew, Tn) * cNew[0];
        const double p = Mixture<double, NS, EOS>::pFromUv(P.mix, cNew, Uv);
        double v2 = 0;
        v2 += vNew[0] * vNew[0];
        v2 += vNew[1] * vNew[1];
        v2 += vNew[2] * vNew[2];
#pragma unroll
        for (int k = 1; k <= NS; ++k) U[(k - 1) * st + i] = cNew[k] * P.mix.M[k - 1];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d < P.nmom) U[(NS + 1 + d) * st + i] = vNew[d] * rho0;
        U[(NS + 4) * st + i] = Uv + rho0 * v2 * 0.5 + 0.0;
        double* sp = X.stagePrim;
#pragma unroll
        for (int k = 1; k <= NS; ++k) sp[(k - 1) * st + i] = cNew[k];
#pragma unroll
        for (int d = 0; d < 3; ++d) sp[(NS + d) * st + i] = vNew[d];
        sp[(NS + 3) * st + i] = p;
        sp[(NS + 4) * st + i] = Uv;
        sp[(NS + 5) * st + i] = Tn;
        // main's CFL signal of the phase (Schemi.cpp:807-823)
        const double sonic = sqrt(Mixture<double, NS, EOS>::sqSonic(Mixture<double, NS, EOS>::coef(P.mix, cNew), cNew,
                                                                     rho0, Uv, p));
        localMax = (mag3<double>(vNew[0], vNew[1], vNew[2]) + sonic) * minLS;
        if (X.dtDiff) {
            // linearInterpolate of the faces' maximal coefficient to the cell (linearInterpolate.hpp:18-38)
            double vol = 0;
#pragma unroll
            for (int s = 0; s < NFC; ++s) vol += maxv[s] * (1 - dist[s] / sumDist);
            minD = vol * minLS * minLS;
        }
    }
    const double bm = blockMaxReduce<double>(localMax, red);
    __syncthreads();
    const double bE = blockMinReduce(minE, red);
    __syncthreads();
    const double bD = blockMinReduce(minD, red);
    if (threadIdx.x == 0) {
        blockMax[blockIdx.x] = bm;
        X.partMin[blockIdx.x] = bE;
        X.partMin[gridDim.x + blockIdx.x] = bD;
    }
    if (i == 0) ck->stagePrim = 1;
}

// the stage's source time step: the explicit enthalpy limit replaces it, the diffusion limit
// bounds it (Diffusion.cpp:688-700, 1036-1049)
__global__ void k_diff_source(const DiffParams X, DevClock* __restrict__ ck, int nblocks) {
    __shared__ double red[32];
    if (ck->done) return;
    double mE = 1.0 / 0.0, mD = 1.0 / 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        mE = smin(mE, X.partMin[b]);
        mD = smin(mD, X.partMin[nblocks + b]);
    }
    mE = blockMinReduce(mE, red);
    __syncthreads();
    mD = blockMinReduce(mD, red);
    if (threadIdx.x != 0) return;
    double src = sourceTimestep(ck);
    if (X.enthalpy && !X.enthImplicit) src = X.coeffSource * mE;
    if (X.dtDiff) src = smin(src, 0.5 * X.coeffDiff / mD);
    ck->dtSource = src;
}

}  // namespace diff
}  // namespace fv
