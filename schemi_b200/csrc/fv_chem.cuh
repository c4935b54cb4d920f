// fv_chem.cuh -- per-cell chemistry source on the device, FP64: the integrator of
// abstractChemicalKinetics (headers/abstractChemicalKinetics.hpp:25-620) with the Cl2 mechanism
// (src/chemicalReactions/chemicalKineticsChlorumDissociation.cpp:47-353) and the A+B->2C
// mechanism (no counterpart in the reference; same integrator, heat release in the form of
// chemicalKineticsH2Cl2Combustion.cpp:362-389), followed by bunchOfFields::average
// (templates/bunchOfFields.hpp:166-204).  Runs after the advection step with the same dt, one
// thread per cell, and writes the CFL block maxima of the resulting state.
//
// Every expression keeps the reference's operation order; results differ from the CPU only
// through the last bit of exp() and pow().  Sub-cycling (the step divided by 10 after a failed
// solve, a lost mass fraction or a negative temperature) is per cell; the reference's serial loop
// carries the finer sub-step on to the cells that follow the failing one.  A cell that would need
// more than kChemMaxSubsteps sub-steps raises systemError (the reference goes on dividing down to
// the minimal time step).
#pragma once

#include "fv_chem_launch.h"
#include "fv_generic.cuh"

namespace fv {
namespace chem {

constexpr double kTol = 100 * 1E-12;      // convergenceTolerance
constexpr double kMassFracTol = 1E-2;     // massFracTolerance
constexpr double kEps = 2.220446049250313e-16;  // numeric_limits<double>::epsilon()
constexpr long long kChemMaxSubsteps = 10000;

__device__ __forceinline__ double stab() { return 5 * kEps; }  // globalConstants.hpp stabilizator

// Sparse system of one cell: diagonal, left (j < i) and right (j > i) entries in list order.
template <int N>
struct System {
    double D[N];
    double A[N][N];
    double B[N];
};

// Entry patterns of the mechanisms: Cl2 (N = 2): right of row 0 = {1}, left of row 1 = {0};
// A+B->2C (N = 3): left of row 2 = {0, 1}.
template <int N> __device__ __forceinline__ int nLeft(int i) {
    if constexpr (N == 2) return i == 1 ? 1 : 0;
    return i == 2 ? 2 : 0;
}
template <int N> __device__ __forceinline__ int nRight(int i) {
    if constexpr (N == 2) return i == 0 ? 1 : 0;
    return 0;
}
template <int N> __device__ __forceinline__ int left(int, int q) { return N == 2 ? 0 : q; }
template <int N> __device__ __forceinline__ int right(int, int) { return 1; }

template <int N>
__device__ __forceinline__ void normalize(double* x) {
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (fabs(x[i]) < kEps) x[i] = 0;
}

// The solvers' convergence test 100 max_i d_i < kTol, d_i = |new_i - old_i| / (|new_i| + stab)
// (the first component's d taken as it is, later ones when larger).  It holds exactly when no
// component has 100 d_i >= kTol (the rounded product is monotone in d), a NaN d_0 failing it and a
// NaN elsewhere passed over.  Each d_i = a / b is compared without the division where the quotient
// is far from the threshold: fl(a 1e14) < b bounds a / b below 1e-14 (1 + eps), so 100 d_i stays
// below 1e-12 (1 + eps)^3 < kTol; fl(b 1e-9) < a bounds it above 1e-9 (1 - eps), so 100 d_i
// exceeds 1e-7 (1 - eps)^2 > kTol (b >= stab, so b 1e-9 does not underflow).  In between, and
// for NaN operands, the quotient is formed as in the reference.
template <int N>
__device__ __forceinline__ bool converged(const double* nw, const double* old) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const double a = fabs(nw[i] - old[i]), b = fabs(nw[i]) + stab();
        bool fails;
        if (a * 1e14 < b) {
            fails = false;
        } else if (a > b * 1e-9) {
            fails = true;
        } else {
            const double d = a / b;
            fails = i == 0 ? !(100. * d < kTol) : (100. * d >= kTol);
        }
        ok = ok && !fails;
    }
    return ok;
}

template <int N>
__device__ __forceinline__ void dot(const System<N>& m, const double* v, double* out) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double s = m.D[i] * v[i];
#pragma unroll
        for (int q = 0; q < nLeft<N>(i); ++q) s += m.A[i][left<N>(i, q)] * v[left<N>(i, q)];
#pragma unroll
        for (int q = 0; q < nRight<N>(i); ++q) s += m.A[i][right<N>(i, q)] * v[right<N>(i, q)];
        out[i] = s;
    }
}

// solveGS (abstractChemicalKinetics.hpp:201-306); 1 / D[i] is the same value in every iteration
template <int N>
__device__ bool solveGS(const System<N>& m, const double* init, int maxIter, double* out) {
    double old[N], nw[N], aii[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        old[i] = nw[i] = init[i];
        aii[i] = 1. / m.D[i];
    }
    for (int it = 1;; ++it) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            nw[i] = m.B[i] * aii[i];
#pragma unroll
            for (int q = 0; q < nLeft<N>(i); ++q) nw[i] -= m.A[i][left<N>(i, q)] * nw[left<N>(i, q)] * aii[i];
#pragma unroll
            for (int q = 0; q < nRight<N>(i); ++q) nw[i] -= m.A[i][right<N>(i, q)] * old[right<N>(i, q)] * aii[i];
        }
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            nw[i] = m.B[i] * aii[i];
#pragma unroll
            for (int q = nLeft<N>(i) - 1; q >= 0; --q) nw[i] -= m.A[i][left<N>(i, q)] * old[left<N>(i, q)] * aii[i];
#pragma unroll
            for (int q = nRight<N>(i) - 1; q >= 0; --q) nw[i] -= m.A[i][right<N>(i, q)] * nw[right<N>(i, q)] * aii[i];
        }
        if (converged<N>(nw, old)) {
            normalize<N>(nw);
#pragma unroll
            for (int i = 0; i < N; ++i) out[i] = nw[i];
            return true;
        }
        if (it >= maxIter) return false;
#pragma unroll
        for (int i = 0; i < N; ++i) old[i] = nw[i];
    }
}

// solveJ (:110-199)
template <int N>
__device__ bool solveJ(const System<N>& m, const double* init, int maxIter, double* out) {
    double old[N], nw[N], aii[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        old[i] = nw[i] = init[i];
        aii[i] = 1. / m.D[i];
    }
    for (int it = 1;; ++it) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double rs = 0;
#pragma unroll
            for (int q = 0; q < nLeft<N>(i); ++q) rs -= m.A[i][left<N>(i, q)] * old[left<N>(i, q)];
#pragma unroll
            for (int q = 0; q < nRight<N>(i); ++q) rs -= m.A[i][right<N>(i, q)] * old[right<N>(i, q)];
            nw[i] = (m.B[i] + rs) * aii[i];
        }
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            double rs = 0;
#pragma unroll
            for (int q = nLeft<N>(i) - 1; q >= 0; --q) rs -= m.A[i][left<N>(i, q)] * old[left<N>(i, q)];
#pragma unroll
            for (int q = nRight<N>(i) - 1; q >= 0; --q) rs -= m.A[i][right<N>(i, q)] * old[right<N>(i, q)];
            nw[i] = (m.B[i] + rs) * aii[i];
        }
        if (converged<N>(nw, old)) {
            normalize<N>(nw);
#pragma unroll
            for (int i = 0; i < N; ++i) out[i] = nw[i];
            return true;
        }
        if (it >= maxIter) return false;
#pragma unroll
        for (int i = 0; i < N; ++i) old[i] = nw[i];
    }
}

template <int N>
__device__ __forceinline__ double sum(const double* a) {
    double s = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) s += a[i];
    return s;
}

// solveCG (:308-389) / solveJCG (:391-495)
template <int N>
__device__ bool solveCG(const System<N>& m, const double* init, int maxIter, bool jacobi, double* out) {
    double x[N], r[N], d[N], Ad[N], P[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        x[i] = init[i];
        P[i] = 1. / m.D[i];
    }
    dot<N>(m, x, Ad);
#pragma unroll
    for (int i = 0; i < N; ++i) r[i] = m.B[i] - Ad[i];
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = jacobi ? P[i] * r[i] : r[i];
    for (int it = 1;; ++it) {
        double diff = 0;
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i == 0 || fabs(r[i]) > diff) diff = fabs(r[i]);
        if (diff < kTol && it > 1) {
            normalize<N>(x);
#pragma unroll
            for (int i = 0; i < N; ++i) out[i] = x[i];
            return true;
        }
        if (it >= maxIter) return false;
        double t[N];
        dot<N>(m, d, Ad);
#pragma unroll
        for (int i = 0; i < N; ++i) t[i] = jacobi ? r[i] * (P[i] * r[i]) : r[i] * r[i];
        const double rr = sum<N>(t);
#pragma unroll
        for (int i = 0; i < N; ++i) t[i] = d[i] * Ad[i];
        const double alpha = rr / (sum<N>(t) + stab());
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] += alpha * d[i];
        double r1[N];
#pragma unroll
        for (int i = 0; i < N; ++i) r1[i] = r[i] - alpha * Ad[i];
#pragma unroll
        for (int i = 0; i < N; ++i) t[i] = jacobi ? r1[i] * (P[i] * r1[i]) : r1[i] * r1[i];
        const double beta = sum<N>(t) / (rr + stab());
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = (jacobi ? P[i] * r1[i] : r1[i]) + beta * d[i];
#pragma unroll
        for (int i = 0; i < N; ++i) r[i] = r1[i];
    }
}

// solveGE (:497-604): row pivoting on the raw value, elimination, back substitution
template <int N>
__device__ bool solveGE(const System<N>& m, double* out) {
    double A[N][N], b[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
#pragma unroll
        for (int j = 0; j < N; ++j) A[i][j] = 0;
        A[i][i] = m.D[i];
#pragma unroll
        for (int q = 0; q < nLeft<N>(i); ++q) A[i][left<N>(i, q)] = m.A[i][left<N>(i, q)];
#pragma unroll
        for (int q = 0; q < nRight<N>(i); ++q) A[i][right<N>(i, q)] = m.A[i][right<N>(i, q)];
        b[i] = m.B[i];
    }
#pragma unroll
    for (int k = 0; k < N - 1; ++k) {
        double mv = A[k][k];
        int c = k;
#pragma unroll
        for (int q = k + 1; q < N; ++q)
            if (A[q][k] > mv) { mv = A[q][k]; c = q; }
        // row swap by value selects (no dynamic register indexing)
#pragma unroll
        for (int q = k + 1; q < N; ++q) {
            if (q != c) continue;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                const double t = A[q][j];
                A[q][j] = A[k][j];
                A[k][j] = t;
            }
            const double t = b[q];
            b[q] = b[k];
            b[k] = t;
        }
    }
#pragma unroll
    for (int k = 0; k < N - 1; ++k)
#pragma unroll
        for (int i = k + 1; i < N; ++i) {
            const double ratio = A[i][k] / (A[k][k] + stab());
#pragma unroll
            for (int j = k + 1; j < N; ++j) A[i][j] = A[i][j] - ratio * A[k][j];
            b[i] = b[i] - ratio * b[k];
        }
    double phi[N];
    phi[N - 1] = b[N - 1] / (A[N - 1][N - 1] + stab());
#pragma unroll
    for (int i = N - 2; i >= 0; --i) {
        double term = 0.0;
#pragma unroll
        for (int j = i + 1; j < N; ++j) term += A[i][j] * phi[j];
        phi[i] = (b[i] - term) / (A[i][i] + stab());
    }
    normalize<N>(phi);
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = phi[i];
    return true;
}

template <int N>
__device__ __forceinline__ bool solve(const ChemParams& C, const System<N>& m, const double* init, double* out) {
    switch (C.solver) {
    case FV_CHEM_JACOBI: return solveJ<N>(m, init, C.maxIter, out);
    case FV_CHEM_GAUSS_ELIMINATION: return solveGE<N>(m, out);
    case FV_CHEM_CONJUGATE_GRADIENT: return solveCG<N>(m, init, C.maxIter, false, out);
    case FV_CHEM_JACOBI_CONJUGATE_GRADIENT: return solveCG<N>(m, init, C.maxIter, true, out);
    default: return solveGS<N>(m, init, C.maxIter, out);
    }
}

// k = A T^n exp(-E / (R T))
__device__ __forceinline__ double arrhenius(double A, double n, double E, double T, double R) {
    const double Tn = n == 0.0 ? 1.0 : pow(T, n);  // pow(T, 0) is exactly 1
    return A * Tn * exp(-E / (R * T));
}

// Mechanism matrix of one sub-step (species order of fvstep.h).
template <int N>
__device__ __forceinline__ void system(const ChemParams& C, const MixParams& mx, double dt, double T, const double* c,
                                       double rho, System<N>& m) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) m.A[i][j] = 0;
    if constexpr (N == 2) {
        // setMatrix (chemicalKineticsChlorumDissociation.cpp:47-70)
        const double kd = arrhenius(C.Af, C.nf, C.Ef, T, mx.R), kr = arrhenius(C.Ab, C.nb, C.Eb, T, mx.R);
        const double Cl2 = c[1], Cl = c[2], M0 = c[0];
        m.D[0] = (1 / dt + kd * M0) / mx.M[0];
        m.A[0][1] = (-kr * Cl * M0) / mx.M[1];
        m.B[0] = Cl2 / (rho * dt);
        m.A[1][0] = (-2 * kd * M0) / mx.M[0];
        m.D[1] = (1 / dt + 2 * kr * Cl * M0) / mx.M[1];
        m.B[1] = Cl / (rho * dt);
    } else {
        // A + B -> 2C with rate k c_B^old c_A^new (A), k c_A^old c_B^new (B); C from the mass of both
        const double k = arrhenius(C.Af, C.nf, C.Ef, T, mx.R);
        const double cA = c[1], cB = c[2], cC = c[3];
        m.D[0] = (1 / dt + k * cB) / mx.M[0];
        m.B[0] = cA / (rho * dt);
        m.D[1] = (1 / dt + k * cA) / mx.M[1];
        m.B[1] = cB / (rho * dt);
        m.A[2][0] = (-k * cB) / mx.M[2];
        m.A[2][1] = (-k * cA) / mx.M[2];
        m.D[2] = (1 / dt) / mx.M[2];
        m.B[2] = cC / (rho * dt);
    }
}

// TFromUv with the mixture heat capacity of the mole fractions (mixtureIdeal.cpp,
// mixtureVanDerWaals.cpp, idealFluid.cpp:37-41, vanDerWaalsFluid.cpp:44-48).
template <int N, int EOS>
__device__ __forceinline__ double TFromUv(const MixParams& mx, const double* c, double Uv) {
    double X[N];
#pragma unroll
    for (int k = 0; k < N; ++k) X[k] = c[k + 1] / c[0];
    double Cvm = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) Cvm += X[k] * mx.Cv[k];
    if (EOS == FV_EOS_IDEAL) return Uv / ((c[0] + stab()) * Cvm);
    double am = 0;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int l = 0; l < N; ++l) am += X[k] * X[l] * mx.a[k][l];
    return (Uv + am * (c[0] * c[0])) / ((c[0] + stab()) * Cvm);
}

template <int N>
struct Cell {
    double Uv, T;
    double c[N + 1];
    double dens[N];
};

// timeStepIntegration of one cell (chemicalKineticsChlorumDissociation.cpp:152-273).
template <int N, int EOS>
__device__ int integrate(const ChemParams& C, const MixParams& mx, double dt, double minDt, double rho,
                         Cell<N>& cell) {
    const Cell<N> oldV = cell;
    const double Tcell = oldV.T;
    long long subIt = 1;
    double subDt = dt / subIt;
    Cell<N> nv = oldV;
    while (true) {
        bool ok = true;
        nv = oldV;
        for (long long st = 0; st < subIt && ok; ++st) {
            double wOld[N];
#pragma unroll
            for (int k = 0; k < N; ++k) wOld[k] = nv.dens[k] / rho;
            double sumOld = 0.;
#pragma unroll
            for (int k = 0; k < N; ++k) sumOld = sumOld + wOld[k];
            if (sumOld == 0.0) continue;
            System<N> m;
            system<N>(C, mx, subDt, Tcell, nv.c, rho, m);
            double w[N];
            if (!solve<N>(C, m, wOld, w)) { ok = false; break; }
#pragma unroll
            for (int k = 0; k < N; ++k) w[k] = fmax(0., w[k]);
            double sumNew = 0.;
#pragma unroll
            for (int k = 0; k < N; ++k) sumNew = sumNew + w[k];
            if (fabs(sumNew - sumOld) > kMassFracTol) { ok = false; break; }
#pragma unroll
            for (int k = 0; k < N; ++k) {
                w[k] /= sumNew;
                w[k] *= sumOld;
            }
            double deltaU = 0;
            if constexpr (N == 3) {
                // A+B->2C: heat release per mol of C formed, (q - dCv (T - 298.15)) / 2
                const double deltaC = w[2] * rho / mx.M[2] - nv.c[3];
                const double deltaCv = 2 * mx.Cv[2] - mx.Cv[0] - mx.Cv[1];
                deltaU = (C.q - deltaCv * (Tcell - 298.15)) * 0.5 * deltaC;
            }
#pragma unroll
            for (int k = 0; k < N; ++k) nv.c[k + 1] = w[k] * rho / mx.M[k];
            nv.c[0] = 0;
#pragma unroll
            for (int k = 1; k <= N; ++k) nv.c[0] += nv.c[k];
            nv.Uv += deltaU;
            nv.T = TFromUv<N, EOS>(mx, nv.c, nv.Uv);
            if (nv.T < 0) { ok = false; break; }
#pragma unroll
            for (int k = 0; k < N; ++k) nv.dens[k] = nv.c[k + 1] * mx.M[k];
        }
        if (ok) break;
        subIt *= 10;
        subDt = dt / subIt;
        if (subDt < minDt || subIt > kChemMaxSubsteps) return FV_ERR_SYSTEM;
    }
    cell = nv;
    return FV_OK;
}

// Chemistry of every cell of U (in place) with the step's dt, then the CFL signal of the result.
// The register budget is sized for two CTAs of 256 threads per SM (the FP64 arithmetic is
// latency-bound; the spills this costs stay in L1).
// CONC: the state keeps its concentrations (C.conc, after a multi-stage average); a separate
// instantiation so that the single-stage pass carries no extra registers.
template <int N, int EOS, int D, bool CONC>
__global__ void __launch_bounds__(256, 2) k_chemistry(const StepParams P, const ChemParams C, double* __restrict__ U,
                                                   DevClock* __restrict__ ck, double* __restrict__ blockMax) {
    __shared__ double red[32];
    if (ck->done) return;  // uniform over the grid
    const double dt = ck->dt;
    const long long st = P.stride;
    const MixParams& mx = P.mix;
    double localMax = -1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        double rhoS[N], m[3];
#pragma unroll
        for (int k = 0; k < N; ++k) rhoS[k] = U[k * st + i];
        const double rho = U[N * st + i];
#pragma unroll
        for (int d = 0; d < 3; ++d) m[d] = d < P.nmom ? U[(N + 1 + d) * st + i] : 0.0;
        double E = U[(N + 4) * st + i];
        // derived fields after the advection (Advection.cpp:455-479), or the concentrations the
        // multi-stage average left (bunchOfFields::average)
        Cell<N> q;
        double cIn[CONC ? N + 1 : 1];
        if constexpr (CONC) {
#pragma unroll
            for (int k = 0; k <= N; ++k) q.c[k] = C.conc[k * st + i];
#pragma unroll
            for (int k = 0; k <= N; ++k) cIn[k] = q.c[k];
        } else if (C.stage) {
            q.c[0] = 0;
#pragma unroll
            for (int k = 1; k <= N; ++k) {
                q.c[k] = C.stage[(k - 1) * st + i];
                q.c[0] += q.c[k];
            }
        } else {
            q.c[0] = 0;
#pragma unroll
            for (int k = 1; k <= N; ++k) {
                q.c[k] = rhoS[k - 1] / mx.M[k - 1];
                q.c[0] += q.c[k];
            }
        }
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = C.stage ? C.stage[(N + d) * st + i] : m[d] / rho;
        double v2 = 0;
        v2 += v[0] * v[0];
        v2 += v[1] * v[1];
        v2 += v[2] * v[2];
        if (C.stage) {
            // the stage's internal energy and temperature (Diffusion.cpp:965-1025)
            q.Uv = C.stage[(N + 4) * st + i];
            q.T = C.stage[(N + 5) * st + i];
        } else {
            q.Uv = E - rho * v2 * 0.5 - 0.0;
            q.T = TFromUv<N, EOS>(mx, q.c, q.Uv);
        }
#pragma unroll
        for (int k = 0; k < N; ++k) q.dens[k] = rhoS[k];
        int status = integrate<N, EOS>(C, mx, dt, P.min_dt, rho, q);
        if (status == FV_OK) status = integrate<N, EOS>(C, mx, dt, P.min_dt, rho, q);
        if (status != FV_OK) {
            raise(ck, status);
        } else {
            // E of the integrated phase, then the 0.5 average with the advected phase
            const double E1 = q.Uv + rho * v2 * 0.5 + 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                rhoS[k] = 0.5 * rhoS[k] + 0.5 * q.dens[k];
                U[k * st + i] = rhoS[k];
            }
            E = 0.5 * E + 0.5 * E1;
            U[(N + 4) * st + i] = E;
            if constexpr (CONC) {
#pragma unroll
                for (int k = 0; k <= N; ++k) {
                    cIn[k] = 0.5 * cIn[k] + 0.5 * q.c[k];
                    C.conc[k * st + i] = cIn[k];
                }
            }
        }
        // CFL signal of the new state
        int ijk[3];
        ijk[0] = (int)(i % P.n[0]);
        ijk[1] = D >= 2 ? (int)((i / P.n[0]) % P.n[1]) : 0;
        ijk[2] = D >= 3 ? (int)(i / ((long long)P.n[0] * P.n[1])) : 0;
        const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
        const double minLS = 1.0 / smin(smin(ex, ey), ez);
        if constexpr (CONC) {
            // the state's own (averaged) concentrations, as main's CFL block reads them
            localMax = smax(localMax, cellSignalC<double, N, EOS, D>(P, cIn, rho, m, E, minLS));
        } else {
            double rr[N + 1];
            rr[0] = rho;
#pragma unroll
            for (int k = 1; k <= N; ++k) rr[k] = rhoS[k - 1];
            localMax = smax(localMax, cellSignal<double, N, EOS, D>(P, rr, rho, m, E, minLS));
        }
    }
    const double bm = blockMaxReduce<double>(localMax, red);
    if (threadIdx.x == 0) blockMax[blockIdx.x] = bm;
    // the averaged phase is the state's (bunchOfFields::average recomputes p and T from it): the
    // next step and the download derive the primitives from the state again (nothing in this
    // kernel reads the flag)
    if (C.stage && blockIdx.x == 0 && threadIdx.x == 0) ck->stagePrim = 0;
}

}  // namespace chem
}  // namespace fv
