/*
 * fv_oracle.cpp -- TEST INFRASTRUCTURE: FP64 CPU restatement of Schemi's explicit
 * finite-volume step, used only as the checker of the CUDA path (parity tests, smoke
 * check, CPU baseline of the bench).  Never linked into the product.
 *
 * It restates, on a structured parallelepiped, the algorithm of the reference (paths are
 * inside the Schemi project):
 *   mesh geometry          src/dataStructures/mesh.cpp:34-86 (normals, weights), :296-500 (1D),
 *                          :522-1200 (2D), :1205-1900 (3D)
 *   Gauss gradient         templates/gradient.hpp:19-58, linear interpolation
 *                          templates/linearInterpolate.hpp:43-80
 *   TVD limiter (r-ratio)  src/limiters/TVDLimiter.cpp:12-125 (vector), :127-272 (tensor)
 *   limiter functions      src/limiters/<name>Limiter.cpp (xiR = 2/(1+r) forms)
 *   reconstruction+closure src/Advections/Advection.cpp:114-387
 *   Hancock predictor      src/Advections/HancockStage.cpp:10-448, headers/HancockStage.hpp:22-95
 *   HLLC / HLL fluxes      src/RiemannSolvers/HLLCSolver.cpp:13-406, HLLSolver.cpp:13-318
 *   update                 src/Advections/Advection.cpp:414-505, templates/divergence.hpp:61-96
 *   CFL block + time loop  main/Schemi.cpp:641-670, 767-940
 *   EOS                    src/thermodynamics/mixtureIdeal.cpp, idealFluid.cpp:13-60,
 *                          mixtureVanDerWaals.cpp:19-58,88-146,309-397, vanDerWaalsFluid.cpp:14-75
 *   boundary values        headers/boundaryConditionValue.hpp:34-515, src/boundary/slipFunction.cpp
 *   chemistry              headers/abstractChemicalKinetics.hpp:25-620,
 *                          src/chemicalReactions/chemicalKineticsChlorumDissociation.cpp:47-353,
 *                          chemicalKineticsH2Cl2Combustion.cpp:362-389, templates/bunchOfFields.hpp:166-204
 * The operation order of every floating-point expression follows the reference so that the
 * restatement reproduces the reference binary to round-off.  Periodic patches and the
 * A+B->2C chemistry have no reference counterpart; they follow the same conventions.
 * Compiled with -ffp-contract=off (the reference build has no FMA).
 */
#include "fv_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace {

constexpr double kStab = 5 * std::numeric_limits<double>::epsilon(); // globalConstants.hpp:33
constexpr double kTwoThirds = 2. / 3.;
constexpr double kPi = 3.14159265358979323846;  // Pi_number (globalConstants.hpp:38-40): the double nearest pi
constexpr double kVeryBig = 1E-3 * std::numeric_limits<double>::max(); // globalConstants.hpp:35

struct V3 {
    double x[3];
};
struct T9 {
    double x[9];
};

inline V3 v3(double a, double b, double c) { return V3{{a, b, c}}; }
inline V3 vadd(const V3& a, const V3& b) { return v3(b.x[0] + a.x[0], b.x[1] + a.x[1], b.x[2] + a.x[2]); }
inline V3 vsub(const V3& a, const V3& b) { return v3(a.x[0] - b.x[0], a.x[1] - b.x[1], a.x[2] - b.x[2]); }
inline V3 vmul(const V3& a, double s) { return v3(a.x[0] * s, a.x[1] * s, a.x[2] * s); }
inline V3 vdiv(const V3& a, double s) { return v3(a.x[0] / s, a.x[1] / s, a.x[2] / s); }
// vector::operator& (vector.cpp:109-119): ((0 + a0 b0) + a1 b1) + a2 b2
inline double vdot(const V3& a, const V3& b) {
    double r = 0;
    r += a.x[0] * b.x[0];
    r += a.x[1] * b.x[1];
    r += a.x[2] * b.x[2];
    return r;
}
inline V3 vcross(const V3& a, const V3& b) {
    return v3(a.x[1] * b.x[2] - a.x[2] * b.x[1], -(a.x[0] * b.x[2] - a.x[2] * b.x[0]),
              a.x[0] * b.x[1] - a.x[1] * b.x[0]);
}
// Scaled 3-argument hypot with the semantics of the reference build's std::hypot(x, y, z):
// a = the largest magnitude, result a * sqrt((x/a)^2 + (y/a)^2 + (z/a)^2).
inline double mag3(const V3& v) {
    double x = std::fabs(v.x[0]), y = std::fabs(v.x[1]), z = std::fabs(v.x[2]);
    double a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == 0) return 0;
    return a * std::sqrt((x / a) * (x / a) + (y / a) * (y / a) + (z / a) * (z / a));
}
// vector * vector (vector.cpp:94-107): T[3i+j] = a_i b_j
inline T9 outer(const V3& a, const V3& b) {
    T9 t;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t.x[3 * i + j] = a.x[i] * b.x[j];
    return t;
}
// tensor & vector (tensor.cpp:163-176)
inline V3 tdot(const T9& t, const V3& v) {
    return v3(t.x[0] * v.x[0] + t.x[1] * v.x[1] + t.x[2] * v.x[2],
              t.x[3] * v.x[0] + t.x[4] * v.x[1] + t.x[5] * v.x[2],
              t.x[6] * v.x[0] + t.x[7] * v.x[1] + t.x[8] * v.x[2]);
}
inline T9 tmul(const T9& t, double s) {
    T9 r;
    for (int i = 0; i < 9; ++i) r.x[i] = t.x[i] * s;
    return r;
}

// ------------------------------------------------------------------ limiter functions
// phi(r, xiR) with xiR = 2 / (1 + r), src/limiters/<name>Limiter.cpp (the "calculate" forms).
double limiterPhi(int lim, double r, double xiR) {
    switch (lim) {
    case FV_LIM_ZERO: return 0;  // zeroLimiter.cpp returns a zero gradient
    case FV_LIM_MINMOD:          // minmodLimiter.cpp:14-27
        if (r <= 0.) return 0;
        if (r <= 1.) return r;
        return std::min(1.0, xiR);
    case FV_LIM_VANLEER:         // vanLeerLimiter.cpp:14-25
        if (r < 0.) return 0;
        return std::min(2 * r / (1 + r), xiR);
    case FV_LIM_LINEAR: return 1;  // linearLimiter.cpp returns the gradient unchanged
    case FV_LIM_VANALBADA:       // vanAlbadaLimiter.cpp:15-28
        if (r <= 0.) return 0;
        return std::min((r * r + r) / (1 + r * r), xiR);
    case FV_LIM_HQUICK:
        if (r <= 0.) return 0;
        return std::min(4 * r / (3 + r), xiR);
    case FV_LIM_VANLEER2: {
        if (r <= 0.) return 0;
        const double denom = 1 + r;
        return std::min(4 * r / (denom * denom), 2 * xiR);
    }
    case FV_LIM_SUPERBEE:        // superbeeLimiter.cpp:14-29
        if (r <= 0.) return 0;
        if (r <= 0.5) return 2 * r;
        if (r <= 1.) return r;
        return std::min({r, 2.0, xiR});
    case FV_LIM_VANALBADA2:
        if (r <= 0.) return 0;
        return std::min(2 * r / (1 + r * r), 2 * xiR);
    case FV_LIM_MINMOD2:
        if (r <= 0.) return 0;
        return std::min({1.0, 4 * r / (1 + r), 2 * xiR});
    case FV_LIM_SWEBY: {
        const double b = 2.0;  // SwebyLimiter.hpp:17
        if (r <= 0.) return 0;
        return std::min({std::min(1.0, b * r), std::min(b, r), b * xiR});
    }
    case FV_LIM_KOREN:
        if (r <= 0) return 0;
        return std::min(std::min({2 * r, (1 + 2 * r) / 3, 2.0}), 2 * xiR);
    case FV_LIM_KOREN2:
        if (r <= 0) return std::min(0.0, std::max(-kTwoThirds, (1 + 2 * r) / 3));
        return std::min({2 * kTwoThirds * r, std::min((1 + 2 * r) / 3, 2.0), 2 * xiR});
    case FV_LIM_UTCDFS:
        if (r < -1) return r * (r + 1) / (r * r + 1);
        if ((r >= -1) && (r < 0)) return 0;
        if ((r >= 0) && (r < 0.5)) return r * r * r - 2 * (r * r) + 2 * r;
        if ((r >= 0.5) && (r < 2)) return 0.75 * r + 0.25;
        return std::min((2 * (r * r) - 2 * r - 9.0 / 4.0) / (r * r - r - 1), 2 * xiR);
    case FV_LIM_SCHMIDTMANN: {
        const double alpha = 1, beta = 2, gamma = 1.5;  // SchmidtmannLimiter.hpp:17
        const double phiO3 = (2 + r) / 3;
        return std::min(std::max(0.0, std::min(phiO3, std::max(-alpha * r, std::min({beta * r, phiO3, gamma})))),
                        2 * xiR);
    }
    }
    return 0;
}

// ------------------------------------------------------------------ geometry
struct Face {
    V3 rC, N;
    double S;
    int own, nei;      // nei = -1 on a boundary patch
    int patch;         // fv_patch of a boundary face, -1 inner, or patch of the wrapped face (periodic)
    V3 neiShift;       // translation applied to the neighbour centre across a periodic patch
    double wOwn, wNei;
};

struct Cell {
    V3 rC;
    double V;
    double minLS;      // 1 / min edge (Schemi.cpp:648-662)
    int faces[6];
    int nFaces;
    int nb[6];         // neighbour cells (mesh.cpp "Set environment cells" order)
    V3 nbShift[6];
    int nNb;
};

// ------------------------------------------------------------------ real-gas fluids
// The cubic of RedlichKwongFluid.cpp in the reference's long-double solver
// (cubicEquationSolver.cpp:15-113: trigonometric / hyperbolic roots, coefficients divided in
// double first) and the choice of its single positive root (returnSinglePosValue, :115-152).
constexpr double kZeroLevel = kStab;         // globalConstants.hpp zeroLevel
constexpr double kOneThird = 1. / 3., kTwoThirdsC = 2. / 3.;
const double kPiD = std::acos(-1.0);

int signOf(double v) {  // sign.cpp
    if (v > kZeroLevel) return 1;
    if (v < -kZeroLevel) return -1;
    return 0;
}

struct Roots {
    double x[3];
    bool ok;
};

Roots cubicRoots(double A, double B, double C, double D) {
    typedef long double L;
    constexpr double crit = 1E-9;
    Roots r{{std::nan("1"), std::nan("2"), std::nan("3")}, true};
    if ((A > crit) || (A < -crit)) {
        const L a{B / A}, b{C / A}, c{D / A};
        const L Q{(a * a - 3 * b) / 9};
        const L R{(a * (2 * (a * a) - 9 * b) + 27 * c) / 54};
        const L S{(Q * Q) * Q - R * R};
        if (S >= kZeroLevel) {
            const L phi{kOneThird * std::acos(R / std::sqrt(Q * Q * Q))};
            r.x[0] = -2. * std::sqrt(Q) * std::cos(phi) - a * kOneThird;
            r.x[1] = -2. * std::sqrt(Q) * std::cos(phi - kTwoThirdsC * kPiD) - a * kOneThird;
            r.x[2] = -2. * std::sqrt(Q) * std::cos(phi + kTwoThirdsC * kPiD) - a * kOneThird;
        } else if ((S < kZeroLevel) && (S >= -kZeroLevel)) {
            r.x[0] = -2. * signOf((double)R) * std::sqrt(Q) - a * kOneThird;
            r.x[1] = signOf((double)R) * std::sqrt(Q) - a * kOneThird;
            r.x[2] = r.x[1];
        } else if (S < -kZeroLevel) {
            if (Q >= kZeroLevel) {
                const L phi{kOneThird * std::acosh(std::abs(R) / (std::sqrt((Q * Q) * Q) + kStab))};
                r.x[0] = -2. * signOf((double)R) * std::sqrt(Q) * std::cosh(phi) - a * kOneThird;
            } else if ((Q < kZeroLevel) && (Q >= -kZeroLevel)) {
                r.x[0] = -std::cbrt(c - (a * a) * a / 27) - a * kOneThird;
            } else if (Q < -kZeroLevel) {
                const L phi{kOneThird * std::asinh(std::abs(R) / (std::sqrt(std::abs((Q * Q) * Q)) + kStab))};
                r.x[0] = -2. * signOf((double)R) * std::sqrt(std::abs(Q)) * std::sinh(phi) - a * kOneThird;
            } else {
                r.ok = false;  // "Q has unknown value"
            }
        } else {
            r.ok = false;  // "S has unknown value"
        }
    } else {
        const L a{B}, b{C}, c{D};
        const auto Discr = b * b - 4 * a * c;
        if (Discr >= 0) {
            const auto a2 = 0.5 / (a + kStab);
            r.x[0] = a2 * (-b + std::sqrt(Discr));
            r.x[1] = a2 * (-b - std::sqrt(Discr));
        }
    }
    return r;
}

// returnSinglePosValue; `ok` false where the reference throws (positivnessError)
double singlePositive(Roots r, bool& ok) {
    int nPositive = 0;
    for (double& v : r.x) {
        if (v >= 0) nPositive++;
        else v = -123.;
    }
    ok = r.ok;
    if (nPositive == 1) return std::max(std::max(r.x[0], r.x[1]), r.x[2]);
    if (nPositive == 2) {
        if (((r.x[0] - r.x[1]) < kZeroLevel) && (r.x[2] < 0)) return r.x[0];
        if (((r.x[1] - r.x[2]) < kZeroLevel) && (r.x[0] < 0)) return r.x[1];
        if (((r.x[0] - r.x[2]) < kZeroLevel) && (r.x[1] < 0)) return r.x[2];
    } else if (nPositive == 3 && ((r.x[0] - r.x[1]) < kZeroLevel) && ((r.x[1] - r.x[2]) < kZeroLevel)) {
        return r.x[0];
    }
    ok = false;
    return std::nan("");
}

// KataokaVanDerWaalsFluid.cpp: the cluster series with M = 13 terms (its header's constant); the
// loops written there as "for (J = 2; M < J; ++J)" run no iteration and leave their sums at zero,
// which the derivatives below keep.
constexpr double kKataokaM = 13;

double kqa(double c, double T, double V0, double eps, double R) {
    const double V0c{V0 * c};
    const double epsRT{0.5 * eps / (R * T)};
    double series{1.0};
    for (std::size_t J = 2; J <= kKataokaM; ++J) series += std::pow(V0c, (J - 1.) / 3.) * std::exp((J - 1.) * epsRT);
    return series;
}
double kUvA(double c, double T, double V0, double eps, double R) {
    const double V0c{V0 * c};
    const double epsRT{0.5 * eps / (R * T)};
    double series{0};
    for (std::size_t J = 2; J <= kKataokaM; ++J)
        series -= (J - 1.) * std::pow(V0c, (J - 1.) / 3.) * std::exp((J - 1.) * epsRT);
    return 0.5 * c * eps * series / kqa(c, T, V0, eps, R);
}
double kpA(double c, double T, double V0, double eps, double R) {
    const double V0c{V0 * c};
    const double epsRT{0.5 * eps / (R * T)};
    double series{0};
    for (std::size_t J = 2; J <= kKataokaM; ++J)
        series -= (J - 1.) / 3. * std::pow(V0c, (J - 1.) / 3.) * std::exp((J - 1.) * epsRT);
    return c * R * T * series / kqa(c, T, V0, eps, R);
}
// the never-running series of the derivatives: 0
double kEmpty() {
    double series{0};
    for (std::size_t J = 2; kKataokaM < J; ++J) series += 1;
    return series;
}
double kdPdC(double c, double T, double V0, double eps, double R, double b) {
    const double V0c{V0 * c};
    const double n13 = kEmpty();
    const double qa1 = kqa(c, T, V0, eps, R);
    return R * T / (1 - c * b) + c * R * T * b / ((1 - c * b) * (1 - c * b)) +
           (R * T * n13 + V0c * R * T * (kEmpty() - n13 * kEmpty() / qa1)) / qa1;
}
double kdPdT(double c, double T, double V0, double eps, double R, double b) {
    const double n13 = kEmpty();
    const double qa1 = kqa(c, T, V0, eps, R);
    return c * R / (1 - c * b) + (c * R * n13 + 0.5 * c * eps / T * (kEmpty() - n13 * kEmpty() / qa1)) / qa1;
}
double kdUvdC(double c, double Cv, double T, double V0, double eps, double R) {
    const double V0c{V0 * c};
    const double n13 = kEmpty();
    const double qa1 = kqa(c, T, V0, eps, R);
    return Cv * T + (0.5 * eps * n13 + 0.5 * V0c * eps * (kEmpty() - n13 * kEmpty() / qa1)) / qa1;
}
double kdUvdT(double c, double Cv, double T, double V0, double eps, double R) {
    const double qa1 = kqa(c, T, V0, eps, R);
    const double s2 = kEmpty();
    return c * Cv + 0.25 * c * (eps * eps) / (R * (T * T)) * kEmpty() / qa1 -
           0.25 * c * (eps * eps) / (R * (T * T)) * (s2 * s2) / (qa1 * qa1);
}
// NewtonMethod.cpp:13-40 (tolerance convergenceToleranceGlobal = 1e-12, at most 100 iterations)
template <class F, class DF>
double newton(double start, F f, DF df) {
    std::size_t it{1};
    double x1{start};
    double x2 = x1 - f(x1) / df(x1);
    if (std::abs(x2 - x1) <= 1E-12) return x2;
    while ((std::abs(x2 - x1) > 1E-12) && (it <= 100)) {
        x1 = x2;
        x2 = x1 - f(x1) / df(x1);
        it++;
    }
    return x2;
}
// T of a Kataoka state from its internal energy per volume (pFromUv, TFromUv, dpdrho, dpdUv)
double kTFromUv(double c, double Cv, double Uv, double V0, double eps, double R) {
    auto f = [&](double T) { return c * Cv * T + kUvA(c, T, V0, eps, R) - Uv; };
    auto df = [&](double T) { return kdUvdT(c, Cv, T, V0, eps, R); };
    const double initT{Uv / ((c + kStab) * Cv)};
    return newton(initT, f, df);
}

struct Mix {
    int N;
    int eos;
    double R;
    double M[FV_MAX_SPECIES], Cv[FV_MAX_SPECIES];
    // pair matrices: van der Waals / Redlich-Kwong a and b, stiffened p0 and gamma, Kataoka V0,
    // eps and b
    double a[FV_MAX_SPECIES][FV_MAX_SPECIES], b[FV_MAX_SPECIES][FV_MAX_SPECIES];
    double p0[FV_MAX_SPECIES][FV_MAX_SPECIES], gam[FV_MAX_SPECIES][FV_MAX_SPECIES];
    double V0[FV_MAX_SPECIES][FV_MAX_SPECIES], eps[FV_MAX_SPECIES][FV_MAX_SPECIES];
    mutable bool failed = false;  // a cubic without a single positive root (positivnessError)

    // calcMolarFrac (fractionCalculation.cpp:36-44) and the mixture sums
    void mixParams(const double* c, double& CvMix, double& aMix, double& bMix, double& MMix) const {
        double X[FV_MAX_SPECIES];
        for (int k = 0; k < N; ++k) X[k] = c[k + 1] / c[0];
        CvMix = 0;
        MMix = 0;
        for (int k = 0; k < N; ++k) {
            CvMix += X[k] * Cv[k];
            MMix += X[k] * M[k];
        }
        aMix = 0;
        bMix = 0;
        if (eos == FV_EOS_VAN_DER_WAALS || eos == FV_EOS_REDLICH_KWONG)
            for (int k = 0; k < N; ++k)
                for (int l = 0; l < N; ++l) {
                    aMix += X[k] * X[l] * a[k][l];
                    bMix += X[k] * X[l] * b[k][l];
                }
    }
    // stiffened: p0 and gamma of the mixture (mixtureStiffened.cpp:73-97)
    void stiffParams(const double* c, double& p0m, double& gm) const {
        double X[FV_MAX_SPECIES];
        for (int k = 0; k < N; ++k) X[k] = c[k + 1] / c[0];
        p0m = 0;
        gm = 0;
        for (int k = 0; k < N; ++k)
            for (int l = 0; l < N; ++l) {
                p0m += X[k] * X[l] * p0[k][l];
                gm += X[k] * X[l] * gam[k][l];
            }
    }
    // Kataoka: V0, eps and b of the mixture (mixtureKataokaVanDerWaals.cpp:116-137)
    void kataokaParams(const double* c, double& V0m, double& em, double& bm) const {
        double X[FV_MAX_SPECIES];
        for (int k = 0; k < N; ++k) X[k] = c[k + 1] / c[0];
        V0m = 0;
        em = 0;
        bm = 0;
        for (int k = 0; k < N; ++k)
            for (int l = 0; l < N; ++l) {
                V0m += X[k] * X[l] * V0[k][l];
                em += X[k] * X[l] * eps[k][l];
                bm += X[k] * X[l] * b[k][l];
            }
    }
    // sqrt(T) of a Redlich-Kwong state from Uv (RedlichKwongFluid.cpp:46-56, 96-102)
    double rkSqrtT(double c, double Cvm, double Uv, double am, double bm) const {
        bool ok;
        const double r = singlePositive(cubicRoots(c * Cvm, 0, -Uv, -1.5 * am * c / bm * std::log1p(c * bm)), ok);
        if (!ok) failed = true;
        return r;
    }
    double pFromUv(const double* c, double Uv) const {
        double Cvm, am, bm, Mm;
        mixParams(c, Cvm, am, bm, Mm);
        if (eos == FV_EOS_STIFFENED) {  // stiffenedFluid.cpp:13-17
            double p0m, gm;
            stiffParams(c, p0m, gm);
            return (gm - 1.0) * Uv - p0m * gm;
        }
        if (eos == FV_EOS_REDLICH_KWONG) {  // RedlichKwongFluid.cpp:46-56
            const double sT = rkSqrtT(c[0], Cvm, Uv, am, bm);
            return c[0] * R * (sT * sT) / (1 - c[0] * bm) - am * (c[0] * c[0]) / (sT * (1 + c[0] * bm));
        }
        if (eos == FV_EOS_KATAOKA) {  // KataokaVanDerWaalsFluid.cpp:237-256
            double V0m, em, bk;
            kataokaParams(c, V0m, em, bk);
            const double T = kTFromUv(c[0], Cvm, Uv, V0m, em, R);
            return c[0] * R * T / (1 - c[0] * bk) + kpA(c[0], T, V0m, em, R);
        }
        const double g1 = R / Cvm;
        if (eos == FV_EOS_IDEAL) return g1 * Uv;  // idealFluid.cpp:13-17
        const double acc = am * (c[0] * c[0]);   // vanDerWaalsFluid.cpp:14-21
        return g1 * (Uv + acc) / (1 - c[0] * bm) - acc;
    }
    double UvFromp(const double* c, double p) const {
        double Cvm, am, bm, Mm;
        mixParams(c, Cvm, am, bm, Mm);
        if (eos == FV_EOS_STIFFENED) {  // stiffenedFluid.cpp:19-23
            double p0m, gm;
            stiffParams(c, p0m, gm);
            return (p + p0m * gm) / (gm - 1.0);
        }
        if (eos == FV_EOS_REDLICH_KWONG) {  // RedlichKwongFluid.cpp:58-68
            const double cc = c[0];
            bool ok;
            const double sT = singlePositive(
                cubicRoots(cc * R, 0, -p * (1 - cc * bm), -am * (cc * cc) * (1 - cc * bm) / (1 + cc * bm)), ok);
            if (!ok) failed = true;
            return cc * Cvm * (sT * sT) - 1.5 * am * cc / (bm * sT) * std::log1p(cc * bm);
        }
        if (eos == FV_EOS_KATAOKA) {  // KataokaVanDerWaalsFluid.cpp:258-277
            double V0m, em, bk;
            kataokaParams(c, V0m, em, bk);
            const double cc = c[0];
            auto f = [&](double T) { return cc * R * T / (1 - cc * bk) + kpA(cc, T, V0m, em, R) - p; };
            auto df = [&](double T) { return kdPdT(cc, T, V0m, em, R, bk); };
            const double initT{p / ((cc + kStab) * R)};
            const double T = newton(initT, f, df);
            return cc * Cvm * T + kUvA(cc, T, V0m, em, R);
        }
        const double g1 = R / Cvm;
        if (eos == FV_EOS_IDEAL) return p / g1;  // idealFluid.cpp:19-23
        const double acc = am * (c[0] * c[0]);   // vanDerWaalsFluid.cpp:23-30
        return (p + acc) * (1 - c[0] * bm) / g1 - acc;
    }
    double TFromUv(const double* c, double Uv) const {
        double Cvm, am, bm, Mm;
        mixParams(c, Cvm, am, bm, Mm);
        if (eos == FV_EOS_STIFFENED) {  // stiffenedFluid.cpp:37-41
            double p0m, gm;
            stiffParams(c, p0m, gm);
            return (Uv - p0m) / ((c[0] + kStab) * Cvm);
        }
        if (eos == FV_EOS_REDLICH_KWONG) {  // RedlichKwongFluid.cpp:84-92
            const double sT = rkSqrtT(c[0], Cvm, Uv, am, bm);
            return sT * sT;
        }
        if (eos == FV_EOS_KATAOKA) {
            double V0m, em, bk;
            kataokaParams(c, V0m, em, bk);
            return kTFromUv(c[0], Cvm, Uv, V0m, em, R);
        }
        if (eos == FV_EOS_IDEAL) return Uv / ((c[0] + kStab) * Cvm);  // idealFluid.cpp:37-41
        return (Uv + am * (c[0] * c[0])) / ((c[0] + kStab) * Cvm);    // vanDerWaalsFluid.cpp:44-48
    }
    double dpdUv(const double* c, double Uv) const {
        double Cvm, am, bm, Mm;
        mixParams(c, Cvm, am, bm, Mm);
        if (eos == FV_EOS_STIFFENED) {  // stiffenedFluid.cpp dpdUv: gamma - 1
            double p0m, gm;
            stiffParams(c, p0m, gm);
            return gm - 1.0;
        }
        if (eos == FV_EOS_REDLICH_KWONG) {  // RedlichKwongFluid.cpp:120-131
            const double sT = rkSqrtT(c[0], Cvm, Uv, am, bm);
            const double T = sT * sT;
            return rkdPdT(c[0], T, am, bm) / rkdUvdT(c[0], Cvm, T, am, bm);
        }
        if (eos == FV_EOS_KATAOKA) {  // KataokaVanDerWaalsFluid.cpp:355-372
            double V0m, em, bk;
            kataokaParams(c, V0m, em, bk);
            const double T = kTFromUv(c[0], Cvm, Uv, V0m, em, R);
            return kdPdT(c[0], T, V0m, em, R, bk) / kdUvdT(c[0], Cvm, T, V0m, em, R);
        }
        const double g1 = R / Cvm;
        if (eos == FV_EOS_IDEAL) return g1;
        return g1 / (1 - c[0] * bm);  // vanDerWaalsFluid.cpp:71-75
    }
    // RedlichKwongFluid.cpp:14-44
    double rkdPdC(double c, double T, double am, double bm) const {
        return R * T / (1 - c * bm) + c * R * T * bm / ((1 - c * bm) * (1 - c * bm)) -
               2 * am * c / (std::sqrt(T) * (1 + bm * c)) +
               am * (c * c) * bm / (std::sqrt(T) * ((1 + bm * c) * (1 + bm * c)));
    }
    double rkdPdT(double c, double T, double am, double bm) const {
        const double sT = std::sqrt(T);
        return c * R / (1 - c * bm) + 0.5 * am * (c * c) / (((sT * sT) * sT) * (1 + c * bm));
    }
    double rkdUvdC(double c, double Cvm, double T, double am, double bm) const {
        return Cvm * T - 1.5 * am * std::log1p(c * bm) / (bm * std::sqrt(T)) - 1.5 * am * c / (std::sqrt(T) * (1 + c * bm));
    }
    double rkdUvdT(double c, double Cvm, double T, double am, double bm) const {
        const double sT = std::sqrt(T);
        return c * Cvm + 0.75 * am * c * std::log1p(c * bm) / (bm * ((sT * sT) * sT));
    }
    // sqSonicSpeed = dpdrho + dpdUv * (Uv + p) / rho (mixtureIdeal.cpp, mixtureVanDerWaals.cpp:390-397,
    // mixtureRedlichKwong.cpp:418-425, mixtureStiffened.cpp:327-334, mixtureKataokaVanDerWaals.cpp:445-452)
    double sqSonicSpeed(const double* c, double rho, double Uv, double p) const {
        double Cvm, am, bm, Mm;
        mixParams(c, Cvm, am, bm, Mm);
        if (eos == FV_EOS_STIFFENED) return 0 + dpdUv(c, Uv) * (Uv + p) / rho;
        if (eos == FV_EOS_REDLICH_KWONG) {  // RedlichKwongFluid.cpp:104-118
            const double sT = rkSqrtT(c[0], Cvm, Uv, am, bm);
            const double T = sT * sT;
            const double dpdrho = (rkdPdC(c[0], T, am, bm) -
                                   rkdPdT(c[0], T, am, bm) * rkdUvdC(c[0], Cvm, T, am, bm) / rkdUvdT(c[0], Cvm, T, am, bm)) /
                                  Mm;
            return dpdrho + dpdUv(c, Uv) * (Uv + p) / rho;
        }
        if (eos == FV_EOS_KATAOKA) {  // KataokaVanDerWaalsFluid.cpp:332-353
            double V0m, em, bk;
            kataokaParams(c, V0m, em, bk);
            const double T = kTFromUv(c[0], Cvm, Uv, V0m, em, R);
            const double dpdrho = (kdPdC(c[0], T, V0m, em, R, bk) -
                                   kdPdT(c[0], T, V0m, em, R, bk) * kdUvdC(c[0], Cvm, T, V0m, em, R) /
                                       kdUvdT(c[0], Cvm, T, V0m, em, R)) /
                                  Mm;
            return dpdrho + dpdUv(c, Uv) * (Uv + p) / rho;
        }
        const double g1 = R / Cvm;
        if (eos == FV_EOS_IDEAL) return 0 + g1 * (Uv + p) / rho;
        const double m_cb = 1 - c[0] * bm;  // vanDerWaalsFluid.cpp:57-69
        const double ac = am * c[0];
        const double dpdrho = (g1 * (2 * ac / m_cb - bm * (Uv + ac * c[0]) / (m_cb * m_cb)) - 2 * ac) / Mm;
        const double dUv = g1 / m_cb;
        return dpdrho + dUv * (Uv + p) / rho;
    }
};

// Face-side state (owner or neighbour side of one face)
struct FState {
    double c[FV_MAX_SPECIES + 1];    // c[0] = total
    double rho[FV_MAX_SPECIES + 1];  // rho[0] = mixture density
    V3 v, m;
    double E, Uv, p;
};

}  // namespace

struct fvo_case {
    fv_config cfg;
    int N, D;
    int n[3];
    long long nCells;
    std::vector<Cell> cells;
    std::vector<Face> faces;
    Mix mix;
    // cell state (homogeneousPhase<cubicCell>)
    std::vector<double> c[FV_MAX_SPECIES + 1], rho[FV_MAX_SPECIES + 1];
    std::vector<V3> v, m;
    std::vector<double> E, Uv, p;
    double time = 0, dt = 0;
    V3 g{};
    // chemistry sub-cycling: carried from cell to cell in cell order like the reference's serial
    // loop (1), or per cell (0)
    int chemCarry = 1;
    std::string err;
    // diffusion stage: the Riemann star velocity of the last advection (starFields::v) and the
    // source time step the stage sets for the next step (mesh::timestepSource, reset by main's
    // CFL block, Schemi.cpp:829-833)
    std::vector<V3> starV;
    std::vector<double> starP;  // the star pressure (starFields::p, HLLCSolver.cpp:400)
    double dtSource = kVeryBig;
    double dtSourceLast = kVeryBig;  // the limit the last CFL block took
    // the temperature a diffusion stage leaves (gasPhase.temperature = the stage's new T,
    // Diffusion.cpp:981, not TFromUv of the recomputed energy); the next advection replaces it
    std::vector<double> Tstate;
    bool Tvalid = false;
};

namespace {

// ---------------------------------------------------------------- boundary values
int bcType(const fvo_case& cs, int field, int k, int patch) {
    // field 0: concentration k, 1: velocity, 2: pressure
    if (field == 0) return cs.cfg.bc_conc[patch][k];
    if (field == 1) return cs.cfg.bc_vel[patch];
    return cs.cfg.bc_p[patch];
}

// boundaryConditionValueSurface for scalars (boundaryConditionValue.hpp:34-66)
double bcSurfaceS(const fvo_case& cs, double in, int field, int k, int patch) {
    const int t = bcType(cs, field, k, patch);
    const double val = field == 0 ? cs.cfg.bc_conc_value[patch][k] : cs.cfg.bc_p_value[patch];
    switch (t) {
    case FV_BC_FREE: return in;
    case FV_BC_SLIP: return in;  // slipFunction(scalar) is the identity
    case FV_BC_FIXED_CELL: return (in + val) * 0.5;
    case FV_BC_FIXED_SURFACE: return val;
    }
    return in;
}
// boundaryConditionValueCell for scalars (boundaryConditionValue.hpp:279-300)
double bcCellS(const fvo_case& cs, double in, int field, int k, int patch, bool& bad) {
    const int t = bcType(cs, field, k, patch);
    const double val = field == 0 ? cs.cfg.bc_conc_value[patch][k] : cs.cfg.bc_p_value[patch];
    switch (t) {
    case FV_BC_FREE: return in;
    case FV_BC_SLIP: return in;
    case FV_BC_FIXED_CELL: return val;
    case FV_BC_FIXED_SURFACE: bad = true; return in;  // the reference throws boundaryConditionError
    }
    return in;
}
// slipFunction(vector): v - (v & n) n  (slipFunction.cpp:21-25)
V3 slipV(const V3& v, const V3& n) { return vsub(v, vmul(n, vdot(v, n))); }

V3 bcSurfaceV(const fvo_case& cs, const V3& in, int patch, const V3& N) {
    const int t = cs.cfg.bc_vel[patch];
    const V3 val = v3(cs.cfg.bc_vel_value[patch][0], cs.cfg.bc_vel_value[patch][1], cs.cfg.bc_vel_value[patch][2]);
    switch (t) {
    case FV_BC_FREE: return in;
    case FV_BC_SLIP: return slipV(in, N);
    case FV_BC_FIXED_CELL: return vmul(vadd(in, val), 0.5);
    case FV_BC_FIXED_SURFACE: return val;
    }
    return in;
}
V3 bcCellV(const fvo_case& cs, const V3& in, int patch, const V3& N, bool& bad) {
    const int t = cs.cfg.bc_vel[patch];
    const V3 val = v3(cs.cfg.bc_vel_value[patch][0], cs.cfg.bc_vel_value[patch][1], cs.cfg.bc_vel_value[patch][2]);
    switch (t) {
    case FV_BC_FREE: return in;
    case FV_BC_SLIP: return vsub(vmul(slipV(in, N), 2), in);  // boundaryConditionValue.hpp:291-294
    case FV_BC_FIXED_CELL: return val;
    case FV_BC_FIXED_SURFACE: bad = true; return in;
    }
    return in;
}

// ---------------------------------------------------------------- geometry builder
struct Quad {
    V3 r00, rX0, r0Y, rXY;
};

void finishFace(Face& f, const Quad& q, const std::vector<Cell>& cells) {
    f.rC = vdiv(vadd(vadd(vadd(q.r00, q.rX0), q.r0Y), q.rXY), 4.);
    f.S = mag3(vsub(q.rX0, q.r00)) * mag3(vsub(q.r0Y, q.r00));
    // mesh.cpp:34-53
    const V3 V1 = vsub(q.rX0, q.r00), V2 = vsub(q.r0Y, q.r00);
    V3 Nn = vcross(V1, V2);
    Nn = vdiv(Nn, mag3(Nn));
    const V3 cs = vsub(f.rC, cells[f.own].rC);
    if (vdot(cs, Nn) < 0.) Nn = vmul(Nn, -1.);
    f.N = Nn;
}

bool buildMesh(fvo_case& cs) {
    const fv_config& cf = cs.cfg;
    const int D = cf.dims;
    const int nx = cf.n[0], ny = D >= 2 ? cf.n[1] : 1, nz = D >= 3 ? cf.n[2] : 1;
    cs.n[0] = nx; cs.n[1] = ny; cs.n[2] = nz;
    cs.nCells = (long long)nx * ny * nz;
    const double Lx = cf.L[0], Ly = cf.L[1], Lz = cf.L[2];
    const double dx = Lx / nx, dy = Ly / ny, dz = Lz / nz;
    auto X = [&](int i) { return 0.0 + dx * (double)(std::size_t)i; };
    auto Y = [&](int j) { return D >= 2 ? 0.0 + dy * (double)(std::size_t)j : (j == 0 ? 0.0 : Ly); };
    auto Z = [&](int k) { return D >= 3 ? 0.0 + dz * (double)(std::size_t)k : (k == 0 ? 0.0 : Lz); };
    auto cellId = [&](int i, int j, int k) { return (int)(i + (long long)nx * (j + (long long)ny * k)); };

    cs.cells.resize(cs.nCells);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                Cell& c = cs.cells[cellId(i, j, k)];
                const double xa = X(i), xb = X(i + 1), ya = Y(j), yb = Y(j + 1), za = Z(k), zb = Z(k + 1);
                const V3 r000 = v3(xa, ya, za), rX00 = v3(xb, ya, za), r0Y0 = v3(xa, yb, za), rXY0 = v3(xb, yb, za);
                const V3 r00Z = v3(xa, ya, zb), rX0Z = v3(xb, ya, zb), r0YZ = v3(xa, yb, zb), rXYZ = v3(xb, yb, zb);
                V3 s = vadd(r000, rX00);
                s = vadd(s, r0Y0); s = vadd(s, rXY0); s = vadd(s, r00Z); s = vadd(s, rX0Z); s = vadd(s, r0YZ); s = vadd(s, rXYZ);
                c.rC = vdiv(s, 8.);
                const double e1 = mag3(vsub(rX00, r000)), e2 = mag3(vsub(r0Y0, r000)), e3 = mag3(vsub(r00Z, r000));
                c.V = e1 * e2 * e3;
                c.minLS = 1. / std::min(std::min(e1, e2), e3);
                c.nFaces = 0;
                c.nNb = 0;
            }

    const bool perX = cf.bc_vel[FV_PATCH_TAIL] == FV_BC_PERIODIC;
    const bool perY = D >= 2 && cf.bc_vel[FV_PATCH_RIGHT] == FV_BC_PERIODIC;
    const bool perZ = D >= 3 && cf.bc_vel[FV_PATCH_BOTTOM] == FV_BC_PERIODIC;

    // Faces.  Per cell the face list follows mesh.cpp: [x-, x+, y+, y-, z-, z+].
    // xFace[i][j][k] for i in [0, nx], yFace[i][j][k] for j in [0, ny], zFace for k in [0, nz].
    std::vector<int> xF((size_t)(nx + 1) * ny * nz), yF, zF;
    if (D >= 2) yF.resize((size_t)nx * (ny + 1) * nz);
    if (D >= 3) zF.resize((size_t)nx * ny * (nz + 1));
    auto xIdx = [&](int i, int j, int k) { return (size_t)i + (size_t)(nx + 1) * (j + (size_t)ny * k); };
    auto yIdx = [&](int i, int j, int k) { return (size_t)i + (size_t)nx * (j + (size_t)(ny + 1) * k); };
    auto zIdx = [&](int i, int j, int k) { return (size_t)i + (size_t)nx * (j + (size_t)ny * k); };

    // x faces
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                Face f{};
                double Xf;
                if (i == 0) Xf = 0.0 + 0.;
                else if (i == nx) Xf = 0.0 + Lx;
                else Xf = X(i);
                Quad q;
                if (D == 1) {
                    q = {v3(Xf, 0., 0.), v3(Xf, 0., Lz), v3(Xf, Ly, 0.), v3(Xf, Ly, Lz)};
                } else if (D == 2) {
                    q = {v3(Xf, Y(j), 0.), v3(Xf, Y(j), Lz), v3(Xf, Y(j + 1), 0.), v3(Xf, Y(j + 1), Lz)};
                } else {
                    q = {v3(Xf, Y(j), Z(k)), v3(Xf, Y(j), Z(k + 1)), v3(Xf, Y(j + 1), Z(k)), v3(Xf, Y(j + 1), Z(k + 1))};
                }
                f.neiShift = v3(0, 0, 0);
                if (i == 0) {
                    if (perX) { xF[xIdx(i, j, k)] = -1; continue; }  // created as the x-max face
                    f.own = cellId(0, j, k); f.nei = -1; f.patch = FV_PATCH_TAIL;
                } else if (i == nx) {
                    if (perX) {
                        f.own = cellId(nx - 1, j, k); f.nei = cellId(0, j, k); f.patch = FV_PATCH_POINT;
                        f.neiShift = v3(Lx, 0, 0);
                    } else {
                        f.own = cellId(nx - 1, j, k); f.nei = -1; f.patch = FV_PATCH_POINT;
                    }
                } else {
                    f.own = cellId(i - 1, j, k); f.nei = cellId(i, j, k); f.patch = -1;
                }
                finishFace(f, q, cs.cells);
                xF[xIdx(i, j, k)] = (int)cs.faces.size();
                cs.faces.push_back(f);
            }
    if (perX)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) xF[xIdx(0, j, k)] = xF[xIdx(nx, j, k)];
    // y faces
    if (D >= 2) {
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    Face f{};
                    f.neiShift = v3(0, 0, 0);
                    Quad q;
                    const double za = D >= 3 ? Z(k) : 0., zb = D >= 3 ? Z(k + 1) : Lz;
                    if (j == 0 || j == ny) {
                        const double Yf = j == 0 ? 0.0 + 0. : 0.0 + Ly;
                        // mesh.cpp:781-860 (right / left patches)
                        q = {v3(X(i), Yf, za), v3(X(i), Yf, zb), v3(X(i + 1), Yf, za), v3(X(i + 1), Yf, zb)};
                    } else {
                        const double Yf = Y(j);
                        // mesh.cpp:689-732 (inner y faces)
                        q = {v3(X(i), Yf, za), v3(X(i + 1), Yf, za), v3(X(i), Yf, zb), v3(X(i + 1), Yf, zb)};
                    }
                    if (j == 0) {
                        if (perY) { yF[yIdx(i, j, k)] = -1; continue; }
                        f.own = cellId(i, 0, k); f.nei = -1; f.patch = FV_PATCH_RIGHT;
                    } else if (j == ny) {
                        if (perY) {
                            f.own = cellId(i, ny - 1, k); f.nei = cellId(i, 0, k); f.patch = FV_PATCH_LEFT;
                            f.neiShift = v3(0, Ly, 0);
                        } else {
                            f.own = cellId(i, ny - 1, k); f.nei = -1; f.patch = FV_PATCH_LEFT;
                        }
                    } else {
                        f.own = cellId(i, j - 1, k); f.nei = cellId(i, j, k); f.patch = -1;
                    }
                    finishFace(f, q, cs.cells);
                    yF[yIdx(i, j, k)] = (int)cs.faces.size();
                    cs.faces.push_back(f);
                }
        if (perY)
            for (int k = 0; k < nz; ++k)
                for (int i = 0; i < nx; ++i) yF[yIdx(i, 0, k)] = yF[yIdx(i, ny, k)];
    }
    // z faces
    if (D >= 3) {
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    Face f{};
                    f.neiShift = v3(0, 0, 0);
                    const double Zf = k == 0 ? 0.0 + 0. : (k == nz ? 0.0 + Lz : Z(k));
                    const Quad q = {v3(X(i), Y(j), Zf), v3(X(i + 1), Y(j), Zf), v3(X(i), Y(j + 1), Zf),
                                    v3(X(i + 1), Y(j + 1), Zf)};
                    if (k == 0) {
                        if (perZ) { zF[zIdx(i, j, k)] = -1; continue; }
                        f.own = cellId(i, j, 0); f.nei = -1; f.patch = FV_PATCH_BOTTOM;
                    } else if (k == nz) {
                        if (perZ) {
                            f.own = cellId(i, j, nz - 1); f.nei = cellId(i, j, 0); f.patch = FV_PATCH_TOP;
                            f.neiShift = v3(0, 0, Lz);
                        } else {
                            f.own = cellId(i, j, nz - 1); f.nei = -1; f.patch = FV_PATCH_TOP;
                        }
                    } else {
                        f.own = cellId(i, j, k - 1); f.nei = cellId(i, j, k); f.patch = -1;
                    }
                    finishFace(f, q, cs.cells);
                    zF[zIdx(i, j, k)] = (int)cs.faces.size();
                    cs.faces.push_back(f);
                }
        if (perZ)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) zF[zIdx(i, j, 0)] = zF[zIdx(i, j, nz)];
    }

    // interpolation weights (mesh.cpp:55-86)
    for (Face& f : cs.faces) {
        if (f.nei >= 0) {
            const double ownR = mag3(vsub(f.rC, cs.cells[f.own].rC));
            const double neiR = mag3(vsub(f.rC, vadd(cs.cells[f.nei].rC, f.neiShift)));
            const double sumR = ownR + neiR;
            f.wOwn = neiR / sumR;
            f.wNei = ownR / sumR;
        } else {
            f.wOwn = 1.0;
            f.wNei = 0.0;
        }
    }

    // per-cell face and neighbour lists
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                Cell& c = cs.cells[cellId(i, j, k)];
                c.faces[c.nFaces++] = xF[xIdx(i, j, k)];
                c.faces[c.nFaces++] = xF[xIdx(i + 1, j, k)];
                if (D >= 2) {
                    c.faces[c.nFaces++] = yF[yIdx(i, j + 1, k)];
                    c.faces[c.nFaces++] = yF[yIdx(i, j, k)];
                }
                if (D >= 3) {
                    c.faces[c.nFaces++] = zF[zIdx(i, j, k)];
                    c.faces[c.nFaces++] = zF[zIdx(i, j, k + 1)];
                }
                // neighbours in order x-, x+, y-, y+, z-, z+ (mesh.cpp "Set environment cells")
                auto addNb = [&](int ii, int jj, int kk, V3 sh) {
                    c.nb[c.nNb] = cellId(ii, jj, kk);
                    c.nbShift[c.nNb] = sh;
                    c.nNb++;
                };
                if (i > 0) addNb(i - 1, j, k, v3(0, 0, 0));
                else if (perX) addNb(nx - 1, j, k, v3(-Lx, 0, 0));
                if (i < nx - 1) addNb(i + 1, j, k, v3(0, 0, 0));
                else if (perX) addNb(0, j, k, v3(Lx, 0, 0));
                if (D >= 2) {
                    if (j > 0) addNb(i, j - 1, k, v3(0, 0, 0));
                    else if (perY) addNb(i, ny - 1, k, v3(0, -Ly, 0));
                    if (j < ny - 1) addNb(i, j + 1, k, v3(0, 0, 0));
                    else if (perY) addNb(i, 0, k, v3(0, Ly, 0));
                }
                if (D >= 3) {
                    if (k > 0) addNb(i, j, k - 1, v3(0, 0, 0));
                    else if (perZ) addNb(i, j, nz - 1, v3(0, 0, -Lz));
                    if (k < nz - 1) addNb(i, j, k + 1, v3(0, 0, 0));
                    else if (perZ) addNb(i, j, 0, v3(0, 0, Lz));
                }
            }
    return true;
}

// ---------------------------------------------------------------- gradients + limiter
// Gauss gradient of a scalar cell field (gradient.hpp:19-58 with linearInterpolate.hpp:43-80)
void gradScalar(const fvo_case& cs, const std::vector<double>& phi, int field, int k, std::vector<V3>& grad) {
    const size_t nf = cs.faces.size();
    std::vector<double> fv(nf);
    for (size_t f = 0; f < nf; ++f) {
        const Face& F = cs.faces[f];
        if (F.nei >= 0) fv[f] = phi[F.own] * F.wOwn + phi[F.nei] * F.wNei;
        else fv[f] = bcSurfaceS(cs, phi[F.own], field, k, F.patch);
    }
    grad.resize(cs.nCells);
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        V3 acc = v3(0, 0, 0);
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            const V3 term = vmul(vmul(n, fv[c.faces[j]]), F.S);
            acc.x[0] += term.x[0]; acc.x[1] += term.x[1]; acc.x[2] += term.x[2];
        }
        grad[i] = vdiv(acc, c.V);
    }
}

void gradVector(const fvo_case& cs, const std::vector<V3>& phi, std::vector<T9>& grad) {
    const size_t nf = cs.faces.size();
    std::vector<V3> fv(nf);
    for (size_t f = 0; f < nf; ++f) {
        const Face& F = cs.faces[f];
        if (F.nei >= 0) fv[f] = vadd(vmul(phi[F.own], F.wOwn), vmul(phi[F.nei], F.wNei));
        else fv[f] = bcSurfaceV(cs, phi[F.own], F.patch, F.N);
    }
    grad.resize(cs.nCells);
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        T9 acc{};
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            const T9 term = tmul(outer(fv[c.faces[j]], n), F.S);
            for (int q = 0; q < 9; ++q) acc.x[q] += term.x[q];
        }
        T9 g;
        for (int q = 0; q < 9; ++q) g.x[q] = acc.x[q] / c.V;
        grad[i] = g;
    }
}

// ---------------------------------------------------------------- ThirdOrder reconstruction
// Limiter functions without the xi bound, as calculateNoRSLimit applies them component by
// component (the <Name>LimiterCalculation(r) overloads of src/limiters/*.cpp); linear returns
// the gradient and zero returns zero (phiNoRSLinear / the caller).
double limiterPhiNoRS(int lim, double r) {
    switch (lim) {
    case FV_LIM_ZERO: return 0;
    case FV_LIM_MINMOD: return r <= 0. ? 0 : (r <= 1. ? r : 1.);
    case FV_LIM_VANLEER: return r < 0. ? 0 : 2 * r / (1 + r);
    case FV_LIM_LINEAR: return 1;
    case FV_LIM_VANALBADA: return r <= 0. ? 0 : (r * r + r) / (1 + r * r);
    case FV_LIM_HQUICK: return r <= 0. ? 0 : 4 * r / (3 + r);
    case FV_LIM_VANLEER2: {
        if (r <= 0.) return 0;
        const double denom = 1 + r;
        return 4 * r / (denom * denom);
    }
    case FV_LIM_SUPERBEE:
        if (r <= 0.) return 0;
        if (r <= 0.5) return 2 * r;
        if (r <= 1.) return r;
        return std::min(r, 2.0);
    case FV_LIM_VANALBADA2: return r <= 0. ? 0 : 2 * r / (1 + r * r);
    case FV_LIM_MINMOD2: return r <= 0. ? 0 : std::min(1.0, 4 * r / (1 + r));
    case FV_LIM_SWEBY: {
        const double b = 2.0;
        return r <= 0. ? 0 : std::min(std::min(1.0, b * r), std::min(b, r));
    }
    case FV_LIM_KOREN: return r <= 0 ? 0 : std::min({2 * r, (1 + 2 * r) / 3, 2.0});
    case FV_LIM_KOREN2:
        if (r <= 0) return std::min(0.0, std::max(-kTwoThirds, (1 + 2 * r) / 3));
        return std::min(2 * kTwoThirds * r, std::min((1 + 2 * r) / 3, 2.0));
    case FV_LIM_UTCDFS:
        if (r < -1) return r * (r + 1) / (r * r + 1);
        if ((r >= -1) && (r < 0)) return 0;
        if ((r >= 0) && (r < 0.5)) return r * r * r - 2 * (r * r) + 2 * r;
        if ((r >= 0.5) && (r < 2)) return 0.75 * r + 0.25;
        return (2 * (r * r) - 2 * r - 9.0 / 4.0) / (r * r - r - 1);
    case FV_LIM_SCHMIDTMANN: {
        const double alpha = 1, beta = 2, gamma = 1.5;
        const double phiO3 = (2 + r) / 3;
        return std::max(0.0, std::min(phiO3, std::max(-alpha * r, std::min({beta * r, phiO3, gamma}))));
    }
    }
    return 0;
}

// centre of face f seen from cell i (the wrap face of a periodic axis sits one period further
// on for its neighbour-side cell)
V3 faceCentreFrom(long long i, const Face& F) {
    return F.own == i ? F.rC : vsub(F.rC, F.neiShift);
}

// surfGrad of a scalar (gradient.hpp:96-168): inner faces (phi_N - phi_O) / |d|^2 * d, patches
// (ghost - phi_O) / |dR| * dR / |dR| with dR = 2 (r_f - r_O)
void surfGradScalar(const fvo_case& cs, const std::vector<double>& phi, int field, int k, std::vector<V3>& sg,
                    bool& bad) {
    const size_t nf = cs.faces.size();
    sg.assign(nf, v3(0, 0, 0));
    for (size_t f = 0; f < nf; ++f) {
        const Face& F = cs.faces[f];
        const V3& rO = cs.cells[F.own].rC;
        if (F.nei >= 0) {
            const V3 d = vsub(vadd(cs.cells[F.nei].rC, F.neiShift), rO);
            const double m = mag3(d);
            const double q = (phi[F.nei] - phi[F.own]) / (m * m);
            sg[f] = v3(q * d.x[0], q * d.x[1], q * d.x[2]);
        } else {
            const double b = bcCellS(cs, phi[F.own], field, k, F.patch, bad);
            const V3 dR = vmul(vsub(F.rC, rO), 2.);
            const double dm = mag3(dR);
            const V3 dn = vdiv(dR, dm);
            const double q = (b - phi[F.own]) / dm;
            sg[f] = v3(q * dn.x[0], q * dn.x[1], q * dn.x[2]);
        }
    }
}

void surfGradVector(const fvo_case& cs, const std::vector<V3>& phi, std::vector<T9>& sg, bool& bad) {
    const size_t nf = cs.faces.size();
    sg.assign(nf, T9{});
    for (size_t f = 0; f < nf; ++f) {
        const Face& F = cs.faces[f];
        const V3& rO = cs.cells[F.own].rC;
        if (F.nei >= 0) {
            const V3 d = vsub(vadd(cs.cells[F.nei].rC, F.neiShift), rO);
            const double m = mag3(d);
            sg[f] = outer(vdiv(vsub(phi[F.nei], phi[F.own]), m * m), d);
        } else {
            const V3 b = bcCellV(cs, phi[F.own], F.patch, F.N, bad);
            const V3 dR = vmul(vsub(F.rC, rO), 2.);
            const double dm = mag3(dR);
            const V3 dn = vdiv(dR, dm);
            sg[f] = outer(vdiv(vsub(b, phi[F.own]), dm), dn);
        }
    }
}

// thirdOrderLimiter (templates/thirdOrderLimiter.hpp:19-72): for face s1 of a cell and its
// farthest other face s2, r = g1 / (g2 + eps), retr = 1 / (r + eps), result
// 0.5 ((1 - 1/3) phi(r) g2 + (1 + 1/3) phi(retr) g1), component by component.
int farFace(const fvo_case& cs, long long i, int j) {
    const Cell& c = cs.cells[i];
    const V3 r1 = faceCentreFrom(i, cs.faces[c.faces[j]]);
    int far = 0;
    double best = 0;
    for (int j2 = 0; j2 < c.nFaces; ++j2) {
        if (j2 == j) continue;
        const double dist = mag3(vsub(faceCentreFrom(i, cs.faces[c.faces[j2]]), r1));
        if (best < dist) {
            best = dist;
            far = j2;
        }
    }
    return far;
}

inline double thirdOrderComponent(int lim, double g1, double g2) {
    const double r = g1 / (g2 + kStab);
    const double retr = 1. / (r + kStab);
    double limGrad, limOpp;
    if (lim == FV_LIM_ZERO) {
        limGrad = 0;
        limOpp = 0;
    } else if (lim == FV_LIM_LINEAR) {
        limGrad = g1;
        limOpp = g2;
    } else {
        limGrad = limiterPhiNoRS(lim, retr) * g1;
        limOpp = limiterPhiNoRS(lim, r) * g2;
    }
    return 0.5 * ((1 - 1. / 3.) * limOpp + (1 + 1. / 3.) * limGrad);
}

// thirdOrderLimiterCada (templates/thirdOrderLimiterCada.hpp:19-133) for one face s1 of cell i
// and its farthest face: with dx2 = (1 / minimalLengthScale_i)^2 (minimalLengthScale = 1 / min
// edge, Schemi.cpp:648-662), delta2 = dx2 (g & g) for the face's gradient gN and the farthest
// face's gO (dot product of the NC components in storage order), eta = (delta2N + delta2O) /
// (sqrt(5/2) (8 pi)^2 dx2).  eta < 1 - 1e-6: the unlimited 0.5 ((1 - 1/3) gO + (1 + 1/3) gN);
// eta > 1 + 1e-6: thirdOrderComponent; otherwise 0.5 ((1 - e) unlimited + (1 + e) limited) with
// e = (eta - 1) / 1e-6.
template <int NC>
void cadaLimit(int lim, const double* gN, const double* gO, double minLS, double* out) {
    const double pi8 = 8 * kPi;
    const double alpha = pi8 * pi8, eps = 1E-6;
    const double inv = 1 / minLS;
    const double dx2 = inv * inv;
    double sN = 0, sO = 0;
    for (int q = 0; q < NC; ++q) sN += gN[q] * gN[q];
    for (int q = 0; q < NC; ++q) sO += gO[q] * gO[q];
    const double delta2Near = dx2 * sN, delta2Oppose = dx2 * sO;
    const double eta = (delta2Near + delta2Oppose) / (std::sqrt(5.0 / 2.0) * alpha * dx2);
    for (int q = 0; q < NC; ++q) {
        const double unlimited = 0.5 * ((1 - 1. / 3.) * gO[q] + (1 + 1. / 3.) * gN[q]);
        if (eta < (1 - eps)) {
            out[q] = unlimited;
        } else if (eta > (1 + eps)) {
            out[q] = thirdOrderComponent(lim, gN[q], gO[q]);
        } else {
            const double limited = thirdOrderComponent(lim, gN[q], gO[q]);
            const double eta1eps = (eta - 1) / eps;
            out[q] = 0.5 * ((1 - eta1eps) * unlimited + (1 + eta1eps) * limited);
        }
    }
}

// TVDLimiter for a scalar field (TVDLimiter.cpp:12-125)
void tvdScalar(const fvo_case& cs, const std::vector<V3>& grad, const std::vector<double>& phi, int field, int k,
               std::vector<V3>& out, bool& bad) {
    out.resize(cs.nCells);
    const int lim = cs.cfg.limiter;
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        V3 list[12] = {};
        int nl = 0;
        for (int cx = 0; cx < c.nNb; ++cx) {
            const V3 d = vsub(vadd(cs.cells[c.nb[cx]].rC, c.nbShift[cx]), c.rC);
            const double dm = mag3(d);
            const V3 dn = vdiv(d, dm);
            V3 g;
            for (int j = 0; j < 3; ++j) g.x[j] = (phi[c.nb[cx]] - phi[i]) / dm * dn.x[j];
            list[nl++] = g;
        }
        if (c.nNb < c.nFaces) {
            for (int j = 0; j < c.nFaces; ++j) {
                const Face& F = cs.faces[c.faces[j]];
                if (F.nei >= 0) continue;
                const V3 d = vmul(vsub(F.rC, c.rC), 2);
                const double dm = mag3(d);
                const V3 dn = vdiv(d, dm);
                const double b = bcCellS(cs, phi[i], field, k, F.patch, bad);
                list[nl++] = v3((b - phi[i]) / dm * dn.x[0], (b - phi[i]) / dm * dn.x[1], (b - phi[i]) / dm * dn.x[2]);
            }
        }
        V3 mn = list[0], mx = list[0];
        for (int cx = 1; cx < nl; ++cx)
            for (int j = 0; j < 3; ++j) {
                mn.x[j] = std::min(mn.x[j], list[cx].x[j]);
                mx.x[j] = std::max(mx.x[j], list[cx].x[j]);
            }
        V3 res;
        for (int j = 0; j < 3; ++j) {
            const double r = mn.x[j] / (mx.x[j] + kStab);
            res.x[j] = limiterPhi(lim, r, 2 / (1 + r)) * grad[i].x[j];
        }
        if (lim == FV_LIM_ZERO) res = v3(0, 0, 0);
        if (lim == FV_LIM_LINEAR) res = grad[i];
        out[i] = res;
    }
}

// TVDLimiter for the velocity (TVDLimiter.cpp:127-272).  Note the index convention: the
// neighbour "gradients" are stored as [3*direction + component] while the Gauss gradient is
// [3*component + direction]; the limiter multiplies them element by element.
void tvdVector(const fvo_case& cs, const std::vector<T9>& grad, const std::vector<V3>& phi, std::vector<T9>& out,
               bool& bad) {
    out.resize(cs.nCells);
    const int lim = cs.cfg.limiter;
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        T9 list[12] = {};
        int nl = 0;
        for (int cx = 0; cx < c.nNb; ++cx) {
            const V3 d = vsub(vadd(cs.cells[c.nb[cx]].rC, c.nbShift[cx]), c.rC);
            const double dm = mag3(d);
            const V3 dn = vdiv(d, dm);
            const V3 dv = vsub(phi[c.nb[cx]], phi[i]);
            T9 g;
            for (int j = 0; j < 3; ++j)
                for (int q = 0; q < 3; ++q) g.x[3 * j + q] = dv.x[q] / dm * dn.x[j];
            list[nl++] = g;
        }
        if (c.nNb < c.nFaces) {
            for (int j = 0; j < c.nFaces; ++j) {
                const Face& F = cs.faces[c.faces[j]];
                if (F.nei >= 0) continue;
                const V3 d = vmul(vsub(F.rC, c.rC), 2);
                const double dm = mag3(d);
                const V3 dn = vdiv(d, dm);
                const V3 b = bcCellV(cs, phi[i], F.patch, F.N, bad);
                const V3 dv = vsub(b, phi[i]);
                T9 g;
                for (int jj = 0; jj < 3; ++jj)
                    for (int q = 0; q < 3; ++q) g.x[3 * jj + q] = dv.x[q] / dm * dn.x[jj];
                list[nl++] = g;
            }
        }
        T9 mn = list[0], mx = list[0];
        for (int cx = 1; cx < nl; ++cx)
            for (int q = 0; q < 9; ++q) {
                mn.x[q] = std::min(mn.x[q], list[cx].x[q]);
                mx.x[q] = std::max(mx.x[q], list[cx].x[q]);
            }
        T9 res;
        for (int q = 0; q < 9; ++q) {
            const double r = mn.x[q] / (mx.x[q] + kStab);
            res.x[q] = limiterPhi(lim, r, 2 / (1 + r)) * grad[i].x[q];
        }
        if (lim == FV_LIM_ZERO) res = T9{};
        if (lim == FV_LIM_LINEAR) res = grad[i];
        out[i] = res;
    }
}

// closure of a reconstructed face state: Advection.cpp:238-303 (owner), :305-387 (neighbour)
void closeFromPrimitive(const Mix& mx, FState& s) {
    s.c[0] = 0;
    s.rho[0] = 0;
    for (int k = 1; k <= mx.N; ++k) {
        s.c[0] += s.c[k];
        s.rho[k] = s.c[k] * mx.M[k - 1];
        s.rho[0] += s.rho[k];
    }
    s.Uv = mx.UvFromp(s.c, s.p);
    s.m = vmul(s.v, s.rho[0]);
    const double v2 = vdot(s.v, s.v);
    s.E = s.Uv + s.rho[0] * v2 * 0.5 + 0.0;
}

// recalculation after the Hancock half step: HancockStage.cpp:177-224 / :248-306
void closeFromConserved(const Mix& mx, FState& s) {
    s.c[0] = 0;
    for (int k = 1; k <= mx.N; ++k) {
        s.c[k] = s.rho[k] / mx.M[k - 1];
        s.c[0] += s.c[k];
    }
    s.v = vdiv(s.m, s.rho[0]);
    const double v2 = vdot(s.v, s.v);
    s.Uv = s.E - s.rho[0] * v2 * 0.5 - 0.0;
    s.p = mx.pFromUv(s.c, s.Uv);
}

struct Flux {
    V3 rho[FV_MAX_SPECIES + 1];
    T9 m;
    V3 E;
};

// HLLC (HLLCSolver.cpp:13-406) and HLL (HLLSolver.cpp:13-318) for one face; returns false
// when no branch applies (NaN wave speeds).  starV (HLLC): the face velocity the solver hands
// the diffusion stage (starValues.v, HLLCSolver.cpp:399): the side's velocity outside the star
// region, the star momentum over the star density inside it.  starP: the pressure beside it
// (starValues.p, :400): the side's pressure outside the star region, inside it pressureStar of
// the star state (pressureStarClass.cpp:12-36).
bool riemann(const fvo_case& cs, const FState& O, const FState& B, const V3& N, Flux& F, V3* starV = nullptr,
             double* starP = nullptr) {
    const Mix& mx = cs.mix;
    const int NS = mx.N;
    const double csO = std::sqrt(mx.sqSonicSpeed(O.c, O.rho[0], O.Uv, O.p) + kTwoThirds * 0.0 * (1. + mx.dpdUv(O.c, O.Uv)));
    const double csN = std::sqrt(mx.sqSonicSpeed(B.c, B.rho[0], B.Uv, B.p) + kTwoThirds * 0.0 * (1. + mx.dpdUv(B.c, B.Uv)));
    const double uO = vdot(O.v, N), uN = vdot(B.v, N);
    const double tpO = kTwoThirds * 0.0, tpN = kTwoThirds * 0.0;
    const double SO = std::min(uO - csO, uN - csN);
    const double SN = std::max(uO + csO, uN + csN);
    const V3 IN = N;  // tensor(1,0,0,0,1,0,0,0,1) & N
    const V3 INe = v3(1 * N.x[0] + 0 * N.x[1] + 0 * N.x[2], 0 * N.x[0] + 1 * N.x[1] + 0 * N.x[2],
                      0 * N.x[0] + 0 * N.x[1] + 1 * N.x[2]);
    (void)IN;
    // pressureStar: c_k = rho_k / M_k, Uv = E - 0.5 (m & m) / rho - rho k
    auto pStar = [&](const double* rs, const V3& ms, double Es) {
        const double kin = 0.5 * vdot(ms, ms) / rs[0];
        const double Uv = Es - kin - 0.0;
        double cst[FV_MAX_SPECIES + 1] = {};
        for (int k = 1; k <= NS; ++k) {
            cst[k] = rs[k] / mx.M[k - 1];
            cst[0] += cst[k];
        }
        return mx.pFromUv(cst, Uv);
    };
    if (cs.cfg.flux == FV_FLUX_HLLC) {
        const double Sc = ((B.p + tpN) - (O.p + tpO) + O.rho[0] * uO * (SO - uO) - B.rho[0] * uN * (SN - uN)) /
                          (O.rho[0] * (SO - uO) - B.rho[0] * (SN - uN));
        const double POwnNei = 0.5 * ((O.p + tpO) + (B.p + tpN) + O.rho[0] * (SO - uO) * (Sc - uO) +
                                      B.rho[0] * (SN - uN) * (Sc - uN));
        if (SO >= 0) {
            for (int k = 0; k <= NS; ++k) F.rho[k] = vmul(vmul(N, uO), O.rho[k]);
            F.m = outer(vadd(vmul(O.m, uO), vmul(INe, O.p + tpO)), N);
            F.E = vmul(N, uO * (O.E + O.p + tpO));
            if (starV) *starV = O.v;
            if (starP) *starP = O.p;
        } else if (Sc >= 0) {
            const double factor = SO - uO;
            const double den = 1 / (SO - Sc);
            double rs[FV_MAX_SPECIES + 1];
            for (int k = 0; k <= NS; ++k) rs[k] = O.rho[k] * factor * den;
            const V3 ms = vmul(vsub(vmul(O.m, factor), vmul(N, O.p + tpO - POwnNei)), den);
            const double Es = (O.E * factor - (O.p + tpO) * uO + POwnNei * Sc) * den;
            for (int k = 0; k <= NS; ++k) F.rho[k] = vmul(N, O.rho[k] * uO + SO * (rs[k] - O.rho[k]));
            F.m = outer(vadd(vadd(vmul(O.m, uO), vmul(INe, O.p + tpO)), vmul(vsub(ms, O.m), SO)), N);
            F.E = vmul(N, (O.E + O.p + tpO) * uO + SO * (Es - O.E));
            if (starV) *starV = vdiv(ms, rs[0]);
            if (starP) *starP = pStar(rs, ms, Es);
        } else if (SN > 0) {
            const double factor = SN - uN;
            const double den = 1 / (SN - Sc);
            double rs[FV_MAX_SPECIES + 1];
            for (int k = 0; k <= NS; ++k) rs[k] = B.rho[k] * factor * den;
            const V3 ms = vmul(vsub(vmul(B.m, factor), vmul(N, B.p + tpN - POwnNei)), den);
            const double Es = (B.E * factor - (B.p + tpN) * uN + POwnNei * Sc) * den;
            for (int k = 0; k <= NS; ++k) F.rho[k] = vmul(N, B.rho[k] * uN + SN * (rs[k] - B.rho[k]));
            F.m = outer(vadd(vadd(vmul(B.m, uN), vmul(INe, B.p + tpN)), vmul(vsub(ms, B.m), SN)), N);
            F.E = vmul(N, (B.E + B.p + tpN) * uN + SN * (Es - B.E));
            if (starV) *starV = vdiv(ms, rs[0]);
            if (starP) *starP = pStar(rs, ms, Es);
        } else if (SN <= 0) {
            for (int k = 0; k <= NS; ++k) F.rho[k] = vmul(vmul(N, uN), B.rho[k]);
            F.m = outer(vadd(vmul(B.m, uN), vmul(INe, B.p + tpN)), N);
            F.E = vmul(N, uN * (B.E + B.p + tpN));
            if (starV) *starV = B.v;
            if (starP) *starP = B.p;
        } else {
            return false;
        }
        return true;
    }
    // HLL
    if (SO >= 0) {
        for (int k = 0; k <= NS; ++k) F.rho[k] = vmul(N, uO * O.rho[k]);
        F.m = outer(vadd(vmul(O.m, uO), vmul(INe, O.p + tpO)), N);
        F.E = vmul(N, uO * (O.E + O.p + tpO));
    } else if (SN > 0) {
        const double den = 1 / (SN - SO);
        for (int k = 0; k <= NS; ++k)
            F.rho[k] = vmul(N, (SN * uO * O.rho[k] - SO * uN * B.rho[k] + SN * SO * (B.rho[k] - O.rho[k])) * den);
        const V3 t1 = vmul(vadd(vmul(O.m, uO), vmul(N, O.p + tpO)), SN);
        const V3 t2 = vmul(vadd(vmul(B.m, uN), vmul(N, B.p + tpN)), SO);
        const V3 t3 = vmul(vsub(B.m, O.m), SN * SO);
        F.m = outer(vmul(vadd(vsub(t1, t2), t3), den), N);
        F.E = vmul(N, (SN * (uO * (O.E + O.p + tpO)) - SO * (uN * (B.E + B.p + tpN)) + SN * SO * (B.E - O.E)) * den);
    } else if (SN <= 0) {
        for (int k = 0; k <= NS; ++k) F.rho[k] = vmul(N, uN * B.rho[k]);
        F.m = outer(vadd(vmul(B.m, uN), vmul(INe, B.p + tpN)), N);
        F.E = vmul(N, uN * (B.E + B.p + tpN));
    } else {
        return false;
    }
    return true;
}

void cellPrimitivesFromConserved(fvo_case& cs, long long i) {
    // Advection.cpp:455-479
    const Mix& mx = cs.mix;
    cs.c[0][i] = 0;
    for (int k = 1; k <= mx.N; ++k) {
        cs.c[k][i] = cs.rho[k][i] / mx.M[k - 1];
        cs.c[0][i] += cs.c[k][i];
    }
    cs.v[i] = vdiv(cs.m[i], cs.rho[0][i]);
    const double v2 = vdot(cs.v[i], cs.v[i]);
    cs.Uv[i] = cs.E[i] - cs.rho[0][i] * v2 * 0.5 - 0.0;
    double cc[FV_MAX_SPECIES + 1];
    for (int k = 0; k <= mx.N; ++k) cc[k] = cs.c[k][i];
    cs.p[i] = mx.pFromUv(cc, cs.Uv[i]);
}

// One advection of the state by dt: MUSCL-Hancock (Advection.cpp, hancock = true) or the same
// TVD reconstruction without the predictor (Advection2dOrder.cpp:20-636, hancock = false), whose
// boundary neighbour is the ghost of the reconstructed owner face (Advection2dOrder.cpp:394-522);
// third = true reconstructs with the per-face limited surface gradients of Advection3dOrder.cpp
// (no predictor either), cada = true with those of Advection3dOrderCada.cpp.
int doStep(fvo_case& cs, double dt, bool hancock = true, bool third = false, bool cada = false) {
    cs.Tvalid = false;  // the advection's temperature is TFromUv of its energy (Advection.cpp:478)
    const Mix& mx = cs.mix;
    const int NS = mx.N;
    const long long nc = cs.nCells;
    const size_t nf = cs.faces.size();
    bool bad = false;

    // 1. limited gradients (Advection.cpp:58-79; Advection3dOrder.cpp:56-107 surface gradients)
    std::vector<V3> limC[FV_MAX_SPECIES + 1];
    std::vector<T9> gv, limV;
    std::vector<V3> gp, limP;
    std::vector<V3> sgC[FV_MAX_SPECIES + 1], sgP;
    std::vector<T9> sgV;
    if (third) {
        for (int k = 1; k <= NS; ++k) surfGradScalar(cs, cs.c[k], 0, k - 1, sgC[k], bad);
        surfGradVector(cs, cs.v, sgV, bad);
        surfGradScalar(cs, cs.p, 2, 0, sgP, bad);
    } else {
        for (int k = 1; k <= NS; ++k) {
            std::vector<V3> g;
            gradScalar(cs, cs.c[k], 0, k - 1, g);
            tvdScalar(cs, g, cs.c[k], 0, k - 1, limC[k], bad);
        }
        gradVector(cs, cs.v, gv);
        tvdVector(cs, gv, cs.v, limV, bad);
        gradScalar(cs, cs.p, 2, 0, gp);
        tvdScalar(cs, gp, cs.p, 2, 0, limP, bad);
    }
    const int lim = cs.cfg.limiter;

    // 2. reconstruction (Advection.cpp:114-235) and closure
    std::vector<FState> own(nf), nei(nf);
    for (long long i = 0; i < nc; ++i) {
        const Cell& c = cs.cells[i];
        for (int j = 0; j < c.nFaces; ++j) {
            const int fi = c.faces[j];
            const Face& F = cs.faces[fi];
            // across a periodic wrap face the neighbour-side cell sits one period further on
            const V3 delta = (F.own == i) ? vsub(F.rC, c.rC) : vsub(F.rC, vadd(c.rC, F.neiShift));
            FState s{};
            if (third) {
                // the cell's limited gradient for this face (thirdOrderLimiter) against its farthest face
                const int far = farFace(cs, i, j);
                const int f2 = c.faces[far];
                for (int k = 1; k <= NS; ++k) {
                    V3 lg;
                    if (cada) cadaLimit<3>(lim, sgC[k][fi].x, sgC[k][f2].x, c.minLS, lg.x);
                    else
                        for (int q = 0; q < 3; ++q) lg.x[q] = thirdOrderComponent(lim, sgC[k][fi].x[q], sgC[k][f2].x[q]);
                    s.c[k] = vdot(lg, delta) + cs.c[k][i];
                }
                T9 lv;
                if (cada) cadaLimit<9>(lim, sgV[fi].x, sgV[f2].x, c.minLS, lv.x);
                else
                    for (int q = 0; q < 9; ++q) lv.x[q] = thirdOrderComponent(lim, sgV[fi].x[q], sgV[f2].x[q]);
                s.v = vadd(tdot(lv, delta), cs.v[i]);
                V3 lp;
                if (cada) cadaLimit<3>(lim, sgP[fi].x, sgP[f2].x, c.minLS, lp.x);
                else
                    for (int q = 0; q < 3; ++q) lp.x[q] = thirdOrderComponent(lim, sgP[fi].x[q], sgP[f2].x[q]);
                s.p = vdot(lp, delta) + cs.p[i];
            } else {
                for (int k = 1; k <= NS; ++k) s.c[k] = vdot(limC[k][i], delta) + cs.c[k][i];
                s.v = vadd(tdot(limV[i], delta), cs.v[i]);
                s.p = vdot(limP[i], delta) + cs.p[i];
            }
            if (F.own == i) own[fi] = s;
            else nei[fi] = s;
        }
    }
    for (size_t f = 0; f < nf; ++f) {
        closeFromPrimitive(mx, own[f]);
        if (cs.faces[f].nei >= 0) closeFromPrimitive(mx, nei[f]);
    }

    // 3. Hancock half step (HancockStage.cpp:10-240)
    const double halfTimestep = 0.5 * dt;
    for (long long i = 0; hancock && i < nc; ++i) {
        const Cell& c = cs.cells[i];
        double divR[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) {
            double acc = 0;
            for (int j = 0; j < c.nFaces; ++j) {
                const Face& F = cs.faces[c.faces[j]];
                const FState& s = (F.own == i) ? own[c.faces[j]] : nei[c.faces[j]];
                const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
                acc += vdot(vmul(s.v, s.rho[k]), n) * F.S;
            }
            divR[k] = acc / c.V;
        }
        V3 divM = v3(0, 0, 0);
        double divE = 0;
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            const FState& s = (F.own == i) ? own[c.faces[j]] : nei[c.faces[j]];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            const V3 tm = vmul(vadd(tdot(outer(s.m, s.v), n), vmul(n, s.p + kTwoThirds * 0.0)), F.S);
            divM.x[0] += tm.x[0]; divM.x[1] += tm.x[1]; divM.x[2] += tm.x[2];
            divE += (vdot(vmul(s.v, s.E), n) + vdot(vmul(s.v, s.p + kTwoThirds * 0.0), n)) * F.S;
        }
        divM = vdiv(divM, c.V);
        divE /= c.V;
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            FState& s = (F.own == i) ? own[c.faces[j]] : nei[c.faces[j]];
            for (int k = 0; k <= NS; ++k) s.rho[k] -= divR[k] * halfTimestep;
            const V3 dm = vmul(divM, halfTimestep);
            s.m.x[0] -= dm.x[0]; s.m.x[1] -= dm.x[1]; s.m.x[2] -= dm.x[2];
            s.E -= divE * halfTimestep;
        }
    }
    for (size_t f = 0; f < nf; ++f) {
        if (hancock) closeFromConserved(mx, own[f]);
        const Face& F = cs.faces[f];
        if (F.nei >= 0) {
            if (hancock) closeFromConserved(mx, nei[f]);
        } else {
            // ghost neighbour state (HancockStage.cpp:324-446)
            FState& s = nei[f];
            s.c[0] = 0;
            s.rho[0] = 0;
            for (int k = 1; k <= NS; ++k) {
                s.c[k] = bcCellS(cs, own[f].c[k], 0, k - 1, F.patch, bad);
                s.rho[k] = s.c[k] * mx.M[k - 1];
                s.c[0] += s.c[k];
                s.rho[0] += s.rho[k];
            }
            s.v = bcCellV(cs, own[f].v, F.patch, F.N, bad);
            s.m = vmul(s.v, s.rho[0]);
            s.p = bcCellS(cs, own[f].p, 2, 0, F.patch, bad);
            s.Uv = mx.UvFromp(s.c, s.p);
            const double v2 = vdot(s.v, s.v);
            s.E = s.Uv + s.rho[0] * v2 * 0.5 + 0.0;
        }
    }
    if (bad) {
        cs.err = "fixedValueSurface is not a valid cell boundary value";
        return FV_ERR_BOUNDARY;
    }

    // 4. fluxes
    std::vector<Flux> flux(nf);
    if (cs.cfg.diffusion) {
        cs.starV.assign(nf, v3(0, 0, 0));
        cs.starP.assign(nf, 0.0);
    }
    for (size_t f = 0; f < nf; ++f)
        if (!riemann(cs, own[f], nei[f], cs.faces[f].N, flux[f], cs.cfg.diffusion ? &cs.starV[f] : nullptr,
                     cs.cfg.diffusion ? &cs.starP[f] : nullptr)) {
            cs.err = "Fatal error in Riemann solver.";
            return FV_ERR_RIEMANN;
        }

    // 5. update (Advection.cpp:414-505)
    const V3 gvec = cs.g;
    for (long long i = 0; i < nc; ++i) {
        const Cell& c = cs.cells[i];
        double dE = 0;
        V3 dM = v3(0, 0, 0);
        double dR[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) dR[k] = 0;
        for (int j = 0; j < c.nFaces; ++j) {
            const int fi = c.faces[j];
            const Face& F = cs.faces[fi];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            dE += vdot(flux[fi].E, n) * F.S;
            const V3 tm = vmul(tdot(flux[fi].m, n), F.S);
            dM.x[0] += tm.x[0]; dM.x[1] += tm.x[1]; dM.x[2] += tm.x[2];
            for (int k = 0; k <= NS; ++k) dR[k] += vdot(flux[fi].rho[k], n) * F.S;
        }
        const double divE = dE / c.V;
        const V3 divM = vdiv(dM, c.V);
        const double rhoOld = cs.rho[0][i];
        const V3 vOld = cs.v[i];
        cs.E[i] -= divE * dt;
        const V3 mdt = vmul(divM, dt);
        cs.m[i].x[0] -= mdt.x[0]; cs.m[i].x[1] -= mdt.x[1]; cs.m[i].x[2] -= mdt.x[2];
        if (cs.cfg.gravity) {
            cs.E[i] += rhoOld * vdot(vOld, gvec) * dt;
            const V3 gm = vmul(vmul(gvec, rhoOld), dt);
            cs.m[i].x[0] += gm.x[0]; cs.m[i].x[1] += gm.x[1]; cs.m[i].x[2] += gm.x[2];
        }
        for (int k = 0; k <= NS; ++k) cs.rho[k][i] -= dR[k] / c.V * dt;
    }
    for (long long i = 0; i < nc; ++i) cellPrimitivesFromConserved(cs, i);
    return FV_OK;
}

// ---------------------------------------------------------------- SecondOrderRK / ThirdOrder
// The state a multi-stage step keeps as its start state Un.
struct StartState {
    std::vector<double> c[FV_MAX_SPECIES + 1], rho[FV_MAX_SPECIES + 1], E;
    std::vector<V3> m;
};

StartState saveState(const fvo_case& cs) {
    StartState u;
    for (int k = 0; k <= cs.mix.N; ++k) {
        u.c[k] = cs.c[k];
        u.rho[k] = cs.rho[k];
    }
    u.E = cs.E;
    u.m = cs.m;
    return u;
}

// gasPhase = (gasPhase).average(Un, ownWeight) followed by copyFrom (bunchOfFields.hpp:166-237):
// concentrations, densities, momentum and energy averaged field by field, then v = m / rho,
// Uv = E - k - 0.5 rho (v & v), p = pFromUv(c, Uv).  The averaged concentrations stay the state
// (the next stage or step reconstructs from them).
void averageWith(fvo_case& cs, const StartState& u, double ownWeight) {
    const int NS = cs.mix.N;
    const double own = ownWeight, in = 1 - ownWeight;
    for (long long i = 0; i < cs.nCells; ++i) {
        for (int k = 0; k <= NS; ++k) {
            cs.c[k][i] = own * cs.c[k][i] + in * u.c[k][i];
            cs.rho[k][i] = own * cs.rho[k][i] + in * u.rho[k][i];
        }
        for (int d = 0; d < 3; ++d) cs.m[i].x[d] = cs.m[i].x[d] * own + u.m[i].x[d] * in;
        cs.E[i] = own * cs.E[i] + in * u.E[i];
        cs.v[i] = vdiv(cs.m[i], cs.rho[0][i]);
        cs.Uv[i] = (cs.E[i] - 0.0) - 0.5 * cs.rho[0][i] * vdot(cs.v[i], cs.v[i]);
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) cc[k] = cs.c[k][i];
        cs.p[i] = cs.mix.pFromUv(cc, cs.Uv[i]);
    }
}

// secondOrderStepSolverRK::calculateStep (secondOrderStepSolverRK.cpp:48-71): two advections
// without the predictor, then Un2.average(Un, 0.5).
int rk2Step(fvo_case& cs, double dt) {
    const StartState u = saveState(cs);
    int st = doStep(cs, dt, false);
    if (st != FV_OK) return st;
    st = doStep(cs, dt, false);
    if (st != FV_OK) return st;
    averageWith(cs, u, 0.5);
    return FV_OK;
}

// thirdOrderStepSolver::calculateStep (thirdOrderStepSolver.cpp:48-82): SSP-RK3 of
// Advection3dOrder -- U1 = L(Un), U2 = 0.25 L(U1) + 0.75 Un, U3 = 2/3 L(U2) + 1/3 Un; with
// cada, of Advection3dOrderCada (thirdOrderStepSolverCada.cpp:48-84, the same stages).
int rk3Step(fvo_case& cs, double dt, bool cada) {
    const StartState u = saveState(cs);
    int st = doStep(cs, dt, false, true, cada);
    if (st != FV_OK) return st;
    st = doStep(cs, dt, false, true, cada);
    if (st != FV_OK) return st;
    averageWith(cs, u, 0.25);
    st = doStep(cs, dt, false, true, cada);
    if (st != FV_OK) return st;
    averageWith(cs, u, kTwoThirds);
    return FV_OK;
}

// ---------------------------------------------------------------- diffusion stage
// Diffusion.cpp:20-1061 for the molecular transport of a constant-coefficient gas
// (abstractTransportModel.cpp:52-187), no turbulence, the explicit solver (noMatrixSolver: each
// field advances as (explOldTime + freeTerm dt) / centralDiagonale, Diffusion.cpp:437-441,
// 787-797,818-825), one pass of its non-linearity loop (with turbulence off its convergence
// measure is 0 and it stops after the first pass, Diffusion.cpp:937-946), ideal and van der
// Waals mixtures.

// mixture functions of the stage (mixtureIdeal.cpp / mixtureVanDerWaals.cpp with
// idealFluid.cpp / vanDerWaalsFluid.cpp)
double dCv(const Mix& mx, const double* c) {  // Cv(concentrations): sum X_k Cv_k
    double Cvm, am, bm, Mm;
    mx.mixParams(c, Cvm, am, bm, Mm);
    return Cvm;
}
double dNonIdeality(const Mix& mx, const double* c) {  // ideal 0; vdW -a c^2
    if (mx.eos == FV_EOS_IDEAL) return 0;
    double Cvm, am, bm, Mm;
    mx.mixParams(c, Cvm, am, bm, Mm);
    return -am * (c[0] * c[0]);
}
double dUvcFromT(const Mix& mx, const double* c, double T) {  // ideal Cv T; vdW Cv T - a c
    double Cvm, am, bm, Mm;
    mx.mixParams(c, Cvm, am, bm, Mm);
    if (mx.eos == FV_EOS_IDEAL) return Cvm * T;
    return Cvm * T - am * c[0];
}
// hkT (mixtureIdeal.cpp:291-298, mixtureVanDerWaals.cpp:452-459): (UvcFromTk + pcFromTk) / T of
// species k alone at concentration ck
double dhkT(const Mix& mx, double ck, double T, int k) {
    if (mx.eos == FV_EOS_IDEAL) return (mx.Cv[k] * T + mx.R * T) / T;
    const double a = mx.a[k][k], b = mx.b[k][k];
    return ((mx.Cv[k] * T - a * ck) + (mx.R * T / (1 - ck * b) - a * ck)) / T;
}

// boundary concentrations of a patch from the owner cell (c_0 their sum in species order), the
// surface (boundaryConditionValueSurface) or the cell (boundaryConditionValueCell) variant
void dBoundaryConc(const fvo_case& cs, long long own, int patch, bool cellVariant, double* cB, bool& bad) {
    cB[0] = 0;
    for (int k = 1; k <= cs.N; ++k) {
        cB[k] = cellVariant ? bcCellS(cs, cs.c[k][own], 0, k - 1, patch, bad)
                            : bcSurfaceS(cs, cs.c[k][own], 0, k - 1, patch);
        cB[0] += cB[k];
    }
}
// calculatedTemperature (boundaryConditionValue.hpp:89-108 / 326-345)
double dBoundaryT(const fvo_case& cs, long long own, int patch, bool cellVariant, bool& bad) {
    double cB[FV_MAX_SPECIES + 1];
    dBoundaryConc(cs, own, patch, cellVariant, cB, bad);
    const double pB = cellVariant ? bcCellS(cs, cs.p[own], 2, 0, patch, bad) : bcSurfaceS(cs, cs.p[own], 2, 0, patch);
    return cs.mix.TFromUv(cB, cs.mix.UvFromp(cB, pB));
}

// surfGrad of a scalar cell field with a ghost value per boundary face (gradient.hpp:96-168)
template <class Ghost>
void dSurfGrad(const fvo_case& cs, const std::vector<double>& phi, Ghost ghost, std::vector<V3>& sg) {
    const size_t nf = cs.faces.size();
    sg.assign(nf, v3(0, 0, 0));
    for (size_t f = 0; f < nf; ++f) {
        const Face& F = cs.faces[f];
        const V3& rO = cs.cells[F.own].rC;
        if (F.nei >= 0) {
            const V3 d = vsub(vadd(cs.cells[F.nei].rC, F.neiShift), rO);
            const double m = mag3(d);
            const double q = (phi[F.nei] - phi[F.own]) / (m * m);
            sg[f] = v3(q * d.x[0], q * d.x[1], q * d.x[2]);
        } else {
            const double b = ghost(f);
            const V3 dR = vmul(vsub(F.rC, rO), 2.);
            const double dm = mag3(dR);
            const V3 dn = vdiv(dR, dm);
            const double q = (b - phi[F.own]) / dm;
            sg[f] = v3(q * dn.x[0], q * dn.x[1], q * dn.x[2]);
        }
    }
}
// linearInterpolate of a scalar cell field with a boundary face value (linearInterpolate.hpp:43-80)
template <class Bnd>
void dInterp(const fvo_case& cs, const std::vector<double>& phi, Bnd bnd, std::vector<double>& out) {
    const size_t nf = cs.faces.size();
    out.assign(nf, 0);
    for (size_t f = 0; f < nf; ++f) {
        const Face& F = cs.faces[f];
        out[f] = F.nei >= 0 ? phi[F.own] * F.wOwn + phi[F.nei] * F.wNei : bnd(f);
    }
}
// divergence of a surface vector field (divergence.hpp:58-88)
void dDivV(const fvo_case& cs, const std::vector<V3>& sf, std::vector<double>& out) {
    out.assign(cs.nCells, 0);
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        double acc = 0;
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            acc += vdot(sf[c.faces[j]], n) * F.S;
        }
        out[i] = acc / c.V;
    }
}
// divergence of a surface tensor field: sum (T & n) S / V
void dDivT(const fvo_case& cs, const std::vector<T9>& sf, std::vector<V3>& out) {
    out.assign(cs.nCells, v3(0, 0, 0));
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        V3 acc = v3(0, 0, 0);
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            const V3 t = vmul(tdot(sf[c.faces[j]], n), F.S);
            acc.x[0] += t.x[0]; acc.x[1] += t.x[1]; acc.x[2] += t.x[2];
        }
        out[i] = vdiv(acc, c.V);
    }
}
inline T9 ttrans(const T9& t) {  // tensor::transpose (tensor.cpp:57-69)
    T9 r = t;
    r.x[1] = t.x[3]; r.x[2] = t.x[6]; r.x[3] = t.x[1]; r.x[5] = t.x[7]; r.x[6] = t.x[2]; r.x[7] = t.x[5];
    return r;
}
inline T9 tadd(const T9& a, const T9& b) {
    T9 r;
    for (int q = 0; q < 9; ++q) r.x[q] = b.x[q] + a.x[q];
    return r;
}

// effectiveTransportCoefficients::caclulateDFluxes without turbulence (transportCoefficients.hpp:
// 256-325) for one face and one direction: the Maxwell-Stefan system of the molar-fraction
// gradients, the row of the least concentration replaced by sum N_k M_k J_k = 0, solved by the
// pivoting Gauss elimination of transportCoefficients.hpp:413-456, scaled by M_k c_k.
void dMaxwellStefan(int NS, const double* Nc, const double* M, const double (*Dm)[FV_MAX_SPECIES],
                    const double* gradXf, double* out) {
    double c[FV_MAX_SPECIES];
    for (int k = 1; k <= NS; ++k) c[k - 1] = Nc[k];
    double cmin = c[0];
    for (int k = 1; k < NS; ++k) cmin = std::min(cmin, c[k]);
    int replaceIndex = 0;
    for (int k = 0; k < NS; ++k)
        if (cmin == c[k]) { replaceIndex = k + 1; break; }
    double A[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
    double b[FV_MAX_SPECIES] = {};
    for (int k = 0; k < NS; ++k) b[k] = -gradXf[k];
    for (int k1 = 1; k1 <= NS; ++k1) {
        if (k1 != replaceIndex) {
            for (int k2 = 1; k2 <= NS; ++k2) {
                if (k1 == k2) continue;
                const double Aij = Nc[k1] * Nc[k2] / (Nc[0] * Nc[0] * Dm[k1 - 1][k2 - 1]);
                A[k1 - 1][k2 - 1] = -Aij;
                A[k1 - 1][k1 - 1] += Aij;
            }
        } else {
            b[k1 - 1] = 0;
            for (int k2 = 1; k2 <= NS; ++k2) A[k1 - 1][k2 - 1] = Nc[k2] * M[k2 - 1];
        }
    }
    // pivoting: each row k takes the row below with the largest (signed) entry of column k
    for (int k = 0; k < NS - 1; ++k) {
        double mv = A[k][k];
        int mi = k;
        for (int r = k + 1; r < NS; ++r)
            if (A[r][k] > mv) { mv = A[r][k]; mi = r; }
        if (mi != k) {
            for (int q = 0; q < NS; ++q) std::swap(A[mi][q], A[k][q]);
            std::swap(b[mi], b[k]);
        }
    }
    for (int k = 0; k < NS - 1; ++k)
        for (int i = k + 1; i < NS; ++i) {
            const double ratio = A[i][k] / (A[k][k] + kStab);
            for (int j = k + 1; j < NS; ++j) A[i][j] = A[i][j] - ratio * A[k][j];
            b[i] = b[i] - ratio * b[k];
        }
    double phi[FV_MAX_SPECIES];
    phi[NS - 1] = b[NS - 1] / (A[NS - 1][NS - 1] + kStab);
    for (int i = NS - 2; i >= 0; --i) {
        double term = 0.0;
        for (int j = i + 1; j < NS; ++j) term += A[i][j] * phi[j];
        phi[i] = (b[i] - term) / (A[i][i] + kStab);
    }
    for (int k = 0; k < NS; ++k) {
        if (std::fabs(phi[k]) < std::numeric_limits<double>::epsilon()) phi[k] = 0;  // normalize
        out[k] = phi[k] * M[k] * c[k];
    }
}

// ---- the implicit solver of the stage: SLEMatrix::generateDTimeLaplacian (SLEMatrix.cpp:410-546
// for a scalar, :706-907 for a vector, whose three components share the coefficients) and
// GaussSeidelSolver::algorithm (GaussSeidelSolver.cpp:12-82)
struct SLE1 {
    std::vector<double> diag, free;
    std::vector<std::vector<std::pair<double, long long>>> lower, upper;  // (coefficient, cell), face order
};
// rNew / dt + the faces' D / |d| (n S / V & d / |d|) on the diagonal; rOld / dt and each patch's
// coefficient times the ghost value in the free term; the neighbours' negated coefficients
template <class Ghost>
void dLaplacian(const fvo_case& cs, Ghost ghost, const std::vector<double>& rOld, const std::vector<double>& rNew,
                const std::vector<double>& Dface, double dt, SLE1& M) {
    const long long nc = cs.nCells;
    const double rt = 1 / dt;
    M.diag.assign(nc, 0.0);
    M.free.assign(nc, 0.0);
    M.lower.assign(nc, {});
    M.upper.assign(nc, {});
    for (long long i = 0; i < nc; ++i) {
        M.diag[i] = rNew[i] * rt;
        M.free[i] = rOld[i] * rt;
    }
    for (long long i = 0; i < nc; ++i) {
        const Cell& c = cs.cells[i];
        for (int j = 0; j < c.nFaces; ++j) {
            const int fi = c.faces[j];
            const Face& F = cs.faces[fi];
            if (F.nei >= 0) {
                long long o;
                V3 outerN, dR;
                if (F.own == i) {
                    o = F.nei;
                    outerN = vdiv(vmul(F.N, F.S), c.V);
                    dR = vsub(vadd(cs.cells[o].rC, F.neiShift), c.rC);
                } else {
                    o = F.own;
                    outerN = vmul(vdiv(vmul(F.N, F.S), c.V), -1);
                    dR = vsub(vsub(cs.cells[o].rC, F.neiShift), c.rC);  // the owner one period back
                }
                const double m = mag3(dR);
                const V3 dn = vdiv(dR, m);
                M.diag[i] += Dface[fi] / m * vdot(outerN, dn);
                const double off = -Dface[fi] / m * vdot(outerN, dn);
                if (o < i) M.lower[i].emplace_back(off, o);
                else M.upper[i].emplace_back(off, o);
            } else {
                const double b = ghost(i, fi);
                const V3 dR = vmul(vsub(F.rC, c.rC), 2);
                const double m = mag3(dR);
                const V3 dn = vdiv(dR, m);
                const V3 outerN = vdiv(vmul(F.N, F.S), c.V);
                M.diag[i] += Dface[fi] / m * vdot(outerN, dn);
                M.free[i] += Dface[fi] / m * vdot(outerN, dn) * b;
            }
        }
    }
}

// SLEMatrix::addNabla (src/SLE/SLEMatrix.cpp:291-401): the upwind term of the flow F across each
// face of each cell (its faces in order), F & (n S / V) with n outward: outgoing onto the
// diagonal, incoming onto the neighbour's entry (added to it, or appended) or, on a patch, times
// the field's cell-variant boundary value off the free term.
template <class Ghost>
void dAddNabla(const fvo_case& cs, Ghost ghost, const std::vector<V3>& Fface, SLE1& M) {
    for (long long i = 0; i < cs.nCells; ++i) {
        const Cell& c = cs.cells[i];
        for (int j = 0; j < c.nFaces; ++j) {
            const int fi = c.faces[j];
            const Face& F = cs.faces[fi];
            if (F.nei >= 0) {
                long long o;
                V3 outerN;
                if (F.own == i) {
                    o = F.nei;
                    outerN = vdiv(vmul(F.N, F.S), c.V);
                } else {
                    o = F.own;
                    outerN = vmul(vdiv(vmul(F.N, F.S), c.V), -1);
                }
                if (vdot(outerN, Fface[fi]) > 0) {
                    M.diag[i] += vdot(Fface[fi], outerN);
                } else {
                    auto& row = o < i ? M.lower[i] : M.upper[i];
                    auto it = std::find_if(row.begin(), row.end(), [o](const auto& p) { return p.second == o; });
                    if (it != row.end()) it->first += vdot(Fface[fi], outerN);
                    else row.emplace_back(vdot(Fface[fi], outerN), o);
                }
            } else {
                const V3 outerN = vdiv(vmul(F.N, F.S), c.V);
                if (vdot(outerN, Fface[fi]) > 0) M.diag[i] += vdot(Fface[fi], outerN);
                else M.free[i] -= vdot(Fface[fi], outerN) * ghost(i, fi);
            }
        }
    }
}
// a forward sweep, then a backward one, until 100 max |(new - old) / (|new| + eps)| is below
// convergenceToleranceGlobal (1e-12) or maxIt sweeps ran; normalize (|x| < DBL_EPSILON -> 0)
std::vector<double> dGaussSeidel(const SLE1& M, const std::vector<double>& start, long long maxIt) {
    const long long n = (long long)start.size();
    std::vector<double> oldI(start), newI(start);
    long long it = 0;
    while (true) {
        ++it;
        for (long long i = 0; i < n; ++i) {
            const double aii = 1. / M.diag[i];
            newI[i] = M.free[i] * aii;
            for (const auto& e : M.lower[i]) newI[i] -= e.first * newI[e.second] * aii;
            for (const auto& e : M.upper[i]) newI[i] -= e.first * oldI[e.second] * aii;
        }
        for (long long i = n - 1; i >= 0; --i) {
            const double aii = 1. / M.diag[i];
            newI[i] = M.free[i] * aii;
            for (size_t j = M.lower[i].size(); j-- > 0;) newI[i] -= M.lower[i][j].first * oldI[M.lower[i][j].second] * aii;
            for (size_t j = M.upper[i].size(); j-- > 0;) newI[i] -= M.upper[i][j].first * newI[M.upper[i][j].second] * aii;
        }
        double mx = 0;
        for (long long i = 0; i < n; ++i) {
            const double r = std::fabs((newI[i] - oldI[i]) / (std::fabs(newI[i]) + kStab));
            if (i == 0 || r > mx) mx = r;
        }
        const double diff = 100. * mx;
        if (diff < 1e-12 || it >= maxIt) {
            for (auto& x : newI)
                if (std::fabs(x) < std::numeric_limits<double>::epsilon()) x = 0;
            return newI;
        }
        oldI = newI;
    }
}

// The matrix solvers' convergence measure (abstractMatrixSolver::relativeIterationDifference,
// src/interfaces/abstractMatrixSolver.cpp:22-29): 100 max |(new - old) / (|new| + eps)|, the
// valarray's max taking the first element as it is and later ones when larger.
double dRelDiff(const std::vector<double>& oldI, const std::vector<double>& newI) {
    double mx = 0;
    for (size_t i = 0; i < newI.size(); ++i) {
        const double r = std::fabs((newI[i] - oldI[i]) / (std::fabs(newI[i]) + kStab));
        if (i == 0 || r > mx) mx = r;
    }
    return 100. * mx;
}
void dNormalize(std::vector<double>& x) {  // abstractMatrixSolver::normalize (:31-38)
    for (auto& v : x)
        if (std::fabs(v) < std::numeric_limits<double>::epsilon()) v = 0;
}

// JacobiSolver::algorithm (src/SLE/JacobiSolver.cpp:9-86): a forward and a backward pass per
// iteration, each row from the old iterate alone, (b + rowSum) / diag with rowSum the negated
// lower then upper terms, each list in reverse in the backward pass (whose values are the
// iterate); stop below the tolerance or at the iteration limit.
std::vector<double> dJacobi(const SLE1& M, const std::vector<double>& start, long long maxIt) {
    const long long n = (long long)start.size();
    std::vector<double> oldI(start), newI(start);
    long long it = 0;
    while (true) {
        ++it;
        for (long long i = 0; i < n; ++i) {
            const double aii = 1. / M.diag[i];
            double rowSum = 0;
            for (const auto& e : M.lower[i]) rowSum -= e.first * oldI[e.second];
            for (const auto& e : M.upper[i]) rowSum -= e.first * oldI[e.second];
            newI[i] = (M.free[i] + rowSum) * aii;
        }
        for (long long i = n - 1; i >= 0; --i) {
            const double aii = 1. / M.diag[i];
            double rowSum = 0;
            for (size_t j = M.lower[i].size(); j-- > 0;) rowSum -= M.lower[i][j].first * oldI[M.lower[i][j].second];
            for (size_t j = M.upper[i].size(); j-- > 0;) rowSum -= M.upper[i][j].first * oldI[M.upper[i][j].second];
            newI[i] = (M.free[i] + rowSum) * aii;
        }
        const double diff = dRelDiff(oldI, newI);
        if (diff < 1e-12 || it >= maxIt) {
            dNormalize(newI);
            return newI;
        }
        oldI = newI;
    }
}

// ThomasSolver::algorithm (src/SLE/ThomasSolver.cpp:9-52): the tridiagonal sweep of a 1D mesh,
// P_i = -u_i / (d_i + l_i P_{i-1}), Q_i = (f_i - l_i Q_{i-1}) / (d_i + l_i P_{i-1}), then
// x_i = P_i x_{i+1} + Q_i from the last row down.
std::vector<double> dThomas(const SLE1& M) {
    const long long N = (long long)M.diag.size();
    std::vector<double> x(N), P(N), Q(N);
    P[0] = -M.upper[0][0].first / M.diag[0];
    Q[0] = M.free[0] / M.diag[0];
    for (long long i = 1; i < N - 1; ++i) {
        const double l = M.lower[i][0].first;
        P[i] = -M.upper[i][0].first / (M.diag[i] + l * P[i - 1]);
        Q[i] = (M.free[i] - l * Q[i - 1]) / (M.diag[i] + l * P[i - 1]);
    }
    P[N - 1] = 0;
    {
        const double l = M.lower[N - 1][0].first;
        Q[N - 1] = (M.free[N - 1] - l * Q[N - 2]) / (M.diag[N - 1] + l * P[N - 2]);
    }
    x[N - 1] = Q[N - 1];
    for (long long i = N - 2; i >= 0; --i) x[i] = P[i] * x[i + 1] + Q[i];
    dNormalize(x);
    return x;
}

// operator& of a matrix and a vector (src/SLE/SLEMatrixDotProduct.cpp:9-31): diag v_i plus the
// lower then the upper entries, each list in order
std::vector<double> dMatVec(const SLE1& M, const std::vector<double>& v) {
    std::vector<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        double acc = M.diag[i] * v[i];
        for (const auto& e : M.lower[i]) acc += e.first * v[e.second];
        for (const auto& e : M.upper[i]) acc += e.first * v[e.second];
        r[i] = acc;
    }
    return r;
}
// sum() of a valarray expression such as (r * r).sum() (libstdc++ bits/valarray_after.h,
// _Expr::sum: from the last element down, a_{n-1} + a_{n-2} + ... + a_0) and the max of |a| (the
// first as it is, later ones when larger)
double dSum(const std::vector<double>& a) {
    if (a.empty()) return 0;
    size_t n = a.size();
    double s = a[--n];
    while (n != 0) s += a[--n];
    return s;
}
double dAbsMax(const std::vector<double>& a) {
    double m = std::fabs(a[0]);
    for (size_t i = 1; i < a.size(); ++i)
        if (std::fabs(a[i]) > m) m = std::fabs(a[i]);
    return m;
}
std::vector<double> dMul(const std::vector<double>& a, const std::vector<double>& b) {
    std::vector<double> r(a.size());
    for (size_t i = 0; i < a.size(); ++i) r[i] = a[i] * b[i];
    return r;
}
// SLEMatrixStorage::transpose (src/SLE/SLEMatrix.cpp:32-64): row i's lower entry (a, j) becomes
// row j's upper entry (a, i) and the reverse, rows appended in the order of i
SLE1 dTranspose(const SLE1& M) {
    SLE1 T;
    T.diag = M.diag;
    T.free = M.free;
    T.lower.assign(M.diag.size(), {});
    T.upper.assign(M.diag.size(), {});
    for (size_t i = 0; i < M.diag.size(); ++i) {
        for (const auto& e : M.lower[i]) T.upper[e.second].push_back({e.first, (long long)i});
        for (const auto& e : M.upper[i]) T.lower[e.second].push_back({e.first, (long long)i});
    }
    return T;
}
// The Jacobi preconditioner's product (JacobiConjugateGradientSolver.cpp:14-24: 1 / diag on the
// diagonal, the off-diagonal entries kept as zeros, so each adds 0 v_j)
std::vector<double> dPrecond(const SLE1& M, const std::vector<double>& v) {
    std::vector<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        double acc = (1. / M.diag[i]) * v[i];
        for (const auto& e : M.lower[i]) acc += 0 * v[e.second];
        for (const auto& e : M.upper[i]) acc += 0 * v[e.second];
        r[i] = acc;
    }
    return r;
}

// conjugateGradientSovler::algorithm (src/SLE/conjugateGradientSolver.cpp:10-53) and, with the
// Jacobi preconditioner, JacobiConjugateGradientSolver::algorithm (JacobiConjugateGradientSolver.
// cpp:10-83): the absolute residual max |r| below the tolerance after the first iteration, or the
// iteration limit.
std::vector<double> dCG(const SLE1& M, const std::vector<double>& start, long long maxIt, bool jacobi) {
    const size_t n = start.size();
    std::vector<double> x(start);
    std::vector<double> r = dMatVec(M, start);
    for (size_t i = 0; i < n; ++i) r[i] = M.free[i] - r[i];
    std::vector<double> d = jacobi ? dPrecond(M, r) : r;
    long long it = 0;
    while (true) {
        ++it;
        const double diff = dAbsMax(r);
        if ((diff < 1e-12 && it > 1) || it >= maxIt) {
            dNormalize(x);
            return x;
        }
        const std::vector<double> Ad = dMatVec(M, d);
        const double rz = jacobi ? dSum(dMul(r, dPrecond(M, r))) : dSum(dMul(r, r));
        const double alpha = rz / (dSum(dMul(d, Ad)) + kStab);
        for (size_t i = 0; i < n; ++i) x[i] += alpha * d[i];
        std::vector<double> r1(n);
        for (size_t i = 0; i < n; ++i) r1[i] = r[i] - alpha * Ad[i];
        const std::vector<double> z1 = jacobi ? dPrecond(M, r1) : r1;
        const double beta = dSum(dMul(r1, z1)) / (rz + kStab);
        for (size_t i = 0; i < n; ++i) d[i] = z1[i] + beta * d[i];
        r = r1;
    }
}

// biConjugateGradientSovler::algorithm (src/SLE/biConjugateGradientSolver.cpp:10-75): the shadow
// residual and direction through the transposed matrix
std::vector<double> dBiCG(const SLE1& M, const std::vector<double>& start, long long maxIt) {
    const size_t n = start.size();
    const SLE1 MT = dTranspose(M);
    std::vector<double> x(start);
    std::vector<double> r = dMatVec(M, start);
    for (size_t i = 0; i < n; ++i) r[i] = M.free[i] - r[i];
    std::vector<double> d = r, ro = r, dO = r;
    long long it = 0;
    while (true) {
        ++it;
        const double diff = dAbsMax(r);
        if ((diff < 1e-12 && it > 1) || it >= maxIt) {
            dNormalize(x);
            return x;
        }
        const std::vector<double> Ad = dMatVec(M, d);
        const double rr = dSum(dMul(ro, r));
        const double alpha = rr / (dSum(dMul(dO, Ad)) + kStab);
        for (size_t i = 0; i < n; ++i) x[i] += alpha * d[i];
        std::vector<double> r1(n), ro1(n);
        for (size_t i = 0; i < n; ++i) r1[i] = r[i] - alpha * Ad[i];
        const std::vector<double> ATdo = dMatVec(MT, dO);
        for (size_t i = 0; i < n; ++i) ro1[i] = ro[i] - alpha * ATdo[i];
        const double beta = dSum(dMul(ro1, r1)) / (rr + kStab);
        for (size_t i = 0; i < n; ++i) {
            d[i] = r1[i] + beta * d[i];
            dO[i] = ro1[i] + beta * dO[i];
        }
        r = r1;
        ro = ro1;
    }
}

// the stage's implicit solver (abstractMatrixSolver::createMatrixSolver, :50-120)
std::vector<double> dSolve(const fv_config& cf, const SLE1& M, const std::vector<double>& start) {
    if (cf.sle_solver == FV_SLE_JACOBI) return dJacobi(M, start, cf.sle_max_iter);
    if (cf.sle_solver == FV_SLE_THOMAS) return dThomas(M);
    if (cf.sle_solver == FV_SLE_NO_SOLVER) return start;  // noMatrixSolver::solve
    if (cf.sle_solver == FV_SLE_CG) return dCG(M, start, cf.sle_max_iter, false);
    if (cf.sle_solver == FV_SLE_JACOBI_CG) return dCG(M, start, cf.sle_max_iter, true);
    if (cf.sle_solver == FV_SLE_BICG) return dBiCG(M, start, cf.sle_max_iter);
    return dGaussSeidel(M, start, cf.sle_max_iter);
}

// ---------------------------------------------------------------- transport models
// Molecular transport coefficients of one point from its temperature T, pressure p and
// concentrations c[0..N] (c[0] the total): transportCoefficients::calculateCoefficients
// (templates/transportCoefficients.hpp:124-133) over the model's calculateMu, calculateDm,
// calculateDs and calculateKappa.
struct Transport {
    double mu = 0, kappa = 0;
    double Dm[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};  // binary coefficients (off the diagonal)
    double Ds[FV_MAX_SPECIES] = {};                  // coefficient of each species in the mixture
};

// Collision integrals of the Lennard-Jones potential at the reduced temperature Ts
// (LennardJonesTransportModel.cpp:10-29): Omega(2,2) for mu and kappa, Omega(1,1) for D.
double ljOmegaMuKappa(double Ts) {
    constexpr double Ac = 1.16145, Bc = 0.14874, Cc = 0.52487, Dc = 0.77320, Ec = 2.16178, Fc = 2.4378;
    return Ac * std::pow(Ts, -Bc) + Cc * std::exp(-Dc * Ts) + Ec * std::exp(-Fc * Ts);
}
double ljOmegaD(double Ts) {
    constexpr double Ac = 1.06036, Bc = 0.1561, Cc = 0.19300, Dc = 0.47635, Ec = 1.03587, Fc = 1.52996,
                     Gc = 1.76474, Hc = 3.89411;
    return Ac * std::pow(Ts, -Bc) + Cc * std::exp(-Dc * Ts) + Ec * std::exp(-Fc * Ts) + Gc * std::exp(-Hc * Ts);
}

// Kinetic-theory values of one species or pair (hardSpheresTransportModel.cpp:11-38 with
// Omega = 1; LennardJonesTransportModel.cpp:31-60): M in kg/mol, sigma in angstrom, each added
// to the model's constant.
double ktMu(const fv_config& cf, double M, double T, double Omega, double sigma) {
    const double v = 2.6693E-6 * std::sqrt(1E3) * std::sqrt(M * T) / Omega / (sigma * sigma);
    return cf.mu_const + v;
}
double ktD(const fv_config& cf, double M, double T, double p, double Omega, double sigma) {
    const double v = 2.6280E-7 / std::sqrt(1E3) / Omega * std::sqrt(T * T * T / M) / (p / 101325. * (sigma * sigma));
    return cf.D_const + v;
}
double ktKappa(const fv_config& cf, double M, double T, double Omega, double sigma) {
    const double v = 4.184 * 1.9891E-2 / std::sqrt(1E3) * std::sqrt(T / M) / Omega / (sigma * sigma);
    return cf.kappa_const + v;
}
// the hard-sphere forms carry no Omega: the same expressions without the division
double hsMu(const fv_config& cf, double M, double T, double sigma) {
    const double v = 2.6693E-6 * std::sqrt(1E3) * std::sqrt(M * T) / (sigma * sigma);
    return cf.mu_const + v;
}
double hsD(const fv_config& cf, double M, double T, double p, double sigma) {
    const double v = 2.6280E-7 / std::sqrt(1E3) * std::sqrt(T * T * T / M) / (p / 101325. * (sigma * sigma));
    return cf.D_const + v;
}
double hsKappa(const fv_config& cf, double M, double T, double sigma) {
    const double v = 4.184 * 1.9891E-2 / std::sqrt(1E3) * std::sqrt(T / M) / (sigma * sigma);
    return cf.kappa_const + v;
}

// Wilke's mixing rule of the species' values q_k (hardSpheresTransportModel.cpp:55-77 for mu,
// :189-210 for kappa with the factor 0.85 on Phi)
double wilke(int N, const double* x, const double* q, const double* M, double phiScale) {
    double Phi[FV_MAX_SPECIES][FV_MAX_SPECIES];
    for (int k1 = 0; k1 < N; ++k1)
        for (int k2 = 0; k2 < N; ++k2) {
            const double num = 1 + std::sqrt(q[k1] / q[k2]) * std::sqrt(std::sqrt(M[k2] / M[k1]));
            const double dem = 8 * (1 + M[k1] / M[k2]);
            Phi[k1][k2] = phiScale == 1.0 ? num * num / std::sqrt(dem) : phiScale * num * num / std::sqrt(dem);
        }
    double mix = 0;
    for (int k1 = 0; k1 < N; ++k1) {
        double Phi_k1 = 0;
        for (int k2 = 0; k2 < N; ++k2) Phi_k1 += x[k2] * Phi[k1][k2];
        mix += x[k1] * q[k1] / Phi_k1;
    }
    return mix;
}

// The coefficients of one point.  surface = true: a face's, whose Ds guards the inverse sum with
// the stabilizator (hardSpheresTransportModel.cpp:360-388); the cells' Ds (:133-170) is not used
// by the stage and is not formed.
void transportPoint(const fv_config& cf, const Mix& mx, double T, double p, const double* c, bool surface,
                    Transport& out) {
    const int N = mx.N;
    out = Transport();
    if (cf.transport == FV_TRANSPORT_CONSTANT) {  // abstractTransportModel.cpp:82-187
        out.mu = cf.mu_const;
        out.kappa = cf.kappa_const;
        for (int k1 = 0; k1 < N; ++k1) {
            out.Ds[k1] = cf.D_const;
            for (int k2 = 0; k2 < N; ++k2)
                if (k1 != k2) out.Dm[k1][k2] = cf.D_const;
        }
        return;
    }
    const bool lj = cf.transport == FV_TRANSPORT_LENNARD_JONES;
    double x[FV_MAX_SPECIES] = {}, muk[FV_MAX_SPECIES] = {}, kk[FV_MAX_SPECIES] = {};
    for (int k = 0; k < N; ++k) x[k] = c[k + 1] / c[0];
    for (int k = 0; k < N; ++k) {
        if (lj) {
            const double Om = ljOmegaMuKappa(T / cf.transport_lj_eps[k]);
            muk[k] = ktMu(cf, mx.M[k], T, Om, cf.transport_lj_sigma[k]);
            kk[k] = ktKappa(cf, mx.M[k], T, Om, cf.transport_lj_sigma[k]);
        } else {
            muk[k] = hsMu(cf, mx.M[k], T, cf.transport_diameter[k]);
            kk[k] = hsKappa(cf, mx.M[k], T, cf.transport_diameter[k]);
        }
    }
    out.mu = wilke(N, x, muk, mx.M, 1.0);
    out.kappa = wilke(N, x, kk, mx.M, 0.85);
    for (int k1 = 0; k1 < N; ++k1)
        for (int k2 = 0; k2 < N; ++k2) {
            if (k1 == k2) continue;
            const double M12 = 2 * mx.M[k1] * mx.M[k2] / (mx.M[k1] + mx.M[k2]);
            if (lj) {
                const double Om = ljOmegaD(T / std::sqrt(cf.transport_lj_eps[k1] * cf.transport_lj_eps[k2]));
                const double s12 = 0.5 * (cf.transport_lj_sigma[k1] + cf.transport_lj_sigma[k2]);
                out.Dm[k1][k2] = ktD(cf, M12, T, p, Om, s12);
            } else {
                const double d12 = 0.5 * (cf.transport_diameter[k1] + cf.transport_diameter[k2]);
                out.Dm[k1][k2] = hsD(cf, M12, T, p, d12);
            }
        }
    if (!surface) return;
    for (int k1 = 0; k1 < N; ++k1) {
        double rDk = 0;
        for (int k2 = 0; k2 < N; ++k2) {
            if (k1 == k2) continue;
            rDk += x[k2] / out.Dm[k1][k2];
        }
        if (rDk >= kStab) {
            rDk *= 1.0 / (1.0 - x[k1] + kStab);
            out.Ds[k1] = 1 / rDk;
        } else {
            out.Ds[k1] = kStab;
        }
    }
}

int diffusionStage(fvo_case& cs, double dt) {
    const Mix& mx = cs.mix;
    const int NS = cs.N;
    const long long nc = cs.nCells;
    const size_t nf = cs.faces.size();
    const fv_config& cf = cs.cfg;
    bool bad = false;
    auto conc = [&](long long i, double* c) { for (int k = 0; k <= NS; ++k) c[k] = cs.c[k][i]; };

    // the phase after the advection: temperature (Advection.cpp:478), mass fractions
    // (diffusiveFields.cpp:24-46), velocity
    std::vector<double> T(nc);
    std::vector<std::vector<double>> w(NS, std::vector<double>(nc));
    for (long long i = 0; i < nc; ++i) {
        double cc[FV_MAX_SPECIES + 1];
        conc(i, cc);
        T[i] = mx.TFromUv(cc, cs.Uv[i]);
        double sum = 0.0;
        for (int k = 0; k < NS; ++k) {
            w[k][i] = cs.rho[k + 1][i] / cs.rho[0][i];
            sum += w[k][i];
        }
        for (int k = 0; k < NS; ++k) w[k][i] /= sum;
    }
    const std::vector<V3>& v = cs.v;

    // Diffusion.cpp:136-176
    std::vector<double> nonIdOld(nc), CVOld(nc), CvM(nc), CCVOld(nc), NonIdRho(nc);
    for (long long i = 0; i < nc; ++i) {
        double cc[FV_MAX_SPECIES + 1];
        conc(i, cc);
        nonIdOld[i] = dNonIdeality(mx, cc);
        const double avMolMass = cs.rho[0][i] / cs.c[0][i];
        CVOld[i] = dCv(mx, cc);
        CvM[i] = CVOld[i] / avMolMass;
        CCVOld[i] = cs.c[0][i] * CVOld[i];
        NonIdRho[i] = nonIdOld[i] / cs.rho[0][i];
    }
    std::vector<double> surfaceCv;
    dInterp(cs, CVOld, [&](size_t f) {  // calculatedCv
        double cB[FV_MAX_SPECIES + 1];
        dBoundaryConc(cs, cs.faces[f].own, cs.faces[f].patch, false, cB, bad);
        return dCv(mx, cB);
    }, surfaceCv);
    std::vector<std::vector<double>> sc(NS + 1, std::vector<double>(nf, 0.0));
    std::vector<double> surfaceRho(nf, 0.0);
    for (int k = 1; k <= NS; ++k) {
        std::vector<double> sk;
        dInterp(cs, cs.c[k], [&](size_t f) {
            return bcSurfaceS(cs, cs.c[k][cs.faces[f].own], 0, k - 1, cs.faces[f].patch);
        }, sk);
        for (size_t f = 0; f < nf; ++f) {
            sc[k][f] = sk[f];
            sc[0][f] += sk[f];
            surfaceRho[f] += sk[f] * mx.M[k - 1];
        }
    }
    std::vector<V3> gradNonIdRho, gradCvM;
    dSurfGrad(cs, NonIdRho, [&](size_t f) {  // calculatedNonidealityCorrectionPerDensity (cell)
        const long long o = cs.faces[f].own;
        const int pt = cs.faces[f].patch;
        double cB[FV_MAX_SPECIES + 1];
        dBoundaryConc(cs, o, pt, true, cB, bad);
        double dens = 0;
        for (int k = 1; k <= NS; ++k) dens += cB[k] * mx.M[k - 1];
        const double Tb = dBoundaryT(cs, o, pt, false, bad);
        (void)Tb;  // the ideal and van der Waals corrections do not depend on T
        return dNonIdeality(mx, cB) / dens;
    }, gradNonIdRho);
    dSurfGrad(cs, CvM, [&](size_t f) {  // calculatedCvM (cell)
        double cB[FV_MAX_SPECIES + 1];
        dBoundaryConc(cs, cs.faces[f].own, cs.faces[f].patch, true, cB, bad);
        double dens = 0;
        for (int k = 1; k <= NS; ++k) dens += cB[k] * mx.M[k - 1];
        return dCv(mx, cB) * cB[0] / dens;
    }, gradCvM);

    // velocity gradients (Diffusion.cpp:178-229): the cell gradient from the Riemann star
    // velocities ("star"; under gravity the interpolated cell velocities, secondOrderStepSolver.cpp:
    // 71-73) or from the cells ("linear")
    std::vector<V3> starV = cs.starV;
    if (cf.gravity || cf.linear_reconstruction)
        for (size_t f = 0; f < nf; ++f) {
            const Face& F = cs.faces[f];
            starV[f] = F.nei >= 0 ? vadd(vmul(v[F.own], F.wOwn), vmul(v[F.nei], F.wNei))
                                  : bcSurfaceV(cs, v[F.own], F.patch, F.N);
        }
    std::vector<T9> gradV(nc);
    std::vector<double> divV;
    for (long long i = 0; i < nc; ++i) {
        const Cell& c = cs.cells[i];
        T9 acc{};
        for (int j = 0; j < c.nFaces; ++j) {
            const Face& F = cs.faces[c.faces[j]];
            const V3 n = (F.own == i) ? F.N : vmul(F.N, -1);
            const T9 term = tmul(outer(starV[c.faces[j]], n), F.S);
            for (int q = 0; q < 9; ++q) acc.x[q] += term.x[q];
        }
        for (int q = 0; q < 9; ++q) gradV[i].x[q] = acc.x[q] / c.V;
    }
    dDivV(cs, starV, divV);
    std::vector<T9> gradVs;
    surfGradVector(cs, v, gradVs, bad);
    std::vector<double> divVs(nf);
    for (size_t f = 0; f < nf; ++f) {  // surfDivergence (divergence.hpp:90-150)
        const Face& F = cs.faces[f];
        const V3& rO = cs.cells[F.own].rC;
        if (F.nei >= 0) {
            const V3 d = vsub(vadd(cs.cells[F.nei].rC, F.neiShift), rO);
            const double m = mag3(d);
            divVs[f] = vdot(vdiv(vsub(v[F.nei], v[F.own]), m * m), d);
        } else {
            const V3 b = bcCellV(cs, v[F.own], F.patch, F.N, bad);
            const V3 dR = vmul(vsub(F.rC, rO), 2.);
            const double dm = mag3(dR);
            divVs[f] = vdot(vdiv(vsub(b, v[F.own]), dm), vdiv(dR, dm));
        }
    }
    std::vector<double> surfaceT;
    dInterp(cs, T, [&](size_t f) { return dBoundaryT(cs, cs.faces[f].own, cs.faces[f].patch, false, bad); }, surfaceT);

    // transport coefficients: the cells' of the phase (its viscosity enters the viscous heating)
    // and the faces' of the interpolated temperature and concentrations and the star pressure
    // (Diffusion.cpp:130-132,238-240)
    std::vector<double> muC(nc);
    for (long long i = 0; i < nc; ++i) {
        double cc[FV_MAX_SPECIES + 1];
        conc(i, cc);
        Transport t;
        transportPoint(cf, mx, T[i], cs.p[i], cc, false, t);
        muC[i] = t.mu;
    }
    std::vector<Transport> trF(nf);
    for (size_t f = 0; f < nf; ++f) {
        double Nc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) Nc[k] = sc[k][f];
        transportPoint(cf, mx, surfaceT[f], cs.starP[f], Nc, true, trF[f]);
    }
    std::vector<T9> strainVol(nc), strainSurf1(nf);
    for (long long i = 0; i < nc; ++i) {
        strainVol[i] = tadd(gradV[i], ttrans(gradV[i]));
        const double l = kTwoThirds * divV[i];
        strainVol[i].x[0] -= l; strainVol[i].x[4] -= l; strainVol[i].x[8] -= l;
    }
    for (size_t f = 0; f < nf; ++f) {
        strainSurf1[f] = ttrans(gradVs[f]);
        const double l = kTwoThirds * divVs[f];
        strainSurf1[f].x[0] -= l; strainSurf1[f].x[4] -= l; strainSurf1[f].x[8] -= l;
    }

    // effective coefficients without turbulence (transportCoefficients.hpp:222-232)
    std::vector<std::vector<double>> rhoD(NS, std::vector<double>(nf));
    for (int k = 0; k < NS; ++k)
        for (size_t f = 0; f < nf; ++f) rhoD[k][f] = surfaceRho[f] * trF[f].Ds[k];

    // mass-fraction matrices (Diffusion.cpp:321-339; SLEMatrix.cpp:2054-2078 explicit,
    // :410-546 implicit)
    const bool gs = cf.sle_solver != FV_SLE_EXPLICIT;  // the implicit branch: Gauss-Seidel, Jacobi, Thomas, noSolver
    std::vector<std::vector<V3>> gradW(NS);
    std::vector<std::vector<double>> diagW(NS, std::vector<double>(nc)), oldW(NS, std::vector<double>(nc)),
        freeW(NS, std::vector<double>(nc, 0.0));
    std::vector<SLE1> MW(gs ? NS : 0);
    for (int k = 0; k < NS; ++k) {
        auto ghostW = [&, k](size_t f) {  // calculatedMassFraction (cell), component k + 1
            double cB[FV_MAX_SPECIES + 1];
            dBoundaryConc(cs, cs.faces[f].own, cs.faces[f].patch, true, cB, bad);
            const double dens = cB[k + 1] * mx.M[k];
            double sum = 0;
            for (int q = 1; q <= NS; ++q) sum += cB[q] * mx.M[q - 1];
            return dens / sum;
        };
        dSurfGrad(cs, w[k], ghostW, gradW[k]);
        for (long long i = 0; i < nc; ++i) oldW[k][i] = w[k][i] * cs.rho[0][i];
        if (gs) {
            dLaplacian(cs, [&](long long, int fi) { return ghostW(fi); }, oldW[k], cs.rho[0], rhoD[k], dt, MW[k]);
            diagW[k] = MW[k].diag;
            freeW[k] = MW[k].free;
            continue;
        }
        std::vector<V3> flow(nf);
        for (size_t f = 0; f < nf; ++f) flow[f] = vmul(vmul(gradW[k][f], rhoD[k][f]), -1.);
        std::vector<double> div;
        dDivV(cs, flow, div);
        for (long long i = 0; i < nc; ++i) {
            diagW[k][i] = cs.rho[0][i];
            freeW[k][i] -= div[i];
        }
    }

    // molar-mass correction and explicit enthalpy flow (Diffusion.cpp:341-422)
    std::vector<V3> entFlow(nf, v3(0, 0, 0));
    if (cf.molmass_diffusion || cf.enthalpy_flow != FV_ENTHALPY_NO) {
        std::vector<std::vector<V3>> gradX(NS);
        std::vector<std::vector<V3>> DFlux(NS, std::vector<V3>(nf, v3(0, 0, 0)));
        if (cf.molmass_diffusion) {
            for (int k = 0; k < NS; ++k) {
                std::vector<double> X(nc);
                for (long long i = 0; i < nc; ++i) X[i] = cs.c[k + 1][i] / cs.c[0][i];
                dSurfGrad(cs, X, [&](size_t f) {  // calculatedMolarFraction (cell), component k + 1
                    double cB[FV_MAX_SPECIES + 1];
                    dBoundaryConc(cs, cs.faces[f].own, cs.faces[f].patch, true, cB, bad);
                    double sum = 0;
                    for (int q = 1; q <= NS; ++q) sum += cB[q];
                    return cB[k + 1] / sum;
                }, gradX[k]);
            }
            for (size_t f = 0; f < nf; ++f) {
                if (NS > 1) {
                    double Nc[FV_MAX_SPECIES + 1];
                    for (int k = 0; k <= NS; ++k) Nc[k] = sc[k][f];
                    for (int d = 0; d < 3; ++d) {
                        double g[FV_MAX_SPECIES], out[FV_MAX_SPECIES];
                        for (int k = 0; k < NS; ++k) g[k] = gradX[k][f].x[d];
                        dMaxwellStefan(NS, Nc, mx.M, trF[f].Dm, g, out);
                        for (int k = 0; k < NS; ++k) DFlux[k][f].x[d] = out[k];
                    }
                }
            }
        }
        for (int k = 0; k < NS; ++k) {
            std::vector<V3> flowW(nf), corr(nf, v3(0, 0, 0));
            for (size_t f = 0; f < nf; ++f) flowW[f] = vmul(gradW[k][f], -1 * rhoD[k][f]);
            if (cf.molmass_diffusion) {
                for (size_t f = 0; f < nf; ++f) corr[f] = vsub(DFlux[k][f], flowW[f]);
                std::vector<double> div;
                dDivV(cs, corr, div);
                for (long long i = 0; i < nc; ++i) {  // distributeSourceTerm (SLEMatrix.cpp:2166-2175)
                    const double s = div[i] * (-1.0);
                    if (s >= 0.) freeW[k][i] += s;
                    else diagW[k][i] -= s / (w[k][i] + kStab);
                }
            }
            if (cf.enthalpy_flow != FV_ENTHALPY_NO)
                for (size_t f = 0; f < nf; ++f) {
                    const double h = dhkT(mx, sc[k + 1][f], surfaceT[f], k);
                    const V3 t = vdiv(vmul(vadd(corr[f], flowW[f]), h), mx.M[k]);
                    entFlow[f] = vadd(entFlow[f], t);
                }
        }
    }

    // non-ideality correction (Diffusion.cpp:424-428; tLambda is zero without turbulence)
    std::vector<V3> nonIdLap(nf);
    for (size_t f = 0; f < nf; ++f) {
        const V3 nonIdFlow = vmul(vadd(vmul(gradCvM[f], surfaceT[f]), gradNonIdRho[f]), -1.);
        nonIdLap[f] = vmul(vmul(nonIdFlow, surfaceRho[f]), 0.0);
    }

    // new mass fractions and concentrations (Diffusion.cpp:430-476)
    std::vector<std::vector<double>> wSol(gs ? NS : 0);
    for (int k = 0; k < (gs ? NS : 0); ++k) {
        MW[k].diag = diagW[k];
        MW[k].free = freeW[k];
        wSol[k] = dSolve(cf, MW[k], w[k]);
    }
    std::vector<std::vector<double>> wNew(NS, std::vector<double>(nc));
    std::vector<std::vector<double>> cN(NS + 1, std::vector<double>(nc));
    for (long long i = 0; i < nc; ++i) {
        double sum = 0.;
        for (int k = 0; k < NS; ++k) {
            double x = gs ? wSol[k][i] : (oldW[k][i] + freeW[k][i] * dt) / diagW[k][i];
            if (x < 0.) x = 0.0;
            wNew[k][i] = x;
            sum += x;
        }
        for (int k = 0; k < NS; ++k) wNew[k][i] /= sum;
        cN[0][i] = 0;
        for (int k = 1; k <= NS; ++k) {
            cN[k][i] = wNew[k - 1][i] * cs.rho[0][i] / mx.M[k - 1];
            cN[0][i] += cN[k][i];
        }
    }
    std::vector<double> CCVNew(nc), oldEnergy(nc);
    for (long long i = 0; i < nc; ++i) {
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) cc[k] = cN[k][i];
        CCVNew[i] = dCv(mx, cc) * cN[0][i];
        const double nonIdNew = dNonIdeality(mx, cc);
        oldEnergy[i] = CCVOld[i] * T[i] + nonIdOld[i] - nonIdNew;
    }

    // the implicit solver with an enthalpy flow: the flow again with the new concentrations, and
    // its 0.5 average with the first (Diffusion.cpp:618-686)
    if (gs && cf.enthalpy_flow != FV_ENTHALPY_NO) {
        std::vector<std::vector<double>> scN(NS + 1, std::vector<double>(nf, 0.0));
        for (int k = 1; k <= NS; ++k) {
            std::vector<double> sk;
            dInterp(cs, cN[k], [&](size_t f) {
                return bcSurfaceS(cs, cN[k][cs.faces[f].own], 0, k - 1, cs.faces[f].patch);
            }, sk);
            for (size_t f = 0; f < nf; ++f) {
                scN[k][f] = sk[f];
                scN[0][f] += sk[f];
            }
        }
        std::vector<std::vector<V3>> DFluxN(NS, std::vector<V3>(nf, v3(0, 0, 0)));
        if (cf.molmass_diffusion && NS > 1) {
            std::vector<std::vector<V3>> gradXN(NS);
            for (int k = 0; k < NS; ++k) {
                std::vector<double> X(nc);
                for (long long i = 0; i < nc; ++i) X[i] = cN[k + 1][i] / cN[0][i];
                dSurfGrad(cs, X, [&](size_t f) {  // calculatedMolarFraction of the phase (cell)
                    double cB[FV_MAX_SPECIES + 1];
                    dBoundaryConc(cs, cs.faces[f].own, cs.faces[f].patch, true, cB, bad);
                    double sum = 0;
                    for (int q = 1; q <= NS; ++q) sum += cB[q];
                    return cB[k + 1] / sum;
                }, gradXN[k]);
            }
            for (size_t f = 0; f < nf; ++f) {
                double Nc[FV_MAX_SPECIES + 1];
                for (int k = 0; k <= NS; ++k) Nc[k] = scN[k][f];
                for (int d = 0; d < 3; ++d) {
                    double g[FV_MAX_SPECIES], out[FV_MAX_SPECIES];
                    for (int k = 0; k < NS; ++k) g[k] = gradXN[k][f].x[d];
                    dMaxwellStefan(NS, Nc, mx.M, trF[f].Dm, g, out);
                    for (int k = 0; k < NS; ++k) DFluxN[k][f].x[d] = out[k];
                }
            }
        }
        std::vector<V3> afDif(nf, v3(0, 0, 0));
        for (int k = 0; k < NS; ++k)
            for (size_t f = 0; f < nf; ++f) {
                const V3 flowW = vmul(gradW[k][f], -1 * rhoD[k][f]);
                const V3 corr = cf.molmass_diffusion ? vsub(DFluxN[k][f], flowW) : v3(0, 0, 0);
                const double h = dhkT(mx, scN[k + 1][f], surfaceT[f], k);
                afDif[f] = vadd(afDif[f], vdiv(vmul(vadd(corr, flowW), h), mx.M[k]));
            }
        for (size_t f = 0; f < nf; ++f) entFlow[f] = vadd(vmul(afDif[f], 0.5), vmul(entFlow[f], 1 - 0.5));
    }

    // velocity and temperature matrices (Diffusion.cpp:480-500; SLEMatrix.cpp:2054-2110
    // explicit, :410-546 and :706-907 implicit)
    std::vector<V3> freeV(nc, v3(0, 0, 0)), oldV(nc);
    SLE1 MV[3];
    for (long long i = 0; i < nc; ++i) oldV[i] = vmul(v[i], cs.rho[0][i]);
    if (gs) {
        for (int d = 0; d < 3; ++d) {
            std::vector<double> rOld(nc);
            for (long long i = 0; i < nc; ++i) rOld[i] = oldV[i].x[d];
            std::vector<double> muF(nf);
            for (size_t f = 0; f < nf; ++f) muF[f] = trF[f].mu;
            dLaplacian(cs, [&, d](long long i, int fi) {
                return bcCellV(cs, v[i], cs.faces[fi].patch, cs.faces[fi].N, bad).x[d];
            }, rOld, cs.rho[0], muF, dt, MV[d]);
            for (long long i = 0; i < nc; ++i) freeV[i].x[d] = MV[d].free[i];
        }
    } else {
        std::vector<T9> flow(nf);
        for (size_t f = 0; f < nf; ++f) flow[f] = tmul(tmul(gradVs[f], trF[f].mu), -1.);
        std::vector<V3> div;
        dDivT(cs, flow, div);
        for (long long i = 0; i < nc; ++i)
            for (int d = 0; d < 3; ++d) freeV[i].x[d] -= div[i].x[d];
    }
    std::vector<double> freeT(nc, 0.0), diagT(CCVNew);
    SLE1 MT;
    {
        auto ghostT = [&](size_t f) { return dBoundaryT(cs, cs.faces[f].own, cs.faces[f].patch, true, bad); };
        if (gs) {
            std::vector<double> kF(nf);
            for (size_t f = 0; f < nf; ++f) kF[f] = trF[f].kappa;
            dLaplacian(cs, [&](long long, int fi) { return ghostT(fi); }, oldEnergy, CCVNew, kF, dt, MT);
            diagT = MT.diag;
            freeT = MT.free;
        } else {
            std::vector<V3> gT;
            dSurfGrad(cs, T, ghostT, gT);
            std::vector<V3> flow(nf);
            for (size_t f = 0; f < nf; ++f) flow[f] = vmul(vmul(gT[f], trF[f].kappa), -1.);
            std::vector<double> div;
            dDivV(cs, flow, div);
            for (long long i = 0; i < nc; ++i) freeT[i] -= div[i];
        }
    }
    // explicit deviatoric viscous stress on the velocity (Diffusion.cpp:503-506,600-605)
    {
        std::vector<T9> dev1(nf);
        for (size_t f = 0; f < nf; ++f) dev1[f] = tmul(strainSurf1[f], trF[f].mu);
        std::vector<V3> div;
        dDivT(cs, dev1, div);
        for (long long i = 0; i < nc; ++i)
            for (int d = 0; d < 3; ++d) freeV[i].x[d] += div[i].x[d];
    }
    {
        std::vector<double> div;
        dDivV(cs, nonIdLap, div);
        for (long long i = 0; i < nc; ++i) {
            const double s = div[i] * (-1.0);
            if (s >= 0.) freeT[i] += s;
            else diagT[i] -= s / (T[i] + kStab);
        }
    }
    if (cf.enthalpy_flow == FV_ENTHALPY_EXPLICIT) {  // Diffusion.cpp:688-706
        for (size_t f = 0; f < nf; ++f) entFlow[f] = vmul(entFlow[f], surfaceT[f]);
        std::vector<double> div;
        dDivV(cs, entFlow, div);
        double mn = std::numeric_limits<double>::infinity();
        for (long long i = 0; i < nc; ++i) mn = std::min(mn, CCVOld[i] * T[i] / std::fabs(div[i] + kStab));
        cs.dtSource = cf.dt_coeff_source * mn;
        for (long long i = 0; i < nc; ++i) {
            const double s = div[i] * -1;
            if (s >= 0.) freeT[i] += s;
            else diagT[i] -= s / (T[i] + kStab);
        }
    }
    for (long long i = 0; i < nc; ++i) {  // viscous heating: devPhysVisc && gradV
        const T9 dev = tmul(strainVol[i], muC[i]);
        double dd = 0;
        for (int q = 0; q < 9; ++q) dd += dev.x[q] * gradV[i].x[q];
        freeT[i] += dd;
    }
    if (bad) {
        cs.err = "fixedValueSurface is not a valid cell boundary value";
        return FV_ERR_BOUNDARY;
    }

    // the implicit solves: velocity by components, then temperature (Diffusion.cpp:786-826)
    std::vector<double> vSol[3], TSol;
    if (gs) {
        for (int d = 0; d < 3; ++d) {
            std::vector<double> start(nc);
            for (long long i = 0; i < nc; ++i) {
                start[i] = v[i].x[d];
                MV[d].free[i] = freeV[i].x[d];
            }
            vSol[d] = dSolve(cf, MV[d], start);
        }
        MT.diag = diagT;
        MT.free = freeT;
        if (cf.enthalpy_flow == FV_ENTHALPY_IMPLICIT)  // Diffusion.cpp:820-826
            dAddNabla(cs, [&](long long, int fi) { return dBoundaryT(cs, cs.faces[fi].own, cs.faces[fi].patch, true, bad); },
                      entFlow, MT);
        TSol = dSolve(cf, MT, T);
    }

    // the phase after the stage (Diffusion.cpp:965-1034)
    double Tmin = std::numeric_limits<double>::infinity();
    cs.Tstate.assign(nc, 0.0);
    cs.Tvalid = true;
    for (long long i = 0; i < nc; ++i) {
        V3 vn;
        for (int d = 0; d < 3; ++d) vn.x[d] = gs ? vSol[d][i] : (oldV[i].x[d] + freeV[i].x[d] * dt) / cs.rho[0][i];
        // (the explicit solver with the implicit enthalpy flow solves the temperature with the
        // factory's second solver, a noMatrixSolver: the temperature stays)
        const double Tn = gs ? TSol[i]
                             : (cf.enthalpy_flow == FV_ENTHALPY_IMPLICIT ? T[i] : (oldEnergy[i] + freeT[i] * dt) / diagT[i]);
        Tmin = std::min(Tmin, Tn);
        cs.Tstate[i] = Tn;
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) cc[k] = cN[k][i];
        cs.c[0][i] = cN[0][i];
        for (int k = 1; k <= NS; ++k) {
            cs.c[k][i] = cN[k][i];
            cs.rho[k][i] = cs.c[k][i] * mx.M[k - 1];
        }
        cs.v[i] = vn;
        cs.m[i] = vmul(vn, cs.rho[0][i]);
        cs.Uv[i] = dUvcFromT(mx, cc, Tn) * cs.c[0][i];
        cs.p[i] = mx.pFromUv(cc, cs.Uv[i]);
        const double v2 = vdot(vn, vn);
        cs.E[i] = cs.Uv[i] + cs.rho[0][i] * v2 * 0.5 + 0.0;
    }
    if (cf.diffusion_timestep) {  // Diffusion.cpp:1036-1049
        std::vector<double> maxVal(nf);
        for (size_t f = 0; f < nf; ++f) {  // effectiveTransportCoefficients::maxValue (:172-184)
            double Dmax = trF[f].Ds[0];
            for (int k = 1; k < NS; ++k) Dmax = std::max(Dmax, trF[f].Ds[k]);
            maxVal[f] = std::max(std::max(trF[f].kappa, surfaceRho[f] * Dmax), trF[f].mu);
        }
        double mn = std::numeric_limits<double>::infinity();
        for (long long i = 0; i < nc; ++i) {
            const Cell& c = cs.cells[i];
            double sumDist = 0;
            double dist[6];
            for (int j = 0; j < c.nFaces; ++j) {
                dist[j] = mag3(vsub(faceCentreFrom(i, cs.faces[c.faces[j]]), c.rC));
                sumDist += dist[j];
            }
            double vol = 0;
            for (int j = 0; j < c.nFaces; ++j) vol += maxVal[c.faces[j]] * (1 - dist[j] / sumDist);
            mn = std::min(mn, vol * c.minLS * c.minLS);
        }
        cs.dtSource = std::min(cs.dtSource, 0.5 * cf.dt_coeff_diffusion / mn);
    }
    if (Tmin < 0.) {
        cs.err = "Negative temperature after diffusion.";
        return FV_ERR_NEGATIVE_T;
    }
    return FV_OK;
}

// ---------------------------------------------------------------- chemistry
// Per-cell backward-Euler kinetics in mass fractions: headers/abstractChemicalKinetics.hpp
// (solvers :110-606, tolerances :30-32), the Cl2 mechanism
// src/chemicalReactions/chemicalKineticsChlorumDissociation.cpp:47-70 (matrix), :128-150 (rates),
// :152-273 (integration), :327-353 (two integrations + average), the heat release of
// chemicalKineticsH2Cl2Combustion.cpp:362-389, and bunchOfFields::average
// (templates/bunchOfFields.hpp:166-204).  A+B->2C is new (no reference counterpart) and uses
// the same integrator.

constexpr double kChemTol = 100 * 1E-12;  // convergenceTolerance = 100 * convergenceToleranceGlobal
constexpr double kMassFracTol = 1E-2;     // massFracTolerance

// Sparse per-cell system in the reference's layout: diagonal, per row the left (j < i) and right
// (j > i) entries in list order, free term.
struct ChemSystem {
    int N = 0;
    double D[FV_MAX_SPECIES] = {};
    double A[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
    int nl[FV_MAX_SPECIES] = {}, l[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
    int nr[FV_MAX_SPECIES] = {}, r[FV_MAX_SPECIES][FV_MAX_SPECIES] = {};
    double B[FV_MAX_SPECIES] = {};
};

// abstractChemicalKinetics::normalize: |x| < epsilon -> 0
void chemNormalize(double* x, int N) {
    for (int i = 0; i < N; ++i)
        if (std::abs(x[i]) < std::numeric_limits<double>::epsilon()) x[i] = 0;
}

// matrixDotProduct (:73-104)
void chemDot(const ChemSystem& m, const double* v, double* out) {
    for (int i = 0; i < m.N; ++i) {
        double s = m.D[i] * v[i];
        for (int q = 0; q < m.nl[i]; ++q) s += m.A[i][m.l[i][q]] * v[m.l[i][q]];
        for (int q = 0; q < m.nr[i]; ++q) s += m.A[i][m.r[i][q]] * v[m.r[i][q]];
        out[i] = s;
    }
}

double chemRelDiff(const double* nw, const double* old, int N) {
    double mx = 0;
    for (int i = 0; i < N; ++i) {
        const double d = std::abs((nw[i] - old[i]) / (std::abs(nw[i]) + kStab));
        if (i == 0 || d > mx) mx = d;
    }
    return 100. * mx;
}

double chemSum(const double* a, int N) {
    double s = 0;
    for (int i = 0; i < N; ++i) s += a[i];
    return s;
}

// solveGS (:201-306): symmetric sweeps; false when it does not converge in maxIter iterations
bool chemSolveGS(const ChemSystem& m, const double* init, int maxIter, double* out) {
    const int N = m.N;
    double old[FV_MAX_SPECIES] = {}, nw[FV_MAX_SPECIES] = {};
    for (int i = 0; i < N; ++i) old[i] = nw[i] = init[i];
    int it = 0;
    while (true) {
        ++it;
        for (int i = 0; i < N; ++i) {
            const double aii = 1. / m.D[i];
            nw[i] = m.B[i] * aii;
            for (int q = 0; q < m.nl[i]; ++q) nw[i] -= m.A[i][m.l[i][q]] * nw[m.l[i][q]] * aii;
            for (int q = 0; q < m.nr[i]; ++q) nw[i] -= m.A[i][m.r[i][q]] * old[m.r[i][q]] * aii;
        }
        for (int i = N - 1; i >= 0; --i) {
            const double aii = 1. / m.D[i];
            nw[i] = m.B[i] * aii;
            for (int q = m.nl[i] - 1; q >= 0; --q) nw[i] -= m.A[i][m.l[i][q]] * old[m.l[i][q]] * aii;
            for (int q = m.nr[i] - 1; q >= 0; --q) nw[i] -= m.A[i][m.r[i][q]] * nw[m.r[i][q]] * aii;
        }
        if (chemRelDiff(nw, old, N) < kChemTol) {
            chemNormalize(nw, N);
            for (int i = 0; i < N; ++i) out[i] = nw[i];
            return true;
        }
        if (it >= maxIter) return false;
        for (int i = 0; i < N; ++i) old[i] = nw[i];
    }
}

// solveJ (:110-199)
bool chemSolveJ(const ChemSystem& m, const double* init, int maxIter, double* out) {
    const int N = m.N;
    double old[FV_MAX_SPECIES] = {}, nw[FV_MAX_SPECIES] = {};
    for (int i = 0; i < N; ++i) old[i] = nw[i] = init[i];
    int it = 0;
    while (true) {
        ++it;
        for (int i = 0; i < N; ++i) {
            const double aii = 1. / m.D[i];
            double rs = 0;
            for (int q = 0; q < m.nl[i]; ++q) rs -= m.A[i][m.l[i][q]] * old[m.l[i][q]];
            for (int q = 0; q < m.nr[i]; ++q) rs -= m.A[i][m.r[i][q]] * old[m.r[i][q]];
            nw[i] = (m.B[i] + rs) * aii;
        }
        for (int i = N - 1; i >= 0; --i) {
            const double aii = 1. / m.D[i];
            double rs = 0;
            for (int q = m.nl[i] - 1; q >= 0; --q) rs -= m.A[i][m.l[i][q]] * old[m.l[i][q]];
            for (int q = m.nr[i] - 1; q >= 0; --q) rs -= m.A[i][m.r[i][q]] * old[m.r[i][q]];
            nw[i] = (m.B[i] + rs) * aii;
        }
        if (chemRelDiff(nw, old, N) < kChemTol) {
            chemNormalize(nw, N);
            for (int i = 0; i < N; ++i) out[i] = nw[i];
            return true;
        }
        if (it >= maxIter) return false;
        for (int i = 0; i < N; ++i) old[i] = nw[i];
    }
}

// solveCG (:308-389) and solveJCG (:391-495); jacobi selects the preconditioned form
bool chemSolveCG(const ChemSystem& m, const double* init, int maxIter, bool jacobi, double* out) {
    const int N = m.N;
    double x[FV_MAX_SPECIES] = {}, r[FV_MAX_SPECIES] = {}, d[FV_MAX_SPECIES] = {}, Ad[FV_MAX_SPECIES] = {},
           P[FV_MAX_SPECIES] = {};
    for (int i = 0; i < N; ++i) {
        x[i] = init[i];
        P[i] = 1. / m.D[i];
    }
    chemDot(m, x, Ad);
    for (int i = 0; i < N; ++i) r[i] = m.B[i] - Ad[i];
    for (int i = 0; i < N; ++i) d[i] = jacobi ? P[i] * r[i] : r[i];
    int it = 0;
    while (true) {
        ++it;
        double diff = 0;
        for (int i = 0; i < N; ++i)
            if (i == 0 || std::abs(r[i]) > diff) diff = std::abs(r[i]);
        if (diff < kChemTol && it > 1) {
            chemNormalize(x, N);
            for (int i = 0; i < N; ++i) out[i] = x[i];
            return true;
        }
        if (it >= maxIter) return false;
        double t[FV_MAX_SPECIES] = {};
        chemDot(m, d, Ad);
        for (int i = 0; i < N; ++i) t[i] = jacobi ? r[i] * (P[i] * r[i]) : r[i] * r[i];
        const double rr = chemSum(t, N);
        for (int i = 0; i < N; ++i) t[i] = d[i] * Ad[i];
        const double alpha = rr / (chemSum(t, N) + kStab);
        for (int i = 0; i < N; ++i) x[i] += alpha * d[i];
        double r1[FV_MAX_SPECIES] = {};
        for (int i = 0; i < N; ++i) r1[i] = r[i] - alpha * Ad[i];
        for (int i = 0; i < N; ++i) t[i] = jacobi ? r1[i] * (P[i] * r1[i]) : r1[i] * r1[i];
        const double rr1 = chemSum(t, N);
        const double beta = rr1 / (rr + kStab);
        for (int i = 0; i < N; ++i) d[i] = (jacobi ? P[i] * r1[i] : r1[i]) + beta * d[i];
        for (int i = 0; i < N; ++i) r[i] = r1[i];
    }
}

// solveGE (:497-604): row pivoting on the raw value, then elimination and back substitution
bool chemSolveGE(const ChemSystem& m, double* out) {
    const int N = m.N;
    double A[FV_MAX_SPECIES][FV_MAX_SPECIES] = {}, b[FV_MAX_SPECIES] = {};
    for (int i = 0; i < N; ++i) {
        A[i][i] = m.D[i];
        for (int q = 0; q < m.nl[i]; ++q) A[i][m.l[i][q]] = m.A[i][m.l[i][q]];
        for (int q = 0; q < m.nr[i]; ++q) A[i][m.r[i][q]] = m.A[i][m.r[i][q]];
        b[i] = m.B[i];
    }
    for (int k = 0; k < N - 1; ++k) {
        double mv = A[k][k];
        int c = k;
        for (int q = k + 1; q < N; ++q)
            if (A[q][k] > mv) { mv = A[q][k]; c = q; }
        if (c != k) {
            for (int j = 0; j < N; ++j) std::swap(A[c][j], A[k][j]);
            std::swap(b[c], b[k]);
        }
    }
    for (int k = 0; k < N - 1; ++k)
        for (int i = k + 1; i < N; ++i) {
            const double ratio = A[i][k] / (A[k][k] + kStab);
            for (int j = k + 1; j < N; ++j) A[i][j] = A[i][j] - ratio * A[k][j];
            b[i] = b[i] - ratio * b[k];
        }
    double phi[FV_MAX_SPECIES] = {};
    phi[N - 1] = b[N - 1] / (A[N - 1][N - 1] + kStab);
    for (int i = N - 2; i >= 0; --i) {
        double term = 0.0;
        for (int j = i + 1; j < N; ++j) term += A[i][j] * phi[j];
        phi[i] = (b[i] - term) / (A[i][i] + kStab);
    }
    chemNormalize(phi, N);
    for (int i = 0; i < N; ++i) out[i] = phi[i];
    return true;
}

bool chemSolve(const fv_config& cf, const ChemSystem& m, const double* init, double* out) {
    switch (cf.chem_solver) {
    case FV_CHEM_JACOBI: return chemSolveJ(m, init, cf.chem_max_iter, out);
    case FV_CHEM_GAUSS_ELIMINATION: return chemSolveGE(m, out);
    case FV_CHEM_CONJUGATE_GRADIENT: return chemSolveCG(m, init, cf.chem_max_iter, false, out);
    case FV_CHEM_JACOBI_CONJUGATE_GRADIENT: return chemSolveCG(m, init, cf.chem_max_iter, true, out);
    default: return chemSolveGS(m, init, cf.chem_max_iter, out);
    }
}

// k = A T^n exp(-E / (R T)) (chemicalKineticsChlorumDissociation.cpp:133-137)
double arrhenius(const fv_arrhenius& k, double T, double R) { return k.A * std::pow(T, k.n) * std::exp(-k.E / (R * T)); }

// Mechanism matrix of one sub-step in mass fractions, with the concentrations c[0..N] of the
// sub-step's start, the cell's temperature of the integration T and mixture density rho.
void chemSystem(const fv_config& cf, const Mix& mx, double dt, double T, const double* c, double rho,
                ChemSystem& m) {
    m = ChemSystem();
    m.N = mx.N;
    if (cf.chemistry == FV_CHEM_CL2) {
        // setMatrix (chemicalKineticsChlorumDissociation.cpp:47-70)
        const double kd = arrhenius(cf.chem_forward, T, mx.R), kr = arrhenius(cf.chem_backward, T, mx.R);
        const double Cl2 = c[1], Cl = c[2], M0 = c[0];
        m.D[0] = (1 / dt + kd * M0) / mx.M[0];
        m.A[0][1] = (-kr * Cl * M0) / mx.M[1];
        m.B[0] = Cl2 / (rho * dt);
        m.A[1][0] = (-2 * kd * M0) / mx.M[0];
        m.D[1] = (1 / dt + 2 * kr * Cl * M0) / mx.M[1];
        m.B[1] = Cl / (rho * dt);
        m.nr[0] = 1; m.r[0][0] = 1;
        m.nl[1] = 1; m.l[1][0] = 0;
    } else {
        // A + B -> 2C: rate k c_A c_B linearised as k c_B^old c_A^new (A) and k c_A^old c_B^new (B);
        // C is produced by the mass of both, so the system conserves mass for any molar masses
        const double k = arrhenius(cf.chem_forward, T, mx.R);
        const double cA = c[1], cB = c[2], cC = c[3];
        m.D[0] = (1 / dt + k * cB) / mx.M[0];
        m.B[0] = cA / (rho * dt);
        m.D[1] = (1 / dt + k * cA) / mx.M[1];
        m.B[1] = cB / (rho * dt);
        m.A[2][0] = (-k * cB) / mx.M[2];
        m.A[2][1] = (-k * cA) / mx.M[2];
        m.D[2] = (1 / dt) / mx.M[2];
        m.B[2] = cC / (rho * dt);
        m.nl[2] = 2; m.l[2][0] = 0; m.l[2][1] = 1;
    }
}

struct ChemCell {
    double Uv, T;
    double c[FV_MAX_SPECIES + 1];
    double dens[FV_MAX_SPECIES];
};

// timeStepIntegration for one cell (chemicalKineticsChlorumDissociation.cpp:152-273).  subIt is the
// sub-step count, carried from cell to cell like the reference's serial loop.  Returns FV_OK or
// the error of an exhausted sub-cycling.
int chemIntegrate(const fv_config& cf, const Mix& mx, double dt, double rho, ChemCell& cell, long long& subIt) {
    const int N = mx.N;
    const ChemCell oldV = cell;
    const double Tcell = oldV.T;
    double subDt = dt / subIt;
    ChemCell nv = oldV;
    while (true) {
        bool ok = true;
        nv = oldV;
        for (long long st = 0; st < subIt && ok; ++st) {
            double wOld[FV_MAX_SPECIES] = {};
            for (int k = 0; k < N; ++k) wOld[k] = nv.dens[k] / rho;
            double sumOld = 0.;
            for (int k = 0; k < N; ++k) sumOld = sumOld + wOld[k];
            if (sumOld == 0.0) continue;
            ChemSystem m;
            chemSystem(cf, mx, subDt, Tcell, nv.c, rho, m);
            double w[FV_MAX_SPECIES] = {};
            if (!chemSolve(cf, m, wOld, w)) { ok = false; break; }
            for (int k = 0; k < N; ++k) w[k] = std::max(0., w[k]);
            double sumNew = 0.;
            for (int k = 0; k < N; ++k) sumNew = sumNew + w[k];
            if (std::abs(sumNew - sumOld) > kMassFracTol) { ok = false; break; }
            for (int k = 0; k < N; ++k) {
                w[k] /= sumNew;
                w[k] *= sumOld;
            }
            double deltaU = 0;
            if (cf.chemistry == FV_CHEM_A_B_2C) {
                // heat release per mol of C formed: (q - dCv (T - 298.15)) / 2 (the form of
                // chemicalKineticsH2Cl2Combustion.cpp:362-389 for a reaction forming 2 C)
                const double deltaC = w[2] * rho / mx.M[2] - nv.c[3];
                const double deltaCv = 2 * mx.Cv[2] - mx.Cv[0] - mx.Cv[1];
                deltaU = (cf.chem_q - deltaCv * (Tcell - 298.15)) * 0.5 * deltaC;
            }
            for (int k = 0; k < N; ++k) nv.c[k + 1] = w[k] * rho / mx.M[k];
            nv.c[0] = 0;
            for (int k = 1; k <= N; ++k) nv.c[0] += nv.c[k];
            nv.Uv += deltaU;
            nv.T = mx.TFromUv(nv.c, nv.Uv);
            if (nv.T < 0) { ok = false; break; }
            for (int k = 0; k < N; ++k) nv.dens[k] = nv.c[k + 1] * mx.M[k];
        }
        if (ok) break;
        subIt *= 10;
        subDt = dt / subIt;
        if (subDt < cf.min_timestep) return FV_ERR_SYSTEM;
    }
    cell = nv;
    return FV_OK;
}

// solveChemicalKinetics (chemicalKineticsChlorumDissociation.cpp:327-353) over all cells.
int chemistryStep(fvo_case& cs, double dt) {
    const Mix& mx = cs.mix;
    const int N = mx.N;
    const long long nc = cs.nCells;
    std::vector<ChemCell> cells(nc);
    for (long long i = 0; i < nc; ++i) {
        ChemCell& q = cells[i];
        for (int k = 0; k <= N; ++k) q.c[k] = cs.c[k][i];
        for (int k = 0; k < N; ++k) q.dens[k] = cs.rho[k + 1][i];
        q.Uv = cs.Uv[i];
        // the phase's temperature: the diffusion stage's when it ran (secondOrderStepSolver.cpp:
        // 69-91), else TFromUv of the advected energy
        q.T = cs.Tvalid ? cs.Tstate[i] : mx.TFromUv(q.c, q.Uv);
    }
    for (int pass = 0; pass < 2; ++pass) {
        long long subIt = 1;
        for (long long i = 0; i < nc; ++i) {
            if (!cs.chemCarry) subIt = 1;  // per-cell sub-cycling (the CUDA path's behaviour)
            const int st = chemIntegrate(cs.cfg, mx, dt, cs.rho[0][i], cells[i], subIt);
            if (st != FV_OK) {
                cs.err = "Timestep become too small.";
                return st;
            }
        }
    }
    for (long long i = 0; i < nc; ++i) {
        const ChemCell& q = cells[i];
        const double v2 = vdot(cs.v[i], cs.v[i]);
        const double E1 = q.Uv + cs.rho[0][i] * v2 * 0.5 + 0.0;
        // bunchOfFields::average(phaseN1, 0.5)
        for (int k = 0; k <= N; ++k) cs.c[k][i] = 0.5 * cs.c[k][i] + 0.5 * q.c[k];
        for (int k = 1; k <= N; ++k) cs.rho[k][i] = 0.5 * cs.rho[k][i] + 0.5 * q.dens[k - 1];
        cs.rho[0][i] = 0.5 * cs.rho[0][i] + 0.5 * cs.rho[0][i];
        cs.m[i] = vadd(vmul(cs.m[i], 0.5), vmul(cs.m[i], 0.5));
        cs.E[i] = 0.5 * cs.E[i] + 0.5 * E1;
        cs.v[i] = vdiv(cs.m[i], cs.rho[0][i]);
        cs.Uv[i] = cs.E[i] - 0.0 - 0.5 * cs.rho[0][i] * vdot(cs.v[i], cs.v[i]);
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= N; ++k) cc[k] = cs.c[k][i];
        cs.p[i] = mx.pFromUv(cc, cs.Uv[i]);
    }
    cs.Tvalid = false;  // bunchOfFields::average: T = TFromUv (bunchOfFields.hpp:197-198)
    return FV_OK;
}

// main's CFL block (Schemi.cpp:807-833); it consumes the source time step a diffusion stage set
double cflTimestep(fvo_case& cs) {
    double maxS = -std::numeric_limits<double>::infinity();
    for (long long i = 0; i < cs.nCells; ++i) {
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= cs.N; ++k) cc[k] = cs.c[k][i];
        const double sonic = std::sqrt(cs.mix.sqSonicSpeed(cc, cs.rho[0][i], cs.Uv[i], cs.p[i]));
        double s = mag3(cs.v[i]) + sonic;
        s *= cs.cells[i].minLS;
        maxS = std::max(maxS, s);
    }
    double dt = cs.cfg.courant / maxS;
    cs.dtSourceLast = cs.dtSource;
    if (!cs.cfg.courant_only) dt = std::min(dt, cs.dtSource);
    dt = std::max(dt, cs.cfg.min_timestep);
    if (cs.cfg.const_timestep <= 0) cs.dtSource = kVeryBig;
    if (cs.cfg.const_timestep > 0) dt = cs.cfg.const_timestep;  // no CFL block (Schemi.cpp:807)
    return dt;
}

bool validate(const fv_config& cf, std::string& err) {
    if (cf.dims < 1 || cf.dims > 3) { err = "dims must be 1, 2 or 3"; return false; }
    for (int d = 0; d < cf.dims; ++d)
        if (cf.n[d] < 1) { err = "cell counts must be positive"; return false; }
    if (cf.n_species < 1 || cf.n_species > FV_MAX_SPECIES) { err = "n_species out of range"; return false; }
    if (cf.eos < FV_EOS_IDEAL || cf.eos > FV_EOS_KATAOKA) { err = "unknown equation of state"; return false; }
    if (cf.flux != FV_FLUX_HLLC && cf.flux != FV_FLUX_HLL) { err = "unknown flux solver"; return false; }
    if (cf.limiter < 0 || cf.limiter > FV_LIM_SCHMIDTMANN) { err = "unknown limiter"; return false; }
    if (cf.chemistry == FV_CHEM_CL2 && cf.n_species != 2) { err = "Cl2 dissociation needs 2 species"; return false; }
    if (cf.chemistry == FV_CHEM_A_B_2C && cf.n_species != 3) { err = "A+B->2C needs 3 species"; return false; }
    if (cf.chemistry < FV_CHEM_NONE || cf.chemistry > FV_CHEM_CL2) { err = "unknown chemistry"; return false; }
    if (cf.chemistry != FV_CHEM_NONE && cf.eos != FV_EOS_IDEAL && cf.eos != FV_EOS_VAN_DER_WAALS) {
        err = "chemistry runs with ideal and van der Waals mixtures";
        return false;
    }
    if (cf.order < FV_ORDER_SECOND || cf.order > FV_ORDER_THIRD_CADA) {
        err = "unknown step solver";
        return false;
    }
    if (cf.diffusion) {
        if (cf.order != FV_ORDER_SECOND) { err = "the diffusion stage runs with the SecondOrder step"; return false; }
        if (cf.flux != FV_FLUX_HLLC) { err = "the diffusion stage runs with the HLLC flux"; return false; }
        if (cf.eos != FV_EOS_IDEAL && cf.eos != FV_EOS_VAN_DER_WAALS) {
            err = "the diffusion stage runs with ideal and van der Waals mixtures";
            return false;
        }
        if (cf.sle_solver < FV_SLE_EXPLICIT || cf.sle_solver > FV_SLE_BICG) {
            err = "unknown matrix solver";
            return false;
        }
        if (cf.sle_solver == FV_SLE_THOMAS && (cf.dims != 1 || cf.n[0] < 2)) {
            err = "the Thomas solver runs on 1D meshes of at least 2 cells";
            return false;
        }
        if (cf.transport < FV_TRANSPORT_CONSTANT || cf.transport > FV_TRANSPORT_LENNARD_JONES) {
            err = "unknown transport model";
            return false;
        }
        for (int k = 0; k < cf.n_species; ++k) {
            if (cf.transport == FV_TRANSPORT_HARD_SPHERES && !(cf.transport_diameter[k] > 0)) {
                err = "hard-sphere diameters must be positive";
                return false;
            }
            if (cf.transport == FV_TRANSPORT_LENNARD_JONES &&
                !(cf.transport_lj_eps[k] > 0 && cf.transport_lj_sigma[k] > 0)) {
                err = "Lennard-Jones parameters must be positive";
                return false;
            }
        }
        if (cf.enthalpy_flow < FV_ENTHALPY_NO || cf.enthalpy_flow > FV_ENTHALPY_IMPLICIT) {
            err = "unknown enthalpy flow flag";
            return false;
        }
    }
    return true;
}

}  // namespace

extern "C" {

fvo_case* fvo_create(const fv_config* cfg, char* err, int err_len) {
    std::string e;
    if (!cfg || !validate(*cfg, e)) {
        if (err && err_len > 0) snprintf(err, err_len, "%s", e.c_str());
        return nullptr;
    }
    fvo_case* cs = new fvo_case();
    cs->cfg = *cfg;
    cs->N = cfg->n_species;
    cs->D = cfg->dims;
    buildMesh(*cs);
    Mix& mx = cs->mix;
    mx.N = cs->N;
    mx.eos = cfg->eos;
    mx.R = cfg->R;
    for (int k = 0; k < mx.N; ++k) {
        mx.M[k] = cfg->M[k];
        mx.Cv[k] = cfg->Cv[k];
    }
    if (cfg->eos == FV_EOS_VAN_DER_WAALS) {
        // mixtureVanDerWaals.cpp:33-52
        for (int k = 0; k < mx.N; ++k) {
            mx.b[k][k] = cfg->Tc[k] * mx.R / (8 * cfg->Pc[k]);
            mx.a[k][k] = cfg->Pc[k] * mx.b[k][k] * mx.b[k][k] * 27;
        }
        for (int k = 0; k < mx.N; ++k)
            for (int l = 0; l < mx.N; ++l)
                if (k != l) {
                    mx.b[k][l] = std::pow(0.5 * (std::cbrt(mx.b[k][k]) + std::cbrt(mx.b[l][l])), 3);
                    mx.a[k][l] = std::sqrt(mx.a[k][k] * mx.a[l][l]);
                }
    } else if (cfg->eos == FV_EOS_REDLICH_KWONG) {
        // mixtureRedlichKwong.cpp:34-60 (the constants folded at compile time, as g++ does there)
        constexpr double chi{std::cbrt(2) - 1.};
        constexpr double Sigma_a{1. / (9. * chi)}, Sigma_b{chi / 3.};
        for (int k = 0; k < mx.N; ++k) {
            mx.b[k][k] = Sigma_b * mx.R * cfg->Tc[k] / cfg->Pc[k];
            mx.a[k][k] = Sigma_a * mx.R * mx.R * cfg->Tc[k] * cfg->Tc[k] * std::sqrt(cfg->Tc[k]) / cfg->Pc[k];
        }
        for (int k = 0; k < mx.N; ++k)
            for (int l = 0; l < mx.N; ++l)
                if (k != l) {
                    mx.b[k][l] = std::pow(0.5 * (std::cbrt(mx.b[k][k]) + std::cbrt(mx.b[l][l])), 3);
                    mx.a[k][l] = std::sqrt(mx.a[k][k] * mx.a[l][l]);
                }
    } else if (cfg->eos == FV_EOS_STIFFENED) {
        // mixtureStiffened.cpp:19-42
        for (int k = 0; k < mx.N; ++k) {
            mx.p0[k][k] = cfg->stiff_p0[k];
            mx.gam[k][k] = cfg->stiff_gamma[k];
        }
        for (int k = 0; k < mx.N; ++k)
            for (int l = 0; l < mx.N; ++l)
                if (k != l) {
                    mx.p0[k][l] = std::sqrt(mx.p0[k][k] * mx.p0[l][l]);
                    mx.gam[k][l] = std::sqrt(mx.gam[k][k] * mx.gam[l][l]);
                }
    } else if (cfg->eos == FV_EOS_KATAOKA) {
        // mixtureKataokaVanDerWaals.cpp:20-75
        constexpr double NA = 6.02214076E23;  // globalConstants.hpp NAvogardro
        for (int k = 0; k < mx.N; ++k) {
            const double sg = cfg->lj_sigma[k];
            mx.b[k][k] = cfg->kataoka_b_critical ? cfg->kataoka_b_coeff * mx.R * cfg->Tc[k] / (8 * cfg->Pc[k])
                                                 : cfg->kataoka_b_coeff * (sg * sg * sg) * NA;
            mx.V0[k][k] = (sg * sg * sg) / std::sqrt(2) * NA;
            mx.eps[k][k] = cfg->lj_eps[k];
        }
        for (int k = 0; k < mx.N; ++k)
            for (int l = 0; l < mx.N; ++l)
                if (k != l) {
                    mx.b[k][l] = std::pow(0.5 * (std::cbrt(mx.b[k][k]) + std::cbrt(mx.b[l][l])), 3);
                    mx.V0[k][l] = std::pow(0.5 * (std::cbrt(mx.V0[k][k]) + std::cbrt(mx.V0[l][l])), 3);
                    mx.eps[k][l] = std::sqrt(mx.eps[k][k] * mx.eps[l][l]);
                }
    }
    for (int k = 0; k <= cs->N; ++k) {
        cs->c[k].assign(cs->nCells, 0.0);
        cs->rho[k].assign(cs->nCells, 0.0);
    }
    cs->v.assign(cs->nCells, v3(0, 0, 0));
    cs->m.assign(cs->nCells, v3(0, 0, 0));
    cs->E.assign(cs->nCells, 0.0);
    cs->Uv.assign(cs->nCells, 0.0);
    cs->p.assign(cs->nCells, 0.0);
    cs->g = v3(cfg->g[0], cfg->g[1], cfg->g[2]);
    cs->dt = cfg->const_timestep > 0 ? cfg->const_timestep : cfg->min_timestep;
    return cs;
}

void fvo_destroy(fvo_case* c) { delete c; }

long long fvo_n_cells(const fvo_case* c) { return c ? c->nCells : 0; }

int fvo_set_chem_carry(fvo_case* c, int carry) {
    if (!c) return FV_ERR_INIT;
    c->chemCarry = carry ? 1 : 0;
    return FV_OK;
}

int fvo_upload(fvo_case* cs, const double* const* prim) {
    cs->Tvalid = false;
    const int NS = cs->N;
    const Mix& mx = cs->mix;
    for (long long i = 0; i < cs->nCells; ++i) {
        // phaseInitialization.cpp:1827-1885
        cs->c[0][i] = 0;
        for (int k = 1; k <= NS; ++k) {
            cs->c[k][i] = prim[k - 1][i];
            cs->c[0][i] += cs->c[k][i];
        }
        for (int k = 1; k <= NS; ++k) cs->rho[k][i] = cs->c[k][i] * mx.M[k - 1];
        cs->rho[0][i] = 0;
        for (int k = 1; k <= NS; ++k) cs->rho[0][i] += cs->rho[k][i];
        cs->v[i] = v3(prim[NS][i], prim[NS + 1][i], prim[NS + 2][i]);
        cs->p[i] = prim[NS + 3][i];
        cs->m[i] = vmul(cs->v[i], cs->rho[0][i]);
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) cc[k] = cs->c[k][i];
        cs->Uv[i] = mx.UvFromp(cc, cs->p[i]);
        const double v2 = vdot(cs->v[i], cs->v[i]);
        cs->E[i] = cs->Uv[i] + cs->rho[0][i] * v2 * 0.5 + 0.0;
    }
    cs->time = 0;
    cs->dt = cs->cfg.const_timestep > 0 ? cs->cfg.const_timestep : cs->cfg.min_timestep;
    cs->g = v3(cs->cfg.g[0], cs->cfg.g[1], cs->cfg.g[2]);
    return FV_OK;
}

int fvo_step(fvo_case* cs, double* dt_used, double* dt_next) {
    const double dt = cs->dt;
    const int order = cs->cfg.order;
    int st = order == FV_ORDER_SECOND_RK                                     ? rk2Step(*cs, dt)
             : (order == FV_ORDER_THIRD || order == FV_ORDER_THIRD_CADA) ? rk3Step(*cs, dt, order == FV_ORDER_THIRD_CADA)
                                                                         : doStep(*cs, dt);
    if (st != FV_OK) return st;
    if (cs->cfg.diffusion) {
        // the diffusion stage after the advection (secondOrderStepSolver.cpp:69-80)
        st = diffusionStage(*cs, dt);
        if (st != FV_OK) return st;
    }
    if (cs->cfg.chemistry != FV_CHEM_NONE) {
        // chemistry after the advection (and after the multi-stage average), same dt:
        // secondOrderStepSolver.cpp:87-91, secondOrderStepSolverRK.cpp:114-118,
        // thirdOrderStepSolver.cpp:125-129
        st = chemistryStep(*cs, dt);
        if (st != FV_OK) return st;
    }
    if (cs->cfg.gravity) {
        cs->g = vadd(cs->g, vmul(v3(cs->cfg.g_delta[0], cs->cfg.g_delta[1], cs->cfg.g_delta[2]), dt));
    }
    cs->time += dt;
    cs->dt = cflTimestep(*cs);
    if (cs->mix.failed) {
        // cubicEquationSolver.cpp / returnSinglePosValue throw: the run stops
        cs->mix.failed = false;
        return FV_ERR_POSITIVENESS;
    }
    if (dt_used) *dt_used = dt;
    if (dt_next) *dt_next = cs->dt;
    return FV_OK;
}

int fvo_run(fvo_case* cs, double t_end, long long max_steps, double* time, long long* steps) {
    long long n = 0;
    cs->dt = std::min(cs->dt, t_end);
    int st = FV_OK;
    do {
        if (n >= max_steps) break;
        st = fvo_step(cs, nullptr, nullptr);
        if (st != FV_OK) break;
        ++n;
        if ((cs->time + cs->dt) > t_end) cs->dt = t_end - cs->time;
    } while (cs->time < t_end);
    if (time) *time = cs->time;
    if (steps) *steps = n;
    return st;
}

int fvo_download(fvo_case* cs, double* const* out) {
    const int NS = cs->N;
    const Mix& mx = cs->mix;
    for (long long i = 0; i < cs->nCells; ++i) {
        double cc[FV_MAX_SPECIES + 1];
        for (int k = 0; k <= NS; ++k) cc[k] = cs->c[k][i];
        for (int k = 0; k < NS; ++k)
            if (out[FV_F_CONC + k]) out[FV_F_CONC + k][i] = cs->c[k + 1][i];
        if (out[FV_F_VX]) out[FV_F_VX][i] = cs->v[i].x[0];
        if (out[FV_F_VY]) out[FV_F_VY][i] = cs->v[i].x[1];
        if (out[FV_F_VZ]) out[FV_F_VZ][i] = cs->v[i].x[2];
        if (out[FV_F_P]) out[FV_F_P][i] = cs->p[i];
        for (int k = 0; k < NS; ++k)
            if (out[FV_F_RHO_K + k]) out[FV_F_RHO_K + k][i] = cs->rho[k + 1][i];
        if (out[FV_F_RHO]) out[FV_F_RHO][i] = cs->rho[0][i];
        if (out[FV_F_MX]) out[FV_F_MX][i] = cs->m[i].x[0];
        if (out[FV_F_MY]) out[FV_F_MY][i] = cs->m[i].x[1];
        if (out[FV_F_MZ]) out[FV_F_MZ][i] = cs->m[i].x[2];
        if (out[FV_F_E]) out[FV_F_E][i] = cs->E[i];
        if (out[FV_F_UV]) out[FV_F_UV][i] = cs->Uv[i];
        if (out[FV_F_T]) out[FV_F_T][i] = cs->Tvalid ? cs->Tstate[i] : mx.TFromUv(cc, cs->Uv[i]);
        if (out[FV_F_SONIC]) out[FV_F_SONIC][i] = std::sqrt(mx.sqSonicSpeed(cc, cs->rho[0][i], cs->Uv[i], cs->p[i]));
        if (out[FV_F_CONC0]) out[FV_F_CONC0][i] = cs->c[0][i];
    }
    return FV_OK;
}

int fvo_get_time(const fvo_case* cs, double* time, double* dt) {
    if (time) *time = cs->time;
    if (dt) *dt = cs->dt;
    return FV_OK;
}

int fvo_get_source_timestep(const fvo_case* cs, double* dt_source) {
    if (dt_source) *dt_source = cs->dtSourceLast;
    return FV_OK;
}

int fvo_set_time(fvo_case* cs, double time, double dt) {
    cs->time = time;
    cs->dt = dt;
    return FV_OK;
}

int fvo_get_conserved(const fvo_case* cs, double* const* out) {
    const int NS = cs->N;
    for (long long i = 0; i < cs->nCells; ++i) {
        for (int k = 0; k < NS; ++k) out[k][i] = cs->rho[k + 1][i];
        out[NS][i] = cs->rho[0][i];
        for (int d = 0; d < 3; ++d) out[NS + 1 + d][i] = cs->m[i].x[d];
        out[NS + 4][i] = cs->E[i];
    }
    return FV_OK;
}

int fvo_set_conserved(fvo_case* cs, const double* const* in) {
    cs->Tvalid = false;
    const int NS = cs->N;
    for (long long i = 0; i < cs->nCells; ++i) {
        for (int k = 0; k < NS; ++k) cs->rho[k + 1][i] = in[k][i];
        cs->rho[0][i] = in[NS][i];
        for (int d = 0; d < 3; ++d) cs->m[i].x[d] = in[NS + 1 + d][i];
        cs->E[i] = in[NS + 4][i];
        cellPrimitivesFromConserved(*cs, i);
    }
    return FV_OK;
}

}  // extern "C"
