// fv_device.cuh -- device-side physics of the explicit finite-volume step.
//
// Point functions of the reference's step, written for registers: mixture EOS, limiter
// functions, face-state closures, boundary ghost values and the HLLC / HLL fluxes.  Each
// expression keeps the reference's operation order (paths inside the Schemi project):
//   EOS          src/thermodynamics/mixtureIdeal.cpp, idealFluid.cpp:13-60,
//                mixtureVanDerWaals.cpp:88-146,309-397, vanDerWaalsFluid.cpp:14-75
//   limiters     src/limiters/<name>Limiter.cpp
//   closures     src/Advections/Advection.cpp:238-387, HancockStage.cpp:177-306
//   ghosts       headers/boundaryConditionValue.hpp:279-300, src/boundary/slipFunction.cpp:21-25
//   HLLC / HLL   src/RiemannSolvers/HLLCSolver.cpp:52-403, HLLSolver.cpp:52-300
// so that the FP64 instantiation, compiled without FMA contraction, reproduces the reference
// bit for bit.  The FP32 instantiation is the "FP32 flux" arithmetic of the fast path.
//
// Normals of the structured mesh are exact signed unit vectors along an axis, so a normal is
// carried as (axis, sign) and v & N reduces to sign * v[axis] exactly.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/fvstep.h"

namespace fv {

constexpr int MAXS = FV_MAX_SPECIES;

// constants of globalConstants.hpp:22-35
__host__ __device__ constexpr double kStabD() { return 5 * 2.220446049250313080847e-16; }
__host__ __device__ constexpr double kVeryBigD() { return 1E-3 * 1.7976931348623157e308; }

template <typename T> struct Num;
template <> struct Num<double> {
    __device__ static double stab() { return kStabD(); }
    __device__ static double sqrt_(double x) { return sqrt(x); }
    __device__ static double abs_(double x) { return fabs(x); }
};
template <> struct Num<float> {
    __device__ static float stab() { return 5.0f * 1.1920929e-07f; }
    __device__ static float sqrt_(float x) { return sqrtf(x); }
    __device__ static float abs_(float x) { return fabsf(x); }
};

// std::min / std::max semantics (first argument wins ties and unordered comparisons)
template <typename T> __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }

// Scaled 3-argument hypot with the semantics of the reference build's std::hypot(x, y, z).
template <typename T> __device__ __forceinline__ T mag3(T x, T y, T z) {
    x = Num<T>::abs_(x); y = Num<T>::abs_(y); z = Num<T>::abs_(z);
    const T a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == T(0)) return T(0);
    const T xa = x / a, ya = y / a, za = z / a;
    return a * Num<T>::sqrt_(xa * xa + ya * ya + za * za);
}

// mag3(x, y, 0): the same value without the third quotient (0 / a = 0 exactly).
template <typename T> __device__ __forceinline__ T mag2z(T x, T y) {
    x = Num<T>::abs_(x); y = Num<T>::abs_(y);
    const T a = x < y ? y : x;
    if (a == T(0)) return T(0);
    const T xa = x / a, ya = y / a;
    return a * Num<T>::sqrt_(xa * xa + ya * ya + T(0));
}

// ------------------------------------------------------------------ mixture parameters
struct MixParams {
    int ns;        // number of species
    int eos_kind;  // fv_eos
    double R;
    double M[MAXS];
    double invM[MAXS];  // 1 / M (FP32-flux arithmetic only)
    double Cv[MAXS];
    double a[MAXS][MAXS];   // van der Waals / Redlich-Kwong a
    double b[MAXS][MAXS];   // van der Waals / Redlich-Kwong / Kataoka b
    double p0[MAXS][MAXS];  // stiffened p0
    double g[MAXS][MAXS];   // stiffened gamma
    double V0[MAXS][MAXS];  // Kataoka V0
    double ep[MAXS][MAXS];  // Kataoka eps
};

// Template value of the EOS parameter for the three real-gas mixtures chosen at run time by
// MixParams::eos_kind (Redlich-Kwong, stiffened, Kataoka): they run on the generic path only.
constexpr int kEosGeneral = 9;

template <typename T, int NS, int EOS>
struct Mixture {
    // X_k = c_k / c_0 ; Cv_mix = sum X_k Cv_k (fractionCalculation.cpp:36-44, mixtureIdeal.cpp)
    __device__ __forceinline__ static void params(const MixParams& mp, const T* c, T& g1, T& am, T& bm, T& Mm) {
        T X[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) X[k] = c[k + 1] / c[0];
        T Cvm = 0;
        Mm = 0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            Cvm += X[k] * T(mp.Cv[k]);
            Mm += X[k] * T(mp.M[k]);
        }
        g1 = T(mp.R) / Cvm;
        am = 0;
        bm = 0;
        if (EOS == FV_EOS_VAN_DER_WAALS) {
#pragma unroll
            for (int k = 0; k < NS; ++k)
#pragma unroll
                for (int l = 0; l < NS; ++l) {
                    am += X[k] * X[l] * T(mp.a[k][l]);
                    bm += X[k] * X[l] * T(mp.b[k][l]);
                }
        }
    }
    // The mixture coefficients of one set of concentrations.  The reference recomputes them in
    // every EOS call; computing them once per state and passing them on gives the same bits (the
    // same operations on the same values) with fewer divisions.
    struct Coef {
        T g1, am, bm, Mm;
    };
    __device__ __forceinline__ static Coef coef(const MixParams& mp, const T* c) {
        Coef k;
        params(mp, c, k.g1, k.am, k.bm, k.Mm);
        return k;
    }
    __device__ __forceinline__ static T pFromUv(const Coef& k, const T* c, T Uv) {
        if (EOS == FV_EOS_IDEAL) return k.g1 * Uv;
        const T acc = k.am * (c[0] * c[0]);
        return k.g1 * (Uv + acc) / (T(1) - c[0] * k.bm) - acc;
    }
    __device__ __forceinline__ static T UvFromp(const Coef& k, const T* c, T p) {
        if (EOS == FV_EOS_IDEAL) return p / k.g1;
        const T acc = k.am * (c[0] * c[0]);
        return (p + acc) * (T(1) - c[0] * k.bm) / k.g1 - acc;
    }
    __device__ __forceinline__ static T pFromUv(const MixParams& mp, const T* c, T Uv) {
        return pFromUv(coef(mp, c), c, Uv);
    }
    __device__ __forceinline__ static T UvFromp(const MixParams& mp, const T* c, T p) {
        return UvFromp(coef(mp, c), c, p);
    }
    // idealFluid.cpp:37-41, vanDerWaalsFluid.cpp:44-48 with Cv_mix = sum X_k Cv_k
    __device__ __forceinline__ static T TFromUv(const MixParams& mp, const T* c, T Uv) {
        T X[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) X[k] = c[k + 1] / c[0];
        T Cvm = 0;
#pragma unroll
        for (int k = 0; k < NS; ++k) Cvm += X[k] * T(mp.Cv[k]);
        if (EOS == FV_EOS_IDEAL) return Uv / ((c[0] + Num<T>::stab()) * Cvm);
        T am = 0;
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int l = 0; l < NS; ++l) am += X[k] * X[l] * T(mp.a[k][l]);
        return (Uv + am * (c[0] * c[0])) / ((c[0] + Num<T>::stab()) * Cvm);
    }
    // sqSonicSpeed = dpdrho + dpdUv * (Uv + p) / rho
    __device__ __forceinline__ static T sqSonic(const Coef& k, const T* c, T rho, T Uv, T p) {
        if (EOS == FV_EOS_IDEAL) return T(0) + k.g1 * (Uv + p) / rho;
        const T m_cb = T(1) - c[0] * k.bm;
        const T ac = k.am * c[0];
        const T dpdrho = (k.g1 * (T(2) * ac / m_cb - k.bm * (Uv + ac * c[0]) / (m_cb * m_cb)) - T(2) * ac) / k.Mm;
        const T dUv = k.g1 / m_cb;
        return dpdrho + dUv * (Uv + p) / rho;
    }
    __device__ __forceinline__ static T sqSonic(const MixParams& mp, const T* c, T rho, T Uv, T p) {
        return sqSonic(coef(mp, c), c, rho, Uv, p);
    }
};

// ------------------------------------------------------------------ real-gas mixtures
// Redlich-Kwong (mixtureRedlichKwong.cpp, RedlichKwongFluid.cpp), stiffened (mixtureStiffened.cpp,
// stiffenedFluid.cpp) and Kataoka-van der Waals (mixtureKataokaVanDerWaals.cpp,
// KataokaVanDerWaalsFluid.cpp) in FP64 whatever the step's arithmetic, each expression in the
// reference's operation order.  The Redlich-Kwong cubic is solved in FP64 where the reference uses
// long double (cubicEquationSolver.cpp), and the device's transcendental functions round their
// last bit differently from the host's, so these agree with the reference to rounding, not bit
// for bit.  A cubic without a single positive root (the reference's positivnessError) gives NaN,
// which the flux reports as a Riemann solver error.
namespace realgas {

__device__ __forceinline__ int signOf(double v) {  // sign.cpp
    const double z = kStabD();
    if (v > z) return 1;
    if (v < -z) return -1;
    return 0;
}

// cubicEquationSolver + returnSinglePosValue: the single positive root of A x^3 + B x^2 + C x + D
__device__ inline double cubicPositiveRoot(double A, double B, double C, double D) {
    const double z = kStabD();
    const double third = 1. / 3., twoThirds = 2. / 3.;
    const double pi = 3.141592653589793;  // acos(-1)
    double x[3] = {CUDART_NAN, CUDART_NAN, CUDART_NAN};
    if ((A > 1E-9) || (A < -1E-9)) {
        const double a = B / A, b = C / A, c = D / A;
        const double Q = (a * a - 3 * b) / 9;
        const double R = (a * (2 * (a * a) - 9 * b) + 27 * c) / 54;
        const double S = (Q * Q) * Q - R * R;
        if (S >= z) {
            const double phi = third * acos(R / sqrt(Q * Q * Q));
            x[0] = -2. * sqrt(Q) * cos(phi) - a * third;
            x[1] = -2. * sqrt(Q) * cos(phi - twoThirds * pi) - a * third;
            x[2] = -2. * sqrt(Q) * cos(phi + twoThirds * pi) - a * third;
        } else if ((S < z) && (S >= -z)) {
            x[0] = -2. * signOf(R) * sqrt(Q) - a * third;
            x[1] = signOf(R) * sqrt(Q) - a * third;
            x[2] = x[1];
        } else if (S < -z) {
            if (Q >= z) {
                const double phi = third * acosh(fabs(R) / (sqrt((Q * Q) * Q) + z));
                x[0] = -2. * signOf(R) * sqrt(Q) * cosh(phi) - a * third;
            } else if ((Q < z) && (Q >= -z)) {
                x[0] = -cbrt(c - (a * a) * a / 27) - a * third;
            } else if (Q < -z) {
                const double phi = third * asinh(fabs(R) / (sqrt(fabs((Q * Q) * Q)) + z));
                x[0] = -2. * signOf(R) * sqrt(fabs(Q)) * sinh(phi) - a * third;
            }
        }
    } else {
        const double a = B, b = C, c = D;
        const double Discr = b * b - 4 * a * c;
        if (Discr >= 0) {
            const double a2 = 0.5 / (a + z);
            x[0] = a2 * (-b + sqrt(Discr));
            x[1] = a2 * (-b - sqrt(Discr));
        }
    }
    int nPositive = 0;
    for (int i = 0; i < 3; ++i) {
        if (x[i] >= 0) nPositive++;
        else x[i] = -123.;
    }
    if (nPositive == 1) return fmax(fmax(x[0], x[1]), x[2]);
    if (nPositive == 2) {
        if (((x[0] - x[1]) < z) && (x[2] < 0)) return x[0];
        if (((x[1] - x[2]) < z) && (x[0] < 0)) return x[1];
        if (((x[0] - x[2]) < z) && (x[1] < 0)) return x[2];
    } else if (nPositive == 3 && ((x[0] - x[1]) < z) && ((x[1] - x[2]) < z)) {
        return x[0];
    }
    return CUDART_NAN;
}

// Kataoka cluster series, M = 13 terms; the derivative series of the reference run no term
constexpr double kKataokaTerms = 13;
__device__ inline double kqa(double c, double T, double V0, double eps, double R) {
    const double V0c = V0 * c, epsRT = 0.5 * eps / (R * T);
    double series = 1.0;
    for (int J = 2; J <= (int)kKataokaTerms; ++J) series += pow(V0c, (J - 1.) / 3.) * exp((J - 1.) * epsRT);
    return series;
}
__device__ inline double kUvA(double c, double T, double V0, double eps, double R) {
    const double V0c = V0 * c, epsRT = 0.5 * eps / (R * T);
    double series = 0;
    for (int J = 2; J <= (int)kKataokaTerms; ++J) series -= (J - 1.) * pow(V0c, (J - 1.) / 3.) * exp((J - 1.) * epsRT);
    return 0.5 * c * eps * series / kqa(c, T, V0, eps, R);
}
__device__ inline double kpA(double c, double T, double V0, double eps, double R) {
    const double V0c = V0 * c, epsRT = 0.5 * eps / (R * T);
    double series = 0;
    for (int J = 2; J <= (int)kKataokaTerms; ++J)
        series -= (J - 1.) / 3. * pow(V0c, (J - 1.) / 3.) * exp((J - 1.) * epsRT);
    return c * R * T * series / kqa(c, T, V0, eps, R);
}
__device__ inline double kdPdC(double c, double T, double V0, double eps, double R, double b) {
    const double V0c = V0 * c, n13 = 0.0, qa1 = kqa(c, T, V0, eps, R);
    return R * T / (1 - c * b) + c * R * T * b / ((1 - c * b) * (1 - c * b)) +
           (R * T * n13 + V0c * R * T * (0.0 - n13 * 0.0 / qa1)) / qa1;
}
__device__ inline double kdPdT(double c, double T, double V0, double eps, double R, double b) {
    const double n13 = 0.0, qa1 = kqa(c, T, V0, eps, R);
    return c * R / (1 - c * b) + (c * R * n13 + 0.5 * c * eps / T * (0.0 - n13 * 0.0 / qa1)) / qa1;
}
__device__ inline double kdUvdC(double c, double Cv, double T, double V0, double eps, double R) {
    const double V0c = V0 * c, n13 = 0.0, qa1 = kqa(c, T, V0, eps, R);
    return Cv * T + (0.5 * eps * n13 + 0.5 * V0c * eps * (0.0 - n13 * 0.0 / qa1)) / qa1;
}
__device__ inline double kdUvdT(double c, double Cv, double T, double V0, double eps, double R) {
    const double qa1 = kqa(c, T, V0, eps, R), s2 = 0.0;
    return c * Cv + 0.25 * c * (eps * eps) / (R * (T * T)) * 0.0 / qa1 -
           0.25 * c * (eps * eps) / (R * (T * T)) * (s2 * s2) / (qa1 * qa1);
}
// NewtonMethod.cpp:13-40 on T (tolerance 1e-12, at most 100 further iterations)
template <class F, class DF> __device__ inline double newton(double x1, F f, DF df) {
    double x2 = x1 - f(x1) / df(x1);
    if (fabs(x2 - x1) <= 1E-12) return x2;
    for (int it = 1; fabs(x2 - x1) > 1E-12 && it <= 100; ++it) {
        x1 = x2;
        x2 = x1 - f(x1) / df(x1);
    }
    return x2;
}
__device__ inline double kTFromUv(double c, double Cv, double Uv, double V0, double eps, double R) {
    auto f = [&](double T) { return c * Cv * T + kUvA(c, T, V0, eps, R) - Uv; };
    auto df = [&](double T) { return kdUvdT(c, Cv, T, V0, eps, R); };
    return newton(Uv / ((c + kStabD()) * Cv), f, df);
}
// Redlich-Kwong derivatives (RedlichKwongFluid.cpp:14-44)
__device__ inline double rkdPdC(double c, double T, double a, double b, double R) {
    return R * T / (1 - c * b) + c * R * T * b / ((1 - c * b) * (1 - c * b)) - 2 * a * c / (sqrt(T) * (1 + b * c)) +
           a * (c * c) * b / (sqrt(T) * ((1 + b * c) * (1 + b * c)));
}
__device__ inline double rkdPdT(double c, double T, double a, double b, double R) {
    const double sT = sqrt(T);
    return c * R / (1 - c * b) + 0.5 * a * (c * c) / (((sT * sT) * sT) * (1 + c * b));
}
__device__ inline double rkdUvdC(double c, double Cv, double T, double a, double b) {
    return Cv * T - 1.5 * a * log1p(c * b) / (b * sqrt(T)) - 1.5 * a * c / (sqrt(T) * (1 + c * b));
}
__device__ inline double rkdUvdT(double c, double Cv, double T, double a, double b) {
    const double sT = sqrt(T);
    return c * Cv + 0.75 * a * c * log1p(c * b) / (b * ((sT * sT) * sT));
}
__device__ inline double rkSqrtT(double c, double Cv, double Uv, double a, double b) {
    return cubicPositiveRoot(c * Cv, 0, -Uv, -1.5 * a * c / b * log1p(c * b));
}

}  // namespace realgas

template <typename T, int NS>
struct Mixture<T, NS, kEosGeneral> {
    // the mixture sums of one set of concentrations (X_k = c_k / c_0), with the EOS kind and R
    struct Coef {
        int kind;
        double R, c0, Cvm, Mm;  // gas constant, total concentration, Cv and M of the mixture
        double a, b;            // Redlich-Kwong a and b; Kataoka b
        double p0, g;           // stiffened p0 and gamma
        double V0, ep;          // Kataoka V0 and eps
    };
    __device__ __forceinline__ static Coef coef(const MixParams& mp, const T* c) {
        Coef k{};
        k.kind = mp.eos_kind;
        k.R = mp.R;
        k.c0 = double(c[0]);
        double X[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) X[q] = double(c[q + 1]) / double(c[0]);
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            k.Cvm += X[q] * mp.Cv[q];
            k.Mm += X[q] * mp.M[q];
        }
#pragma unroll
        for (int q = 0; q < NS; ++q)
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                if (k.kind == FV_EOS_STIFFENED) {
                    k.p0 += X[q] * X[l] * mp.p0[q][l];
                    k.g += X[q] * X[l] * mp.g[q][l];
                } else if (k.kind == FV_EOS_KATAOKA) {
                    k.V0 += X[q] * X[l] * mp.V0[q][l];
                    k.ep += X[q] * X[l] * mp.ep[q][l];
                    k.b += X[q] * X[l] * mp.b[q][l];
                } else {
                    k.a += X[q] * X[l] * mp.a[q][l];
                    k.b += X[q] * X[l] * mp.b[q][l];
                }
            }
        return k;
    }
    // stiffenedFluid.cpp:13-17, RedlichKwongFluid.cpp:46-56, KataokaVanDerWaalsFluid.cpp:237-256
    __device__ __noinline__ static double pFromUvD(const Coef& k, double Uv) {
        const double c = k.c0;
        if (k.kind == FV_EOS_STIFFENED) return (k.g - 1.0) * Uv - k.p0 * k.g;
        if (k.kind == FV_EOS_KATAOKA) {
            const double Tk = realgas::kTFromUv(c, k.Cvm, Uv, k.V0, k.ep, k.R);
            return c * k.R * Tk / (1 - c * k.b) + realgas::kpA(c, Tk, k.V0, k.ep, k.R);
        }
        const double sT = realgas::rkSqrtT(c, k.Cvm, Uv, k.a, k.b);
        return c * k.R * (sT * sT) / (1 - c * k.b) - k.a * (c * c) / (sT * (1 + c * k.b));
    }
    // stiffenedFluid.cpp:19-23, RedlichKwongFluid.cpp:58-68, KataokaVanDerWaalsFluid.cpp:258-277
    __device__ __noinline__ static double UvFrompD(const Coef& k, double p) {
        const double c = k.c0;
        if (k.kind == FV_EOS_STIFFENED) return (p + k.p0 * k.g) / (k.g - 1.0);
        if (k.kind == FV_EOS_KATAOKA) {
            const double V0 = k.V0, ep = k.ep, R = k.R, b = k.b;
            auto f = [&](double Tk) { return c * R * Tk / (1 - c * b) + realgas::kpA(c, Tk, V0, ep, R) - p; };
            auto df = [&](double Tk) { return realgas::kdPdT(c, Tk, V0, ep, R, b); };
            const double Tk = realgas::newton(p / ((c + kStabD()) * R), f, df);
            return c * k.Cvm * Tk + realgas::kUvA(c, Tk, V0, ep, R);
        }
        const double sT = realgas::cubicPositiveRoot(c * k.R, 0, -p * (1 - c * k.b),
                                                     -k.a * (c * c) * (1 - c * k.b) / (1 + c * k.b));
        return c * k.Cvm * (sT * sT) - 1.5 * k.a * c / (k.b * sT) * log1p(c * k.b);
    }
    // sqSonicSpeed = dpdrho + dpdUv (Uv + p) / rho
    __device__ __noinline__ static double sqSonicD(const Coef& k, double rho, double Uv, double p) {
        const double c = k.c0;
        if (k.kind == FV_EOS_STIFFENED) return 0 + (k.g - 1.0) * (Uv + p) / rho;
        if (k.kind == FV_EOS_KATAOKA) {  // KataokaVanDerWaalsFluid.cpp:332-372
            const double Tk = realgas::kTFromUv(c, k.Cvm, Uv, k.V0, k.ep, k.R);
            const double dpdrho = (realgas::kdPdC(c, Tk, k.V0, k.ep, k.R, k.b) -
                                   realgas::kdPdT(c, Tk, k.V0, k.ep, k.R, k.b) *
                                       realgas::kdUvdC(c, k.Cvm, Tk, k.V0, k.ep, k.R) /
                                       realgas::kdUvdT(c, k.Cvm, Tk, k.V0, k.ep, k.R)) /
                                  k.Mm;
            const double dpdUv =
                realgas::kdPdT(c, Tk, k.V0, k.ep, k.R, k.b) / realgas::kdUvdT(c, k.Cvm, Tk, k.V0, k.ep, k.R);
            return dpdrho + dpdUv * (Uv + p) / rho;
        }
        // RedlichKwongFluid.cpp:104-131
        const double sT = realgas::rkSqrtT(c, k.Cvm, Uv, k.a, k.b);
        const double Tr = sT * sT;
        const double dpdrho = (realgas::rkdPdC(c, Tr, k.a, k.b, k.R) -
                               realgas::rkdPdT(c, Tr, k.a, k.b, k.R) * realgas::rkdUvdC(c, k.Cvm, Tr, k.a, k.b) /
                                   realgas::rkdUvdT(c, k.Cvm, Tr, k.a, k.b)) /
                              k.Mm;
        const double dpdUv = realgas::rkdPdT(c, Tr, k.a, k.b, k.R) / realgas::rkdUvdT(c, k.Cvm, Tr, k.a, k.b);
        return dpdrho + dpdUv * (Uv + p) / rho;
    }
    // stiffenedFluid.cpp:37-41, RedlichKwongFluid.cpp:84-92, KataokaVanDerWaalsFluid.cpp:291-306
    __device__ __noinline__ static double TFromUvD(const Coef& k, double Uv) {
        const double c = k.c0;
        if (k.kind == FV_EOS_STIFFENED) return (Uv - k.p0) / ((c + kStabD()) * k.Cvm);
        if (k.kind == FV_EOS_KATAOKA) return realgas::kTFromUv(c, k.Cvm, Uv, k.V0, k.ep, k.R);
        const double sT = realgas::rkSqrtT(c, k.Cvm, Uv, k.a, k.b);
        return sT * sT;
    }

    __device__ __forceinline__ static T pFromUv(const Coef& k, const T*, T Uv) { return T(pFromUvD(k, double(Uv))); }
    __device__ __forceinline__ static T UvFromp(const Coef& k, const T*, T p) { return T(UvFrompD(k, double(p))); }
    __device__ __forceinline__ static T sqSonic(const Coef& k, const T*, T rho, T Uv, T p) {
        return T(sqSonicD(k, double(rho), double(Uv), double(p)));
    }
    __device__ __forceinline__ static T pFromUv(const MixParams& mp, const T* c, T Uv) {
        return pFromUv(coef(mp, c), c, Uv);
    }
    __device__ __forceinline__ static T UvFromp(const MixParams& mp, const T* c, T p) {
        return UvFromp(coef(mp, c), c, p);
    }
    __device__ __forceinline__ static T sqSonic(const MixParams& mp, const T* c, T rho, T Uv, T p) {
        return sqSonic(coef(mp, c), c, rho, Uv, p);
    }
    __device__ __forceinline__ static T TFromUv(const MixParams& mp, const T* c, T Uv) {
        return T(TFromUvD(coef(mp, c), double(Uv)));
    }
};

// ------------------------------------------------------------------ limiter functions
template <typename T> __device__ __forceinline__ T limiterPhi(int lim, T r, T xiR) {
    const T one = 1, two = 2;
    switch (lim) {
    case FV_LIM_ZERO: return 0;
    case FV_LIM_MINMOD:
        if (r <= T(0)) return 0;
        if (r <= one) return r;
        return smin(one, xiR);
    case FV_LIM_VANLEER:
        if (r < T(0)) return 0;
        return smin(two * r / (one + r), xiR);
    case FV_LIM_LINEAR: return one;
    case FV_LIM_VANALBADA:
        if (r <= T(0)) return 0;
        return smin((r * r + r) / (one + r * r), xiR);
    case FV_LIM_HQUICK:
        if (r <= T(0)) return 0;
        return smin(T(4) * r / (T(3) + r), xiR);
    case FV_LIM_VANLEER2: {
        if (r <= T(0)) return 0;
        const T denom = one + r;
        return smin(T(4) * r / (denom * denom), two * xiR);
    }
    case FV_LIM_SUPERBEE:
        if (r <= T(0)) return 0;
        if (r <= T(0.5)) return two * r;
        if (r <= one) return r;
        return smin(smin(r, two), xiR);
    case FV_LIM_VANALBADA2:
        if (r <= T(0)) return 0;
        return smin(two * r / (one + r * r), two * xiR);
    case FV_LIM_MINMOD2:
        if (r <= T(0)) return 0;
        return smin(smin(one, T(4) * r / (one + r)), two * xiR);
    case FV_LIM_SWEBY: {
        const T b = 2;
        if (r <= T(0)) return 0;
        return smin(smin(smin(one, b * r), smin(b, r)), b * xiR);
    }
    case FV_LIM_KOREN:
        if (r <= T(0)) return 0;
        return smin(smin(smin(two * r, (one + two * r) / T(3)), two), two * xiR);
    case FV_LIM_KOREN2: {
        const T tt = T(2. / 3.);
        if (r <= T(0)) return smin(T(0), smax(-tt, (one + two * r) / T(3)));
        return smin(smin(two * tt * r, smin((one + two * r) / T(3), two)), two * xiR);
    }
    case FV_LIM_UTCDFS:
        if (r < T(-1)) return r * (r + one) / (r * r + one);
        if ((r >= T(-1)) && (r < T(0))) return 0;
        if ((r >= T(0)) && (r < T(0.5))) return r * r * r - two * (r * r) + two * r;
        if ((r >= T(0.5)) && (r < two)) return T(0.75) * r + T(0.25);
        return smin((two * (r * r) - two * r - T(9.0 / 4.0)) / (r * r - r - one), two * xiR);
    case FV_LIM_SCHMIDTMANN: {
        const T alpha = 1, beta = 2, gamma = 1.5;
        const T phiO3 = (two + r) / T(3);
        return smin(smax(T(0), smin(phiO3, smax(-alpha * r, smin(smin(beta * r, phiO3), gamma)))), two * xiR);
    }
    }
    return 0;
}

// True when phi(r) == 0 for every r <= 0: on a multi-dimensional structured mesh the r-ratio
// of every gradient component is <= 0 (transverse neighbours contribute an exact 0 to the
// component-wise min/max of TVDLimiter.cpp:103-119), so these limiters give zero slopes and
// the reconstruction is piecewise constant.
__host__ __device__ inline bool limiterZeroForNonPositiveR(int lim) {
    switch (lim) {
    case FV_LIM_LINEAR: case FV_LIM_KOREN2: case FV_LIM_UTCDFS: case FV_LIM_SCHMIDTMANN: return false;
    default: return true;
    }
}

// ------------------------------------------------------------------ face states
// One side of one face: primitives + conserved + sound speed.
template <typename T, int NS>
struct FaceState {
    T c[NS + 1];    // c[0] = total concentration
    T rho[NS + 1];  // rho[0] = mixture density (evolved separately)
    T v[3], m[3];
    T E, Uv, p, cs;
};

// Closure of a reconstructed primitive state (Advection.cpp:238-303 / :305-387).
// `known`: the mixture coefficients of these concentrations when the caller has them already.
template <typename T, int NS, int EOS>
__device__ __forceinline__ void closeFromPrimitive(const MixParams& mp, FaceState<T, NS>& s,
                                                   const typename Mixture<T, NS, EOS>::Coef* known = nullptr) {
    s.c[0] = 0;
    s.rho[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        s.c[0] += s.c[k];
        s.rho[k] = s.c[k] * T(mp.M[k - 1]);
        s.rho[0] += s.rho[k];
    }
    s.Uv = known ? Mixture<T, NS, EOS>::UvFromp(*known, s.c, s.p) : Mixture<T, NS, EOS>::UvFromp(mp, s.c, s.p);
#pragma unroll
    for (int d = 0; d < 3; ++d) s.m[d] = s.v[d] * s.rho[0];
    T v2 = 0;
    v2 += s.v[0] * s.v[0];
    v2 += s.v[1] * s.v[1];
    v2 += s.v[2] * s.v[2];
    s.E = s.Uv + s.rho[0] * v2 * T(0.5) + T(0);
}

// Recalculation from conserved face values (HancockStage.cpp:177-224, Advection.cpp:455-479).
// `nmom` momentum components are carried; the others are exactly zero and so is their
// velocity (0 / rho = +0 for a positive density).
// `out`: receives the mixture coefficients of the new concentrations (for soundSpeed).
template <typename T, int NS, int EOS>
__device__ __forceinline__ void closeFromConserved(const MixParams& mp, FaceState<T, NS>& s, int nmom = 3,
                                                   typename Mixture<T, NS, EOS>::Coef* out = nullptr) {
    s.c[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        s.c[k] = s.rho[k] / T(mp.M[k - 1]);
        s.c[0] += s.c[k];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) s.v[d] = d < nmom ? s.m[d] / s.rho[0] : T(0);
    T v2 = 0;
    v2 += s.v[0] * s.v[0];
    v2 += s.v[1] * s.v[1];
    v2 += s.v[2] * s.v[2];
    s.Uv = s.E - s.rho[0] * v2 * T(0.5) - T(0);
    const typename Mixture<T, NS, EOS>::Coef k = Mixture<T, NS, EOS>::coef(mp, s.c);
    s.p = Mixture<T, NS, EOS>::pFromUv(k, s.c, s.Uv);
    if (out) *out = k;
}

// Sound speed of HLLCSolver.cpp:26-50 with zero turbulent energy.
template <typename T, int NS, int EOS>
__device__ __forceinline__ void soundSpeed(const MixParams& mp, FaceState<T, NS>& s) {
    s.cs = Num<T>::sqrt_(Mixture<T, NS, EOS>::sqSonic(mp, s.c, s.rho[0], s.Uv, s.p) + T(0));
}
template <typename T, int NS, int EOS>
__device__ __forceinline__ void soundSpeed(const typename Mixture<T, NS, EOS>::Coef& k, FaceState<T, NS>& s) {
    s.cs = Num<T>::sqrt_(Mixture<T, NS, EOS>::sqSonic(k, s.c, s.rho[0], s.Uv, s.p) + T(0));
}

// ------------------------------------------------------------------ boundary conditions
struct BCParams {
    int conc[6][MAXS];
    double conc_value[6][MAXS];
    int vel[6];
    double vel_value[6][3];
    int p[6];
    double p_value[6];
};

// boundaryConditionValueCell for a scalar (free / slip -> value, fixedValueCell -> fixed value)
template <typename T> __device__ __forceinline__ T ghostScalar(int type, double fixed, T in) {
    return type == FV_BC_FIXED_CELL ? T(fixed) : in;
}

// boundaryConditionValueCell for the velocity; the patch normal is sign * e_axis.
// slip: (v - (v & n) n) * 2 - v, evaluated in the reference's component order.
template <typename T>
__device__ __forceinline__ void ghostVelocity(int type, const double* fixed, int axis, int sign, const T* in, T* out) {
    if (type == FV_BC_FIXED_CELL) {
        out[0] = T(fixed[0]); out[1] = T(fixed[1]); out[2] = T(fixed[2]);
        return;
    }
    if (type == FV_BC_SLIP) {
        // n = sign * e_axis ; v & n = ((0 + v0 n0) + v1 n1) + v2 n2
        T n[3] = {T(0), T(0), T(0)};
        n[axis] = T(sign);
        T vn = 0;
        vn += in[0] * n[0];
        vn += in[1] * n[1];
        vn += in[2] * n[2];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T s = in[d] - n[d] * vn;
            out[d] = s * T(2) - in[d];
        }
        return;
    }
    out[0] = in[0]; out[1] = in[1]; out[2] = in[2];
}

// Ghost neighbour state of a boundary face from the owner-side state (HancockStage.cpp:324-446).
template <typename T, int NS, int EOS>
__device__ __forceinline__ void ghostState(const MixParams& mp, const BCParams& bc, int patch, int axis, int sign,
                                           const FaceState<T, NS>& own, FaceState<T, NS>& g) {
    g.c[0] = 0;
    g.rho[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        g.c[k] = ghostScalar<T>(bc.conc[patch][k - 1], bc.conc_value[patch][k - 1], own.c[k]);
        g.rho[k] = g.c[k] * T(mp.M[k - 1]);
        g.c[0] += g.c[k];
        g.rho[0] += g.rho[k];
    }
    ghostVelocity<T>(bc.vel[patch], bc.vel_value[patch], axis, sign, own.v, g.v);
#pragma unroll
    for (int d = 0; d < 3; ++d) g.m[d] = g.v[d] * g.rho[0];
    g.p = ghostScalar<T>(bc.p[patch], bc.p_value[patch], own.p);
    g.Uv = Mixture<T, NS, EOS>::UvFromp(mp, g.c, g.p);
    T v2 = 0;
    v2 += g.v[0] * g.v[0];
    v2 += g.v[1] * g.v[1];
    v2 += g.v[2] * g.v[2];
    g.E = g.Uv + g.rho[0] * v2 * T(0.5) + T(0);
    soundSpeed<T, NS, EOS>(mp, g);
}

// ------------------------------------------------------------------ fluxes
// Scalar fluxes through a face with normal N = sign * e_axis, expressed along N: the
// reference stores F (x) N and every consumer contracts it with +-N, which returns these
// scalars exactly.  rho[0..NS], m[0..2], E.
template <typename T, int NS>
struct FaceFlux {
    T rho[NS + 1];
    T m[3];
    T E;
};

// pressureStar (pressureStarClass.cpp:12-36) of a star state: c_k = rho_k / M_k,
// Uv = E - 0.5 (m & m) / rho - rho k, p = pFromUv(c, Uv)
template <typename T, int NS, int EOS>
__device__ __forceinline__ T starPressure(const MixParams& mp, const T* rs, const T* ms, T Es) {
    T m2 = 0;
    m2 += ms[0] * ms[0];
    m2 += ms[1] * ms[1];
    m2 += ms[2] * ms[2];
    const T kin = T(0.5) * m2 / rs[0];
    const T Uv = Es - kin - T(0);
    T c[NS + 1];
    c[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = rs[k] / T(mp.M[k - 1]);
        c[0] += c[k];
    }
    return Mixture<T, NS, EOS>::pFromUv(mp, c, Uv);
}

// HLLC (HLLCSolver.cpp:52-403) or HLL (HLLSolver.cpp:52-300); returns false when no branch
// applies (NaN wave speeds), which the reference reports as RiemannSolverError.
template <typename T, int NS, int EOS = -1>
__device__ __forceinline__ bool riemann(int flux, int axis, int sign, const FaceState<T, NS>& O,
                                        const FaceState<T, NS>& B, FaceFlux<T, NS>& F, T* sv = nullptr,
                                        T* sp = nullptr, const MixParams* mp = nullptr) {
    // sv (HLLC, not null): the face velocity the solver hands the diffusion stage (starValues.v,
    // HLLCSolver.cpp:399): the side's velocity outside the star region, the star momentum over
    // the star density inside it; sp (EOS given, not null): the pressure beside it (starValues.p,
    // :400), the side's outside the star region, pressureStar of the star state inside it
    const T sg = T(sign);
    const T uO = O.v[axis] * sg, uN = B.v[axis] * sg;
    const T SO = smin(uO - O.cs, uN - B.cs);
    const T SN = smax(uO + O.cs, uN + B.cs);
    // (I & N)_d * p is sign * p on the normal axis and 0 * p elsewhere
    if (flux == FV_FLUX_HLLC) {
        const T Sc = ((B.p + T(0)) - (O.p + T(0)) + O.rho[0] * uO * (SO - uO) - B.rho[0] * uN * (SN - uN)) /
                     (O.rho[0] * (SO - uO) - B.rho[0] * (SN - uN));
        const T PON = T(0.5) * ((O.p + T(0)) + (B.p + T(0)) + O.rho[0] * (SO - uO) * (Sc - uO) +
                                B.rho[0] * (SN - uN) * (Sc - uN));
        if (SO >= T(0)) {
#pragma unroll
            for (int k = 0; k <= NS; ++k) F.rho[k] = (sg * uO) * O.rho[k] * sg;
#pragma unroll
            for (int d = 0; d < 3; ++d) F.m[d] = O.m[d] * uO + (d == axis ? sg : T(0)) * (O.p + T(0));
            F.E = uO * (O.E + O.p + T(0));
            if (sv) {
#pragma unroll
                for (int d = 0; d < 3; ++d) sv[d] = O.v[d];
            }
            if (sp) *sp = O.p;
        } else if (Sc >= T(0) || SN > T(0)) {
            // star flux of the side the contact leaves (owner when Sc >= 0): the reference's two
            // branches are the same expression on (O, uO, SO) or (B, uN, SN)
            auto star = [&](const T* rw, const T* mw, T Ew, T pw, T u, T S) {
                const T factor = S - u;
                const T den = T(1) / (S - Sc);
                T rsa[NS + 1], msa[3];
#pragma unroll
                for (int k = 0; k <= NS; ++k) {
                    const T rs = rw[k] * factor * den;
                    rsa[k] = rs;
                    F.rho[k] = rw[k] * u + S * (rs - rw[k]);
                }
                const T rs0 = rw[0] * factor * den;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const T ms = (mw[d] * factor - (d == axis ? sg : T(0)) * (pw + T(0) - PON)) * den;
                    msa[d] = ms;
                    F.m[d] = mw[d] * u + (d == axis ? sg : T(0)) * (pw + T(0)) + (ms - mw[d]) * S;
                    if (sv) sv[d] = ms / rs0;
                }
                const T Es = (Ew * factor - (pw + T(0)) * u + PON * Sc) * den;
                F.E = (Ew + pw + T(0)) * u + S * (Es - Ew);
                if constexpr (EOS >= 0) {
                    if (sp) *sp = starPressure<T, NS, EOS>(*mp, rsa, msa, Es);
                }
                (void)rsa;
                (void)msa;
            };
            const bool own = Sc >= T(0);
            if constexpr (sizeof(T) == 8) {
                // FP64 (latency-bound): select the side by value and evaluate once, so that a warp
                // whose faces see contacts moving both ways does not run both branches
                T rw[NS + 1], mw[3];
#pragma unroll
                for (int k = 0; k <= NS; ++k) rw[k] = own ? O.rho[k] : B.rho[k];
#pragma unroll
                for (int d = 0; d < 3; ++d) mw[d] = own ? O.m[d] : B.m[d];
                star(rw, mw, own ? O.E : B.E, own ? O.p : B.p, own ? uO : uN, own ? SO : SN);
            } else {
                // FP32 (issue-bound): the selects cost more than the divergence they save
                if (own) star(O.rho, O.m, O.E, O.p, uO, SO);
                else star(B.rho, B.m, B.E, B.p, uN, SN);
            }
        } else if (SN <= T(0)) {
#pragma unroll
            for (int k = 0; k <= NS; ++k) F.rho[k] = (sg * uN) * B.rho[k] * sg;
#pragma unroll
            for (int d = 0; d < 3; ++d) F.m[d] = B.m[d] * uN + (d == axis ? sg : T(0)) * (B.p + T(0));
            F.E = uN * (B.E + B.p + T(0));
            if (sv) {
#pragma unroll
                for (int d = 0; d < 3; ++d) sv[d] = B.v[d];
            }
            if (sp) *sp = B.p;
        } else {
            return false;
        }
        return true;
    }
    // HLL
    if (SO >= T(0)) {
#pragma unroll
        for (int k = 0; k <= NS; ++k) F.rho[k] = sg * (uO * O.rho[k]) * sg;
#pragma unroll
        for (int d = 0; d < 3; ++d) F.m[d] = O.m[d] * uO + (d == axis ? sg : T(0)) * (O.p + T(0));
        F.E = uO * (O.E + O.p + T(0));
    } else if (SN > T(0)) {
        const T den = T(1) / (SN - SO);
#pragma unroll
        for (int k = 0; k <= NS; ++k)
            F.rho[k] = (SN * uO * O.rho[k] - SO * uN * B.rho[k] + SN * SO * (B.rho[k] - O.rho[k])) * den;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T nd = (d == axis ? sg : T(0));
            const T t1 = (O.m[d] * uO + nd * (O.p + T(0))) * SN;
            const T t2 = (B.m[d] * uN + nd * (B.p + T(0))) * SO;
            const T t3 = (B.m[d] - O.m[d]) * (SN * SO);
            F.m[d] = ((t1 - t2) + t3) * den;
        }
        F.E = (SN * (uO * (O.E + O.p + T(0))) - SO * (uN * (B.E + B.p + T(0))) + SN * SO * (B.E - O.E)) * den;
    } else if (SN <= T(0)) {
#pragma unroll
        for (int k = 0; k <= NS; ++k) F.rho[k] = sg * (uN * B.rho[k]) * sg;
#pragma unroll
        for (int d = 0; d < 3; ++d) F.m[d] = B.m[d] * uN + (d == axis ? sg : T(0)) * (B.p + T(0));
        F.E = uN * (B.E + B.p + T(0));
    } else {
        return false;
    }
    return true;
}

}  // namespace fv
