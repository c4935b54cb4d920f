// fv_adjoint.cuh -- hand-written reverse mode (vector-Jacobian products) of the zero-slope
// finite-volume step for ideal-gas mixtures, and the adjoint step kernel.  No reference
// counterpart: the reference has no adjoint.
//
// The forward map differentiated here is the mathematics of the step the fused march computes
// (fv_kernels.cuh), i.e. secondOrderStepSolver + Advection with a limiter whose multi-dimensional
// slopes are zero (TVDLimiter.cpp:12-272): per cell the face state W(U) -- densities, momenta and
// energy as stored (the Hancock half step cancels exactly for equal face states), velocity
// v = m / rho, internal energy Uv = E - |m|^2 / (2 rho), pressure p = g1 Uv with
// g1 = R / sum_k X_k Cv_k, X_k = c_k / c_0, c_k = rho_k / M_k (mixtureIdeal.cpp), sound speed
// sqrt(g1 (Uv + p) / rho) -- the HLLC or HLL face flux (HLLCSolver.cpp:52-403,
// HLLSolver.cpp:52-300), the ghost state of a boundary face (HancockStage.cpp:324-446,
// boundaryConditionValue.hpp) and the conservative update with the gravity source
// (Advection.cpp:414-431).  The time step and the gravity vector of every step are the recorded
// ones (frozen: the CFL reduction is not differentiated).  NMOM momentum components are carried
// (the others are not updated by the step and are zero).
//
// Convention: every face is evaluated with the normal +e_axis, left state L and right state R.
// For a wall face below a cell this is the mirror image of the forward's (owner, ghost, -e_axis)
// evaluation; HLLC and HLL satisfy F(L, R; n) = -F(R, L; -n), so both define the same map.
//
// Packed order of a cell's conserved values, adjoints and flux adjoints (NL = NS + 2 + NMOM):
// [rho_1 .. rho_NS, rho, m_0 .. m_{NMOM-1}, E].
#pragma once

#include "fv_kernels.cuh"

namespace fv {
namespace adj {

// Per-step record of a trajectory: the step taken, the gravity vector it used and whether the
// step ran (a step enqueued after the end time is a no-op).
struct StepRecord {
    double dt;
    double g[3];
    int ran;
    int pad;
};

// The face-state fields a flux reads.
template <typename T, int NS, int NMOM>
struct FState {
    T rho[NS + 1];  // rho[0] mixture density, rho[1..NS] species
    T m[NMOM], v[NMOM];
    T E, p, cs;
};

// Adjoint of an FState.
template <typename T, int NS, int NMOM>
struct FBar {
    T rho[NS + 1];
    T m[NMOM], v[NMOM];
    T E, p, cs;
};

// Face state with the closure intermediates its reverse pass needs.
template <typename T, int NS, int NMOM>
struct WState {
    FState<T, NS, NMOM> f;
    T Uv;
    T c[NS + 1];  // c[0] = sum of c[1..NS]
    T X[NS];
    T Cvm, g1;
};

// Adjoint of a WState.
template <typename T, int NS, int NMOM>
struct WBar {
    FBar<T, NS, NMOM> f;
    T c[NS + 1];
    T g1;
};

template <typename T, int NS, int NMOM>
__device__ __forceinline__ void zero(FBar<T, NS, NMOM>& b) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) b.rho[k] = 0;
#pragma unroll
    for (int d = 0; d < NMOM; ++d) { b.m[d] = 0; b.v[d] = 0; }
    b.E = b.p = b.cs = 0;
}

template <typename T, int NS, int NMOM>
__device__ __forceinline__ void zero(WBar<T, NS, NMOM>& b) {
    zero<T, NS, NMOM>(b.f);
#pragma unroll
    for (int k = 0; k <= NS; ++k) b.c[k] = 0;
    b.g1 = 0;
}

template <typename T, int NS, int NMOM>
__device__ __forceinline__ void add(FBar<T, NS, NMOM>& a, const FBar<T, NS, NMOM>& b) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) a.rho[k] += b.rho[k];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) { a.m[d] += b.m[d]; a.v[d] += b.v[d]; }
    a.E += b.E;
    a.p += b.p;
    a.cs += b.cs;
}

// a += (on ? b : 0)
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void addIf(FBar<T, NS, NMOM>& a, const FBar<T, NS, NMOM>& b, bool on) {
    const T s = on ? T(1) : T(0);
#pragma unroll
    for (int k = 0; k <= NS; ++k) a.rho[k] += s * b.rho[k];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) { a.m[d] += s * b.m[d]; a.v[d] += s * b.v[d]; }
    a.E += s * b.E;
    a.p += s * b.p;
    a.cs += s * b.cs;
}

template <typename T, int NS, int NMOM>
__device__ __forceinline__ FState<T, NS, NMOM> select(bool left, const FState<T, NS, NMOM>& L,
                                                      const FState<T, NS, NMOM>& R) {
    FState<T, NS, NMOM> s;
#pragma unroll
    for (int k = 0; k <= NS; ++k) s.rho[k] = left ? L.rho[k] : R.rho[k];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        s.m[d] = left ? L.m[d] : R.m[d];
        s.v[d] = left ? L.v[d] : R.v[d];
    }
    s.E = left ? L.E : R.E;
    s.p = left ? L.p : R.p;
    s.cs = left ? L.cs : R.cs;
    return s;
}

// Packing of an FState / FBar into NFS consecutive values (shared-memory exchange).
template <int NS, int NMOM>
constexpr int fsSize() { return NS + 1 + 2 * NMOM + 3; }

template <typename T, int NS, int NMOM, typename S>
__device__ __forceinline__ void pack(const S& s, T* out, int stride) {
    int i = 0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) out[(i++) * stride] = s.rho[k];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) out[(i++) * stride] = s.m[d];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) out[(i++) * stride] = s.v[d];
    out[(i++) * stride] = s.E;
    out[(i++) * stride] = s.p;
    out[(i++) * stride] = s.cs;
}

template <typename T, int NS, int NMOM, typename S>
__device__ __forceinline__ void unpack(const T* in, int stride, S& s) {
    int i = 0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) s.rho[k] = in[(i++) * stride];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) s.m[d] = in[(i++) * stride];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) s.v[d] = in[(i++) * stride];
    s.E = in[(i++) * stride];
    s.p = in[(i++) * stride];
    s.cs = in[(i++) * stride];
}

template <typename T, int NS, int NMOM, typename S>
__device__ __forceinline__ void unpackAdd(const T* in, int stride, S& s) {
    int i = 0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) s.rho[k] += in[(i++) * stride];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) s.m[d] += in[(i++) * stride];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) s.v[d] += in[(i++) * stride];
    s.E += in[(i++) * stride];
    s.p += in[(i++) * stride];
    s.cs += in[(i++) * stride];
}

// g1 = R / sum_k X_k Cv_k from the concentrations.
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void mixtureG1(const MixParams& mp, WState<T, NS, NMOM>& w) {
    w.Cvm = 0;
    const T invc0 = T(1) / w.c[0];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        w.X[k] = w.c[k + 1] * invc0;
        w.Cvm += w.X[k] * T(mp.Cv[k]);
    }
    w.g1 = T(mp.R) / w.Cvm;
}

// W(U) from the packed conserved values.
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void wForward(const MixParams& mp, const T* u, WState<T, NS, NMOM>& w) {
    FState<T, NS, NMOM>& f = w.f;
    f.rho[0] = u[NS];
#pragma unroll
    for (int k = 1; k <= NS; ++k) f.rho[k] = u[k - 1];
    const T inv = T(1) / f.rho[0];
    T v2 = 0;
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        f.m[d] = u[NS + 1 + d];
        f.v[d] = f.m[d] * inv;
        v2 += f.v[d] * f.v[d];
    }
    f.E = u[NS + 1 + NMOM];
    w.Uv = f.E - T(0.5) * f.rho[0] * v2;
    w.c[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) { w.c[k] = f.rho[k] * T(mp.invM[k - 1]); w.c[0] += w.c[k]; }
    mixtureG1<T, NS, NMOM>(mp, w);
    f.p = w.g1 * w.Uv;
    f.cs = sqrt(w.g1 * (w.Uv + f.p) * inv);
}

// Reverse of mixtureG1: adds to cbar[1..NS].
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void g1Reverse(const MixParams& mp, const WState<T, NS, NMOM>& w, T g1bar, T* cbar) {
    const T Cvmbar = -g1bar * w.g1 / w.Cvm;
    T c0bar = 0;
    const T invc0 = T(1) / w.c[0];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const T Xbar = Cvmbar * T(mp.Cv[k]);
        cbar[k + 1] += Xbar * invc0;
        c0bar -= Xbar * w.X[k] * invc0;
    }
#pragma unroll
    for (int k = 1; k <= NS; ++k) cbar[k] += c0bar;
}

// Reverse of wForward: the packed conserved adjoint ub[0..NL-1] (overwritten).
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void wReverse(const MixParams& mp, const WState<T, NS, NMOM>& w, WBar<T, NS, NMOM> b,
                                         T* ub) {
    const FState<T, NS, NMOM>& f = w.f;
    const T inv = T(1) / f.rho[0];
    T rho0bar = b.f.rho[0], Ebar = b.f.E, mbar[NMOM];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) mbar[d] = b.f.m[d];
    // cs = sqrt(q), q = g1 (Uv + p) / rho
    const T qbar = b.f.cs / (T(2) * f.cs);
    b.g1 += qbar * (w.Uv + f.p) * inv;
    const T t = qbar * w.g1 * inv;
    T Uvbar = t;
    b.f.p += t;
    rho0bar -= qbar * f.cs * f.cs * inv;
    // p = g1 Uv
    Uvbar += b.f.p * w.g1;
    b.g1 += b.f.p * w.Uv;
    // Uv = E - |m|^2 / (2 rho)
    Ebar += Uvbar;
    T v2 = 0;
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        mbar[d] -= Uvbar * f.v[d];
        v2 += f.v[d] * f.v[d];
    }
    rho0bar += Uvbar * T(0.5) * v2;
    // v = m / rho
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        mbar[d] += b.f.v[d] * inv;
        rho0bar -= b.f.v[d] * f.v[d] * inv;
    }
    // g1(c), c_k = rho_k / M_k
    g1Reverse<T, NS, NMOM>(mp, w, b.g1, b.c);
#pragma unroll
    for (int k = 1; k <= NS; ++k) ub[k - 1] = b.f.rho[k] + b.c[k] * T(mp.invM[k - 1]);
    ub[NS] = rho0bar;
#pragma unroll
    for (int d = 0; d < NMOM; ++d) ub[NS + 1 + d] = mbar[d];
    ub[NS + 1 + NMOM] = Ebar;
}

// Ghost state of a boundary face from the owner's W, and the reverse into the owner's
// primitive adjoints.  fixedValueCell fields are constants; slip reflects the normal velocity;
// every other type copies the owner's value (the ghost cell of HancockStage.cpp:324-446).
template <typename T, int NS, int NMOM>
struct Ghost {
    WState<T, NS, NMOM> g;
    bool reflect, fixedV, fixedP;
    bool fixedC[NS];
};

template <typename T, int NS, int NMOM>
__device__ __forceinline__ void ghostForward(const MixParams& mp, const BCParams& bc, int patch, int axis,
                                             const WState<T, NS, NMOM>& w, Ghost<T, NS, NMOM>& G) {
    WState<T, NS, NMOM>& g = G.g;
    G.reflect = bc.vel[patch] == FV_BC_SLIP;
    G.fixedV = bc.vel[patch] == FV_BC_FIXED_CELL;
    G.fixedP = bc.p[patch] == FV_BC_FIXED_CELL;
    g.c[0] = 0;
    g.f.rho[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        G.fixedC[k - 1] = bc.conc[patch][k - 1] == FV_BC_FIXED_CELL;
        g.c[k] = G.fixedC[k - 1] ? T(bc.conc_value[patch][k - 1]) : w.c[k];
        g.f.rho[k] = g.c[k] * T(mp.M[k - 1]);
        g.c[0] += g.c[k];
        g.f.rho[0] += g.f.rho[k];
    }
    T v2 = 0;
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        if (G.fixedV) g.f.v[d] = T(bc.vel_value[patch][d]);
        else g.f.v[d] = (G.reflect && d == axis) ? -w.f.v[d] : w.f.v[d];
        g.f.m[d] = g.f.v[d] * g.f.rho[0];
        v2 += g.f.v[d] * g.f.v[d];
    }
    g.f.p = G.fixedP ? T(bc.p_value[patch]) : w.f.p;
    mixtureG1<T, NS, NMOM>(mp, g);
    g.Uv = g.f.p / g.g1;
    g.f.E = g.Uv + T(0.5) * g.f.rho[0] * v2;
    g.f.cs = sqrt(g.g1 * (g.Uv + g.f.p) / g.f.rho[0]);
}

// Adds the owner's c, v, p adjoints implied by the ghost's adjoint b into wb.
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void ghostReverse(const MixParams& mp, int axis, const Ghost<T, NS, NMOM>& G,
                                             const FBar<T, NS, NMOM>& b, WBar<T, NS, NMOM>& wb) {
    const WState<T, NS, NMOM>& g = G.g;
    const T inv = T(1) / g.f.rho[0];
    T rho0bar = b.rho[0], pbar = b.p, g1bar = 0;
    // cs = sqrt(g1 (Uv + p) / rho)
    const T qbar = b.cs / (T(2) * g.f.cs);
    g1bar += qbar * (g.Uv + g.f.p) * inv;
    T Uvbar = qbar * g.g1 * inv;
    pbar += qbar * g.g1 * inv;
    rho0bar -= qbar * g.f.cs * g.f.cs * inv;
    // E = Uv + rho |v|^2 / 2
    Uvbar += b.E;
    T v2 = 0;
    T vbar[NMOM];
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        v2 += g.f.v[d] * g.f.v[d];
        vbar[d] = b.v[d] + b.E * g.f.rho[0] * g.f.v[d];
    }
    rho0bar += b.E * T(0.5) * v2;
    // m = v rho
#pragma unroll
    for (int d = 0; d < NMOM; ++d) {
        vbar[d] += b.m[d] * g.f.rho[0];
        rho0bar += b.m[d] * g.f.v[d];
    }
    // Uv = p / g1
    pbar += Uvbar / g.g1;
    g1bar -= Uvbar * g.f.p / (g.g1 * g.g1);
    T cbar[NS + 1];
#pragma unroll
    for (int k = 0; k <= NS; ++k) cbar[k] = 0;
    g1Reverse<T, NS, NMOM>(mp, g, g1bar, cbar);
    // rho = sum rho_k, rho_k = c_k M_k
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        cbar[k] += (b.rho[k] + rho0bar) * T(mp.M[k - 1]);
        if (!G.fixedC[k - 1]) wb.c[k] += cbar[k];
    }
    if (!G.fixedP) wb.f.p += pbar;
    if (!G.fixedV) {
#pragma unroll
        for (int d = 0; d < NMOM; ++d) wb.f.v[d] += (G.reflect && d == axis) ? -vbar[d] : vbar[d];
    }
}

// Reverse of the HLLC / HLL flux through a face with normal +e_axis between L and R.  Fb is the
// flux adjoint in packed order.  Adds into Lb and Rb.
template <typename T, int NS, int NMOM>
__device__ __forceinline__ void fluxReverse(int flux, int axis, const FState<T, NS, NMOM>& L,
                                            const FState<T, NS, NMOM>& R, const T* Fb, FBar<T, NS, NMOM>& Lb,
                                            FBar<T, NS, NMOM>& Rb) {
    auto FrB = [&](int k) -> T { return k == 0 ? Fb[NS] : Fb[k - 1]; };
    const T* FmB = Fb + NS + 1;
    const T FEB = Fb[NS + 1 + NMOM];
    const T uL = L.v[axis], uR = R.v[axis];
    const T aL = uL - L.cs, aR = uR - R.cs;
    const bool minR = aR < aL;  // std::min returns its second argument only when strictly smaller
    const T SL = minR ? aR : aL;
    const T bL = uL + L.cs, bR = uR + R.cs;
    const bool maxR = bL < bR;  // std::max returns its second argument when the first is smaller
    const T SR = maxR ? bR : bL;
    const T rL = L.rho[0], rR = R.rho[0];
    T uLb = 0, uRb = 0, SLb = 0, SRb = 0, rLb = 0, rRb = 0;
    // adjoint of a one-sided (supersonic) flux f(W) = (rho u, m u + n p, (E + p) u)
    auto full = [&](const FState<T, NS, NMOM>& W, FBar<T, NS, NMOM>& Wb, T u, T& ub) {
#pragma unroll
        for (int k = 0; k <= NS; ++k) {
            ub += FrB(k) * W.rho[k];
            Wb.rho[k] += FrB(k) * u;
        }
#pragma unroll
        for (int d = 0; d < NMOM; ++d) {
            Wb.m[d] += FmB[d] * u;
            ub += FmB[d] * W.m[d];
        }
        Wb.p += FmB[axis];
        ub += FEB * (W.E + W.p);
        Wb.E += FEB * u;
        Wb.p += FEB * u;
    };
    if (flux == FV_FLUX_HLLC) {
        const T num = R.p - L.p + rL * uL * (SL - uL) - rR * uR * (SR - uR);
        const T dnm = rL * (SL - uL) - rR * (SR - uR);
        const T Sc = num / dnm;
        if (SL >= T(0)) {
            full(L, Lb, uL, uLb);
        } else if (!(Sc >= T(0)) && !(SR > T(0))) {
            full(R, Rb, uR, uRb);
        } else {
            // the star flux F = f(W) + S (W* - W) of the side W the contact leaves (Sc >= 0: left),
            // evaluated once on the selected side so that a warp does not run both
            const bool left = Sc >= T(0);
            const FState<T, NS, NMOM> W = select<T, NS, NMOM>(left, L, R);
            const T u = left ? uL : uR;
            const T S = left ? SL : SR;
            const T P = T(0.5) * (L.p + R.p + rL * (SL - uL) * (Sc - uL) + rR * (SR - uR) * (Sc - uR));
            FBar<T, NS, NMOM> Wb;
            zero<T, NS, NMOM>(Wb);
            T ub = 0, Sb = 0, Scb = 0, Pb = 0;
            const T fac = S - u;
            const T den = T(1) / (S - Sc);
            T facb = 0, denb = 0;
#pragma unroll
            for (int k = 0; k <= NS; ++k) {
                const T F = FrB(k);
                const T rs = W.rho[k] * fac * den;
                Sb += F * (rs - W.rho[k]);
                Wb.rho[k] += F * (u - S);
                ub += F * W.rho[k];
                const T rsb = F * S;
                Wb.rho[k] += rsb * fac * den;
                facb += rsb * W.rho[k] * den;
                denb += rsb * W.rho[k] * fac;
            }
#pragma unroll
            for (int d = 0; d < NMOM; ++d) {
                const T F = FmB[d];
                const T nd = d == axis ? T(1) : T(0);
                const T Am = W.m[d] * fac - nd * (W.p - P);
                const T ms = Am * den;
                Sb += F * (ms - W.m[d]);
                Wb.m[d] += F * (u - S);
                ub += F * W.m[d];
                Wb.p += F * nd;
                const T msb = F * S;
                Wb.m[d] += msb * fac * den;
                facb += msb * W.m[d] * den;
                Wb.p -= msb * nd * den;
                Pb += msb * nd * den;
                denb += msb * Am;
            }
            {
                const T F = FEB;
                const T Be = W.E * fac - W.p * u + P * Sc;
                const T Es = Be * den;
                Sb += F * (Es - W.E);
                Wb.E += F * (u - S);
                Wb.p += F * u;
                ub += F * (W.E + W.p);
                const T Esb = F * S;
                Wb.E += Esb * fac * den;
                facb += Esb * W.E * den;
                Wb.p -= Esb * u * den;
                ub -= Esb * W.p * den;
                Pb += Esb * Sc * den;
                Scb += Esb * P * den;
                denb += Esb * Be;
            }
            Sb += facb;
            ub -= facb;
            Sb -= denb * den * den;
            Scb += denb * den * den;
            addIf<T, NS, NMOM>(Lb, Wb, left);
            addIf<T, NS, NMOM>(Rb, Wb, !left);
            if (left) { uLb += ub; SLb += Sb; } else { uRb += ub; SRb += Sb; }
            // P = (pL + pR + rL (SL - uL)(Sc - uL) + rR (SR - uR)(Sc - uR)) / 2
            const T h = T(0.5) * Pb;
            Lb.p += h;
            Rb.p += h;
            rLb += h * (SL - uL) * (Sc - uL);
            SLb += h * rL * (Sc - uL);
            Scb += h * rL * (SL - uL);
            uLb -= h * rL * ((Sc - uL) + (SL - uL));
            rRb += h * (SR - uR) * (Sc - uR);
            SRb += h * rR * (Sc - uR);
            Scb += h * rR * (SR - uR);
            uRb -= h * rR * ((Sc - uR) + (SR - uR));
            // Sc = num / dnm
            const T numb = Scb / dnm, dnmb = -Scb * Sc / dnm;
            Rb.p += numb;
            Lb.p -= numb;
            rLb += numb * uL * (SL - uL);
            uLb += numb * rL * (SL - T(2) * uL);
            SLb += numb * rL * uL;
            rRb -= numb * uR * (SR - uR);
            uRb -= numb * rR * (SR - T(2) * uR);
            SRb -= numb * rR * uR;
            rLb += dnmb * (SL - uL);
            SLb += dnmb * rL;
            uLb -= dnmb * rL;
            rRb -= dnmb * (SR - uR);
            SRb -= dnmb * rR;
            uRb += dnmb * rR;
        }
    } else {
        if (SL >= T(0)) {
            full(L, Lb, uL, uLb);
        } else if (SR > T(0)) {
            // F = (SR fL - SL fR + SR SL (qR - qL)) / (SR - SL)
            const T den = T(1) / (SR - SL);
            auto term = [&](T fL, T fR, T qL, T qR, T F, T& fLb, T& fRb, T& qLb, T& qRb) {
                const T Fv = (SR * fL - SL * fR + SR * SL * (qR - qL)) * den;
                fLb += F * SR * den;
                fRb -= F * SL * den;
                qRb += F * SR * SL * den;
                qLb -= F * SR * SL * den;
                SRb += F * ((fL + SL * (qR - qL)) - Fv) * den;
                SLb += F * ((SR * (qR - qL) - fR) + Fv) * den;
            };
#pragma unroll
            for (int k = 0; k <= NS; ++k) {
                T fLb = 0, fRb = 0;
                term(uL * L.rho[k], uR * R.rho[k], L.rho[k], R.rho[k], FrB(k), fLb, fRb, Lb.rho[k], Rb.rho[k]);
                uLb += fLb * L.rho[k];
                Lb.rho[k] += fLb * uL;
                uRb += fRb * R.rho[k];
                Rb.rho[k] += fRb * uR;
            }
#pragma unroll
            for (int d = 0; d < NMOM; ++d) {
                const T nd = d == axis ? T(1) : T(0);
                T fLb = 0, fRb = 0;
                term(L.m[d] * uL + nd * L.p, R.m[d] * uR + nd * R.p, L.m[d], R.m[d], FmB[d], fLb, fRb, Lb.m[d],
                     Rb.m[d]);
                Lb.m[d] += fLb * uL;
                uLb += fLb * L.m[d];
                Lb.p += fLb * nd;
                Rb.m[d] += fRb * uR;
                uRb += fRb * R.m[d];
                Rb.p += fRb * nd;
            }
            T fLb = 0, fRb = 0;
            term(uL * (L.E + L.p), uR * (R.E + R.p), L.E, R.E, FEB, fLb, fRb, Lb.E, Rb.E);
            uLb += fLb * (L.E + L.p);
            Lb.E += fLb * uL;
            Lb.p += fLb * uL;
            uRb += fRb * (R.E + R.p);
            Rb.E += fRb * uR;
            Rb.p += fRb * uR;
        } else {
            full(R, Rb, uR, uRb);
        }
    }
    // wave speeds SL = min(uL - cL, uR - cR), SR = max(uL + cL, uR + cR)
    if (minR) { uRb += SLb; Rb.cs -= SLb; } else { uLb += SLb; Lb.cs -= SLb; }
    if (maxR) { uRb += SRb; Rb.cs += SRb; } else { uLb += SRb; Lb.cs += SRb; }
    Lb.rho[0] += rLb;
    Rb.rho[0] += rRb;
    Lb.v[axis] += uLb;
    Rb.v[axis] += uRb;
}

// One adjoint step: lamOut = (dU^{n+1}/dU^n)^T lamIn + objGain * dt_{n-1} * dW/dU^n (n >= 1),
// with W = objScale * sum_cells X_h (1 - X_h) * (cell area in 2D, volume in 3D).
struct AdjParams {
    const double* U;        // U^n, storage order, stride P.stride
    const double* lamIn;    // adjoint of U^{n+1}
    double* lamOut;         // adjoint of U^n
    const StepRecord* rec;  // rec[n]: the step U^n -> U^{n+1}
    long long n;
    double objGain;         // 0: no objective term
    double objScale;
    int heavy;
    int rows;               // rows per tile along the marching axis (<= 0: the launcher's choice)
};

// Storage field of packed index i.
template <int NS, int NMOM>
__device__ __forceinline__ int storageField(int i) {
    return i <= NS + NMOM ? i : NS + 4;
}

template <int NS, int NMOM>
__device__ __forceinline__ void loadPacked(const StepParams& P, const double* __restrict__ A, long long cell,
                                           double* u) {
    const long long st = P.stride;
#pragma unroll
    for (int i = 0; i < NS + 2 + NMOM; ++i) u[i] = A[storageField<NS, NMOM>(i) * st + cell];
}

// Dynamic shared memory of k_adjoint per in-plane thread slot: the published face state, the
// adjoint divided by the cell volume, and the face-state adjoints handed over by the low
// neighbours (along x, and along y in 3D).  Layout [array][field][BY][BX].
template <typename T, int NS, int D, int NMOM, int BX, int BY>
constexpr size_t adjointExchangeBytes() {
    return (sizeof(T) * size_t(BX) * BY *
                (size_t(fsSize<NS, NMOM>()) + (NS + 2 + NMOM) + fsSize<NS, NMOM>() * (D == 3 ? 2 : 1)) +
            15) / 16 * 16;
}

// FP64 2D tiles fetch the next rows' conserved values and adjoint (2 NL doubles per column) into
// a ring of kAdjRingSlots rows with cp.async, one row ahead of their use.  Layout
// [slot][value][BX].  FP32 and 3D tiles read them directly (in FP32 the ring measured no
// faster: the kernel's stalls there are arithmetic dependencies, not the row loads).
constexpr int kAdjRingSlots = 2;
template <typename T, int D>
constexpr bool adjointRing() { return D == 2 && sizeof(T) == 8; }
template <typename T, int NS, int D, int NMOM, int BX, int BY>
constexpr size_t adjointRingBytes() {
    return adjointRing<T, D>() ? sizeof(double) * size_t(kAdjRingSlots) * 2 * (NS + 2 + NMOM) * BX * BY : 0;
}

template <typename T, int NS, int D, int NMOM, int BX, int BY>
constexpr size_t adjointSmemBytes() {
    return adjointExchangeBytes<T, NS, D, NMOM, BX, BY>() + adjointRingBytes<T, NS, D, NMOM, BX, BY>();
}

__device__ __forceinline__ void ringCopy8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void ringCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ringWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// CTAs per SM the register budget of k_adjoint is sized for: 384 threads per SM (170 registers)
// in FP64, 512 (128 registers) with FP32 face arithmetic.
template <typename T, int BX, int BY>
constexpr int adjointMinBlocks() {
    return (sizeof(T) == 8 ? 256 : 512) / (BX * BY) > 0 ? (sizeof(T) == 8 ? 256 : 512) / (BX * BY) : 1;
}

// The adjoint march: the same tiling as the forward march (in-plane halo of one cell, marching
// along y in 2D and z in 3D), one thread per in-plane column.  Every face is reversed once: the
// x (and y) faces by the thread of their low cell, which hands the high cell's share of the
// face-state adjoint over through shared memory; the marching-axis faces in registers, carrying
// the high cell's share to the next row.  Each cell's closure is evaluated and reversed once.
template <typename T, int NS, int D, int NMOM, int BX, int BY>
__global__ void __launch_bounds__(BX * BY, adjointMinBlocks<T, BX, BY>()) k_adjoint(const StepParams P, const AdjParams A) {
    constexpr int NL = NS + 2 + NMOM;
    constexpr int NFS = fsSize<NS, NMOM>();
    constexpr int MA = D - 1;
    constexpr int SL = BX * BY;
    using FS = FState<T, NS, NMOM>;
    using FB = FBar<T, NS, NMOM>;
    using WS = WState<T, NS, NMOM>;
    using WB = WBar<T, NS, NMOM>;
    extern __shared__ __align__(16) unsigned char adj_smem[];
    T* sF = reinterpret_cast<T*>(adj_smem);
    T* sL = sF + NFS * SL;
    T* sBx = sL + NL * SL;
    T* sBy = sBx + NFS * SL;  // 3D only
    constexpr bool RING = adjointRing<T, D>();
    double* sRing = reinterpret_cast<double*>(adj_smem + adjointExchangeBytes<T, NS, D, NMOM, BX, BY>());

    const int tx = threadIdx.x, ty = D == 3 ? threadIdx.y : 0;
    const int slot = ty * BX + tx;
    const int tileX = blockIdx.x, tileY = D == 3 ? blockIdx.y : 0, tileZ = D == 3 ? blockIdx.z : blockIdx.y;
    const int nx = P.n[0], ny = P.n[1], nm = P.n[MA];
    const bool perX = P.periodic[0], perY = D == 3 && P.periodic[1], perM = P.periodic[MA];
    const int X = tileX * (BX - 2) - 1 + tx;
    const int Y = D == 3 ? tileY * (BY - 2) - 1 + ty : 0;
    const int z0 = tileZ * A.rows, z1 = min(z0 + A.rows, nm);

    int cx = X, cy = Y;
    bool has = true;
    if (X < 0 || X >= nx) {
        if (perX && X >= -1 && X <= nx) cx = X < 0 ? X + nx : X - nx;
        else has = false;
    }
    if (D == 3 && (Y < 0 || Y >= ny)) {
        if (perY && Y >= -1 && Y <= ny) cy = Y < 0 ? Y + ny : Y - ny;
        else has = false;
    }
    auto interiorAt = [&](int t, int u) {
        const int Xt = tileX * (BX - 2) - 1 + t;
        const int Yu = D == 3 ? tileY * (BY - 2) - 1 + u : 0;
        return t >= 1 && t <= BX - 2 && Xt < nx && (D == 2 || (u >= 1 && u <= BY - 2 && Yu < ny));
    };
    const bool interior = interiorAt(tx, ty);
    const bool doX = has && tx <= BX - 2 && (interior || interiorAt(tx + 1, ty));
    const bool doY = D == 3 && has && ty <= BY - 2 && (interior || interiorAt(tx, ty + 1));

    const StepRecord rec = A.rec[A.n];
    const double dt = rec.dt;
    const bool objTerm = A.objGain != 0.0 && A.n >= 1;
    const double objW = objTerm ? A.objGain * A.rec[A.n - 1].dt * A.objScale : 0.0;
    const double hx = has ? P.geo.h[0][cx] : 1.0;
    const double hy = D == 3 ? (has ? P.geo.h[1][cy] : 1.0) : 0.0;
    const double Lz = P.ext[2];
    // face areas of this column's cell and the inverse cell volume of a row of height hm
    // (mesh.cpp)
    double Sx = 0, Sy = 0, Sm = 0;
    auto invVol = [&](double hm) -> double { return D == 2 ? 1.0 / (hx * hm * Lz) : 1.0 / (hx * hy * hm); };
    auto areas = [&](double hm) {
        if (D == 2) {
            Sx = Lz * hm;
            Sm = hx * Lz;
        } else {
            Sx = hm * hy;
            Sy = hx * hm;
            Sm = hx * hy;
        }
    };
    auto cellAt = [&](int zm) -> long long { return D == 2 ? cellIndex(P, cx, zm, 0) : cellIndex(P, cx, cy, zm); };
    auto wrapM = [&](int zm, bool& ok) -> int {
        ok = true;
        if (zm < 0) { if (perM) return zm + nm; ok = false; return 0; }
        if (zm >= nm) { if (perM) return zm - nm; ok = false; return 0; }
        return zm;
    };
    const MixParams& mp = P.mix;
    auto loadW = [&](long long cell, WS& w) {
        double u[NL];
        loadPacked<NS, NMOM>(P, A.U, cell, u);
        T ut[NL];
#pragma unroll
        for (int i = 0; i < NL; ++i) ut[i] = T(u[i]);
        wForward<T, NS, NMOM>(mp, ut, w);
    };
    // flux adjoint of a face from the volume-scaled adjoints of its two sides
    auto faceBar = [&](double dtS, const T* lvR, const T* lvL, T* Fb) {
#pragma unroll
        for (int i = 0; i < NL; ++i) Fb[i] = T(dtS) * (lvR[i] - lvL[i]);
    };
    const T zeros[NL] = {};
    // ring slot of loop row z (2D): the next rows' values, fetched a row ahead
    auto ringSlot = [&](int z) { return sRing + (size_t)(z & (kAdjRingSlots - 1)) * 2 * NL * SL + slot; };
    auto ringIssue = [&](int z, long long cell) {
        double* dst = ringSlot(z);
        const long long st = P.stride;
#pragma unroll
        for (int i = 0; i < NL; ++i) {
            ringCopy8(dst + i * SL, A.U + storageField<NS, NMOM>(i) * st + cell);
            ringCopy8(dst + (NL + i) * SL, A.lamIn + storageField<NS, NMOM>(i) * st + cell);
        }
    };

    WS Wc, Wn;
    WB Bc;
    FB Bn;
    // lvc, lvn: the adjoint of rows z and z + 1 divided by the cell volume (face arithmetic); the
    // FP64 adjoint of row z is read again for its output rather than kept through the row
    T lvc[NL], lvn[NL];
    double ivc = 1, ivn = 1;
    double hmC = P.geo.h[MA][z0 < z1 ? z0 : 0], hmN = hmC;  // heights of rows z and z + 1
    zero<T, NS, NMOM>(Bc);
    zero<T, NS, NMOM>(Bn);
    bool ok;

    // ---- prologue: row z0 and the face below it
    if (has && z0 < z1) {
        loadW(cellAt(z0), Wc);
        double l0[NL];
        loadPacked<NS, NMOM>(P, A.lamIn, cellAt(z0), l0);
        ivc = invVol(hmC);
#pragma unroll
        for (int i = 0; i < NL; ++i) lvc[i] = T(l0[i] * ivc);
        areas(hmC);
        if (interior) {
            const int zb = wrapM(z0 - 1, ok);
            T Fb[NL];
            FB Bb;
            zero<T, NS, NMOM>(Bb);
            if (ok) {
                double lb[NL];
                loadPacked<NS, NMOM>(P, A.lamIn, cellAt(zb), lb);
                const double ivb = invVol(P.geo.h[MA][zb]);
                T lvb[NL];
#pragma unroll
                for (int i = 0; i < NL; ++i) lvb[i] = T(lb[i] * ivb);
                WS Wb;
                loadW(cellAt(zb), Wb);
                faceBar(dt * Sm, lvc, lvb, Fb);
                fluxReverse<T, NS, NMOM>(P.flux, MA, Wb.f, Wc.f, Fb, Bb, Bc.f);
            } else {
                Ghost<T, NS, NMOM> G;
                ghostForward<T, NS, NMOM>(mp, P.bc, D == 2 ? FV_PATCH_RIGHT : FV_PATCH_BOTTOM, MA, Wc, G);
                faceBar(dt * Sm, lvc, zeros, Fb);
                fluxReverse<T, NS, NMOM>(P.flux, MA, G.g.f, Wc.f, Fb, Bb, Bc.f);
                ghostReverse<T, NS, NMOM>(mp, MA, G, Bb, Bc);
            }
        }
    }

    if constexpr (RING) {
        if (z0 < z1) {
            const int zq = wrapM(z0 + 1, ok);
            if (has && ok) ringIssue(z0 + 1, cellAt(zq));
        }
        ringCommit();
    }

    for (int z = z0; z < z1; ++z) {
        const int zn = wrapM(z + 1, ok);
        const bool hasNext = has && ok;
        if (ok) hmN = P.geo.h[MA][zn];
        areas(hmC);
        if constexpr (RING) {
            bool okq;
            const int zq = wrapM(z + 2, okq);
            if (has && okq && z + 1 < z1) ringIssue(z + 2, cellAt(zq));
            ringCommit();
            ringWait<1>();  // the values of row z + 1 have landed
        }
        if (hasNext) {
            double ln[NL];
            if constexpr (RING) {
                const double* src = ringSlot(z + 1);
                T ut[NL];
#pragma unroll
                for (int i = 0; i < NL; ++i) {
                    ut[i] = T(src[i * SL]);
                    ln[i] = src[(NL + i) * SL];
                }
                wForward<T, NS, NMOM>(mp, ut, Wn);
            } else {
                loadW(cellAt(zn), Wn);
                loadPacked<NS, NMOM>(P, A.lamIn, cellAt(zn), ln);
            }
            if constexpr (sizeof(T) == 4) {
                // FP32 face arithmetic: the volume scaling of the adjoint in FP32 as well
                const T ivf = T(1) / (T(hx) * T(hmN) * T(D == 2 ? Lz : hy));
#pragma unroll
                for (int i = 0; i < NL; ++i) lvn[i] = T(ln[i]) * ivf;
            } else {
                ivn = invVol(hmN);
#pragma unroll
                for (int i = 0; i < NL; ++i) lvn[i] = T(ln[i] * ivn);
            }
        }
        // publish this row
        if (has) {
            pack<T, NS, NMOM>(Wc.f, sF + slot, SL);
#pragma unroll
            for (int i = 0; i < NL; ++i) sL[i * SL + slot] = lvc[i];
        }
#pragma unroll
        for (int i = 0; i < NFS; ++i) {
            sBx[i * SL + slot] = T(0);
            if (D == 3) sBy[i * SL + slot] = T(0);
        }
        __syncthreads();
        // x face X + 1/2 (the point wall when X = nx - 1)
        if (doX) {
            const bool rReal = !(X == nx - 1 && !perX);
            T Fb[NL];
            FB BL, BR;
            zero<T, NS, NMOM>(BL);
            zero<T, NS, NMOM>(BR);
            if (rReal) {
                FS R;
                unpack<T, NS, NMOM>(sF + slot + 1, SL, R);
                T lvR[NL];
#pragma unroll
                for (int i = 0; i < NL; ++i) lvR[i] = sL[i * SL + slot + 1];
                faceBar(dt * Sx, lvR, lvc, Fb);
                fluxReverse<T, NS, NMOM>(P.flux, 0, Wc.f, R, Fb, BL, BR);
                if (interiorAt(tx + 1, ty)) pack<T, NS, NMOM>(BR, sBx + slot + 1, SL);
            } else {
                Ghost<T, NS, NMOM> G;
                ghostForward<T, NS, NMOM>(mp, P.bc, FV_PATCH_POINT, 0, Wc, G);
                faceBar(dt * Sx, zeros, lvc, Fb);
                fluxReverse<T, NS, NMOM>(P.flux, 0, Wc.f, G.g.f, Fb, BL, BR);
                ghostReverse<T, NS, NMOM>(mp, 0, G, BR, Bc);
            }
            if (interior) add<T, NS, NMOM>(Bc.f, BL);
        }
        // tail wall below X = 0
        if (interior && X == 0 && !perX) {
            Ghost<T, NS, NMOM> G;
            ghostForward<T, NS, NMOM>(mp, P.bc, FV_PATCH_TAIL, 0, Wc, G);
            T Fb[NL];
            FB BG;
            zero<T, NS, NMOM>(BG);
            faceBar(dt * Sx, lvc, zeros, Fb);
            fluxReverse<T, NS, NMOM>(P.flux, 0, G.g.f, Wc.f, Fb, BG, Bc.f);
            ghostReverse<T, NS, NMOM>(mp, 0, G, BG, Bc);
        }
        if (D == 3) {
            if (doY) {
                const bool rReal = !(Y == ny - 1 && !perY);
                T Fb[NL];
                FB BL, BR;
                zero<T, NS, NMOM>(BL);
                zero<T, NS, NMOM>(BR);
                if (rReal) {
                    FS R;
                    unpack<T, NS, NMOM>(sF + slot + BX, SL, R);
                    T lvR[NL];
#pragma unroll
                    for (int i = 0; i < NL; ++i) lvR[i] = sL[i * SL + slot + BX];
                    faceBar(dt * Sy, lvR, lvc, Fb);
                    fluxReverse<T, NS, NMOM>(P.flux, 1, Wc.f, R, Fb, BL, BR);
                    if (interiorAt(tx, ty + 1)) pack<T, NS, NMOM>(BR, sBy + slot + BX, SL);
                } else {
                    Ghost<T, NS, NMOM> G;
                    ghostForward<T, NS, NMOM>(mp, P.bc, FV_PATCH_LEFT, 1, Wc, G);
                    faceBar(dt * Sy, zeros, lvc, Fb);
                    fluxReverse<T, NS, NMOM>(P.flux, 1, Wc.f, G.g.f, Fb, BL, BR);
                    ghostReverse<T, NS, NMOM>(mp, 1, G, BR, Bc);
                }
                if (interior) add<T, NS, NMOM>(Bc.f, BL);
            }
            if (interior && Y == 0 && !perY) {
                Ghost<T, NS, NMOM> G;
                ghostForward<T, NS, NMOM>(mp, P.bc, FV_PATCH_RIGHT, 1, Wc, G);
                T Fb[NL];
                FB BG;
                zero<T, NS, NMOM>(BG);
                faceBar(dt * Sy, lvc, zeros, Fb);
                fluxReverse<T, NS, NMOM>(P.flux, 1, G.g.f, Wc.f, Fb, BG, Bc.f);
                ghostReverse<T, NS, NMOM>(mp, 1, G, BG, Bc);
            }
        }
        // marching-axis face z + 1/2 (the high wall when z is the last row)
        if (interior) {
            T Fb[NL];
            if (hasNext) {
                faceBar(dt * Sm, lvn, lvc, Fb);
                fluxReverse<T, NS, NMOM>(P.flux, MA, Wc.f, Wn.f, Fb, Bc.f, Bn);
            } else {
                Ghost<T, NS, NMOM> G;
                ghostForward<T, NS, NMOM>(mp, P.bc, D == 2 ? FV_PATCH_LEFT : FV_PATCH_TOP, MA, Wc, G);
                faceBar(dt * Sm, zeros, lvc, Fb);
                FB BG;
                zero<T, NS, NMOM>(BG);
                fluxReverse<T, NS, NMOM>(P.flux, MA, Wc.f, G.g.f, Fb, Bc.f, BG);
                ghostReverse<T, NS, NMOM>(mp, MA, G, BG, Bc);
            }
        }
        __syncthreads();
        if (interior) {
            unpackAdd<T, NS, NMOM>(sBx + slot, SL, Bc.f);
            if (D == 3) unpackAdd<T, NS, NMOM>(sBy + slot, SL, Bc.f);
            T ub[NL];
            wReverse<T, NS, NMOM>(mp, Wc, Bc, ub);
            const long long ic = cellAt(z);
            double lc[NL];
            loadPacked<NS, NMOM>(P, A.lamIn, ic, lc);
            double out[NL];
#pragma unroll
            for (int i = 0; i < NL; ++i) out[i] = lc[i] + double(ub[i]);
            if (P.gravity) {
                // E += dt m.g, m_d += dt g_d rho (Advection.cpp:424-431 with v = m / rho)
                double r0bar = 0;
#pragma unroll
                for (int d = 0; d < NMOM; ++d) {
                    out[NS + 1 + d] += dt * rec.g[d] * lc[NS + 1 + NMOM];
                    r0bar += dt * rec.g[d] * lc[NS + 1 + d];
                }
                out[NS] += r0bar;
            }
            if (objTerm) {
                if constexpr (sizeof(T) == 4) {
                    // the objective's gradient term in the face arithmetic, added to the FP64 sum
                    const T c0 = Wc.c[0];
                    T ch = 0;
#pragma unroll
                    for (int k = 0; k < NS; ++k) ch = k == A.heavy ? Wc.c[k + 1] : ch;
                    const T ic0 = T(1) / c0;
                    const T Xh = ch * ic0;
                    const T meas = D == 2 ? T(hx * hmC) : T(hx * hy * hmC);
                    const T dWdX = T(objW) * meas * (T(1) - T(2) * Xh);
#pragma unroll
                    for (int k = 0; k < NS; ++k)
                        out[k] += double(dWdX * ((k == A.heavy ? T(1) : T(0)) - Xh) * ic0 * T(mp.invM[k]));
                } else {
                    const double c0 = double(Wc.c[0]);
                    double ch = 0;
#pragma unroll
                    for (int k = 0; k < NS; ++k) ch = k == A.heavy ? double(Wc.c[k + 1]) : ch;
                    const double Xh = ch / c0;
                    const double meas = D == 2 ? hx * hmC : hx * hy * hmC;
                    const double dWdX = objW * meas * (1.0 - 2.0 * Xh);
#pragma unroll
                    for (int k = 0; k < NS; ++k) out[k] += dWdX * ((k == A.heavy ? 1.0 : 0.0) - Xh) / c0 * mp.invM[k];
                }
            }
            const long long st = P.stride;
#pragma unroll
            for (int i = 0; i < NL; ++i) A.lamOut[storageField<NS, NMOM>(i) * st + ic] = out[i];
        }
        // roll the marching window
        if (hasNext) {
            Wc = Wn;
#pragma unroll
            for (int i = 0; i < NL; ++i) lvc[i] = lvn[i];
            ivc = ivn;
        }
        hmC = hmN;
        Bc.f = Bn;
#pragma unroll
        for (int k = 0; k <= NS; ++k) Bc.c[k] = 0;
        Bc.g1 = 0;
        zero<T, NS, NMOM>(Bn);
        __syncthreads();
    }
    if constexpr (RING) ringWait<0>();  // no copy outlives the tile
}

}  // namespace adj
}  // namespace fv
