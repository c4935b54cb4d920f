// fv_warp2d.cuh -- warp-strip march: the FP32-flux step on a 2D mesh whose limiter gives zero
// slopes (the fused march of fv_kernels.cuh, laid out for the least instructions per cell).
//
// Each warp owns a strip of 30 columns (lanes 1..30; lanes 0 and 31 are the halo columns on
// either side) and marches along y over `rows` rows.  Per row a lane
//   * recovers the FP32 face state W of the next row from its FP64 conserved values, which were
//     loaded one row earlier into registers (coalesced 8-byte loads, 32 lanes = 256 bytes);
//   * takes W of lane - 1 by shuffle and computes the flux through its low x face, and the flux
//     through the face between its row and the next (kept in registers for the next row);
//   * takes the high-x-face flux from lane + 1 by shuffle and updates its cell in FP64
//     (U_new = U_old - dt * div F, with the gravity source of Advection.cpp:424-431);
//   * derives the CFL signal (|v| + c) / min edge of the updated cell.
// Warps never wait for one another: no shared-memory exchange and no CTA barrier; each warp
// writes its own CFL partial maximum.
//
// Arithmetic follows the FP32-flux contract of the CTA march (same HLLC / HLL, FP32 closure,
// FP64 accumulation), with the area-to-volume ratios of the uniform-axis cells written as
// 1 / h (the face area over the cell volume); results agree with the FP64 oracle to the FP32
// tolerance of this mode.
#pragma once

#include "fv_kernels.cuh"

// Resident threads per SM the register budget of the warp-strip march is sized for.
#ifndef FV_WARP2D_THREADS_PER_SM
#define FV_WARP2D_THREADS_PER_SM 512
#endif

namespace fv {

constexpr int kWarp2dThreadsPerSM = FV_WARP2D_THREADS_PER_SM;

// FP32 state of one cell as its faces see it (2 momentum components).
template <int NS>
struct LeanW {
    float rho[NS + 1];  // rho[0]: mixture density
    float m[2];
    float E, p, cs;
    float v[2];
};

// Scalar fluxes along +e_axis through one face.
template <int NS>
struct LeanF {
    float rho[NS + 1];
    float m[2];
    float E;
};

// Reciprocal (an approximate MUFU reciprocal in the fast-math FP32 units).
__device__ __forceinline__ float rcpf(float x) { return 1.f / x; }

// Float copies of the mixture constants a lane needs.
template <int NS>
struct LeanMix {
    float invM[NS], M[NS], cvOverM[NS], Cv[NS];
    float R;
    float a[NS][NS], b[NS][NS];
};

template <int NS, int EOS>
__device__ __forceinline__ void leanMix(const MixParams& mp, LeanMix<NS>& L) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        L.invM[k] = float(mp.invM[k]);
        L.M[k] = float(mp.M[k]);
        L.Cv[k] = float(mp.Cv[k]);
        L.cvOverM[k] = float(mp.Cv[k] * mp.invM[k]);
    }
    L.R = float(mp.R);
    if (EOS == FV_EOS_VAN_DER_WAALS) {
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                L.a[k][l] = float(mp.a[k][l]);
                L.b[k][l] = float(mp.b[k][l]);
            }
    }
}

// Pressure and squared sound speed of a mixture state (mixtureIdeal / mixtureVanDerWaals with
// Cv_mix = sum X_k Cv_k), from the densities, 1 / rho and the internal energy per volume.
template <int NS, int EOS>
__device__ __forceinline__ void leanEos(const LeanMix<NS>& L, const float* rho, float inv, float Uv, float& p,
                                        float& cs2) {
    float c0 = 0.f, rcv = 0.f;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        c0 = fmaf(rho[k + 1], L.invM[k], c0);
        rcv = fmaf(rho[k + 1], L.cvOverM[k], rcv);
    }
    // R / Cv_mix with Cv_mix = (sum c_k Cv_k) / c0
    const float g1 = L.R * c0 * rcpf(rcv);
    if (EOS == FV_EOS_IDEAL) {
        p = g1 * Uv;
        cs2 = g1 * (Uv + p) * inv;
        return;
    }
    const float ic0 = rcpf(c0);
    float X[NS], am = 0.f, bm = 0.f, Mm = 0.f;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        X[k] = rho[k + 1] * L.invM[k] * ic0;
        Mm = fmaf(X[k], L.M[k], Mm);
    }
#pragma unroll
    for (int k = 0; k < NS; ++k)
#pragma unroll
        for (int l = 0; l < NS; ++l) {
            const float xx = X[k] * X[l];
            am = fmaf(xx, L.a[k][l], am);
            bm = fmaf(xx, L.b[k][l], bm);
        }
    const float acc = am * c0 * c0;
    const float im = rcpf(1.f - c0 * bm);
    p = g1 * (Uv + acc) * im - acc;
    const float ac = am * c0;
    const float dpdrho = (g1 * (2.f * ac * im - bm * (Uv + ac * c0) * im * im) - 2.f * ac) / Mm;
    cs2 = dpdrho + g1 * im * (Uv + p) * inv;
}

// W from the conserved values d[0..NS-1] = rho_k, d[NS] = rho, d[NS+1..NS+2] = m, d[NS+3] = E.
template <int NS, int EOS>
__device__ __forceinline__ void leanClose(const LeanMix<NS>& L, const double* d, LeanW<NS>& W) {
#pragma unroll
    for (int k = 1; k <= NS; ++k) W.rho[k] = float(d[k - 1]);
    W.rho[0] = float(d[NS]);
    W.m[0] = float(d[NS + 1]);
    W.m[1] = float(d[NS + 2]);
    W.E = float(d[NS + 3]);
    const float inv = rcpf(W.rho[0]);
    W.v[0] = W.m[0] * inv;
    W.v[1] = W.m[1] * inv;
    const float Uv = W.E - 0.5f * W.rho[0] * (W.v[0] * W.v[0] + W.v[1] * W.v[1]);
    float cs2;
    leanEos<NS, EOS>(L, W.rho, inv, Uv, W.p, cs2);
    W.cs = sqrtf(cs2);
}

// CFL signal (|v| + c) / min edge of an updated cell from its FP32 state.
template <int NS, int EOS>
__device__ __forceinline__ float leanSignal(const LeanMix<NS>& L, const float* rho, const float* m, float E,
                                            float minLS) {
    const float inv = rcpf(rho[0]);
    const float v0 = m[0] * inv, v1 = m[1] * inv;
    const float vv = v0 * v0 + v1 * v1;
    const float Uv = E - 0.5f * rho[0] * vv;
    float p, cs2;
    leanEos<NS, EOS>(L, rho, inv, Uv, p, cs2);
    return (sqrtf(vv) + sqrtf(cs2)) * minLS;
}

// HLLC / HLL flux through a face normal to AX between the states O (low side) and B (high
// side), along +e_AX.  Same expressions as riemann() in fv_device.cuh; false for NaN speeds.
template <int NS, int AX>
__device__ __forceinline__ bool leanRiemann(int flux, const LeanW<NS>& O, const LeanW<NS>& B, LeanF<NS>& F) {
    const float uO = O.v[AX], uN = B.v[AX];
    // std::min / std::max order: a NaN speed reaches the branch tests and is reported
    const float SO = smin(uO - O.cs, uN - B.cs);
    const float SN = smax(uO + O.cs, uN + B.cs);
    if (flux == FV_FLUX_HLLC) {
        const float dO = O.rho[0] * (SO - uO), dN = B.rho[0] * (SN - uN);
        const float Sc = (B.p - O.p + dO * uO - dN * uN) * rcpf(dO - dN);
        const float PON = 0.5f * (O.p + B.p + dO * (Sc - uO) + dN * (Sc - uN));
        if (SO >= 0.f) {
#pragma unroll
            for (int k = 0; k <= NS; ++k) F.rho[k] = uO * O.rho[k];
#pragma unroll
            for (int d = 0; d < 2; ++d) F.m[d] = O.m[d] * uO + (d == AX ? O.p : 0.f);
            F.E = uO * (O.E + O.p);
        } else if (Sc >= 0.f || SN > 0.f) {
            auto star = [&](const LeanW<NS>& W, float u, float S) {
                const float factor = S - u;
                const float den = rcpf(S - Sc);
                const float fd = factor * den;
#pragma unroll
                for (int k = 0; k <= NS; ++k) F.rho[k] = W.rho[k] * u + S * (W.rho[k] * fd - W.rho[k]);
#pragma unroll
                for (int d = 0; d < 2; ++d) {
                    const float ms = (W.m[d] * factor - (d == AX ? W.p - PON : 0.f)) * den;
                    F.m[d] = W.m[d] * u + (d == AX ? W.p : 0.f) + (ms - W.m[d]) * S;
                }
                const float Es = (W.E * factor - W.p * u + PON * Sc) * den;
                F.E = (W.E + W.p) * u + S * (Es - W.E);
            };
            if (Sc >= 0.f) star(O, uO, SO);
            else star(B, uN, SN);
        } else if (SN <= 0.f) {
#pragma unroll
            for (int k = 0; k <= NS; ++k) F.rho[k] = uN * B.rho[k];
#pragma unroll
            for (int d = 0; d < 2; ++d) F.m[d] = B.m[d] * uN + (d == AX ? B.p : 0.f);
            F.E = uN * (B.E + B.p);
        } else {
            return false;
        }
        return true;
    }
    if (SO >= 0.f) {
#pragma unroll
        for (int k = 0; k <= NS; ++k) F.rho[k] = uO * O.rho[k];
#pragma unroll
        for (int d = 0; d < 2; ++d) F.m[d] = O.m[d] * uO + (d == AX ? O.p : 0.f);
        F.E = uO * (O.E + O.p);
    } else if (SN > 0.f) {
        const float den = rcpf(SN - SO);
#pragma unroll
        for (int k = 0; k <= NS; ++k) F.rho[k] = (SN * uO * O.rho[k] - SO * uN * B.rho[k] + SN * SO * (B.rho[k] - O.rho[k])) * den;
#pragma unroll
        for (int d = 0; d < 2; ++d) {
            const float t1 = (O.m[d] * uO + (d == AX ? O.p : 0.f)) * SN;
            const float t2 = (B.m[d] * uN + (d == AX ? B.p : 0.f)) * SO;
            F.m[d] = ((t1 - t2) + (B.m[d] - O.m[d]) * (SN * SO)) * den;
        }
        F.E = (SN * (uO * (O.E + O.p)) - SO * (uN * (B.E + B.p)) + SN * SO * (B.E - O.E)) * den;
    } else if (SN <= 0.f) {
#pragma unroll
        for (int k = 0; k <= NS; ++k) F.rho[k] = uN * B.rho[k];
#pragma unroll
        for (int d = 0; d < 2; ++d) F.m[d] = B.m[d] * uN + (d == AX ? B.p : 0.f);
        F.E = uN * (B.E + B.p);
    } else {
        return false;
    }
    return true;
}

// ---- paired FP32 arithmetic: one FFMA2 / FADD2 / FMUL2 computes two independent lanes of work
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sel2(bool a, bool b, float2 x, float2 y) {
    return make_float2(a ? x.x : y.x, b ? x.y : y.y);
}

// The two HLLC fluxes a lane computes per row, paired: component .x is the low x face (owner Ox,
// neighbour Bx), component .y the face above the row (owner Oy, neighbour By); momenta as
// normal / tangential pairs.  Without branches: each face takes the flux of the side K the
// contact leaves (the owner when SO >= 0 or Sc >= 0, else the neighbour) plus S_K times the
// star correction where the star region applies -- the cases and expressions of leanRiemann.
// okx / oky are false for NaN speeds.
template <int NS>
__device__ __forceinline__ void hllcPair(const LeanW<NS>& Ox, const LeanW<NS>& Bx, const LeanW<NS>& Oy,
                                         const LeanW<NS>& By, LeanF<NS>& Fx, LeanF<NS>& Fy, bool& okx, bool& oky) {
    const float2 uO = make_float2(Ox.v[0], Oy.v[1]), uN = make_float2(Bx.v[0], By.v[1]);
    const float2 cO = make_float2(Ox.cs, Oy.cs), cN = make_float2(Bx.cs, By.cs);
    const float2 pO = make_float2(Ox.p, Oy.p), pN = make_float2(Bx.p, By.p);
    const float2 a = sub2(uO, cO), b = sub2(uN, cN), c = add2(uO, cO), d = add2(uN, cN);
    const float2 SO = make_float2(smin(a.x, b.x), smin(a.y, b.y));
    const float2 SN = make_float2(smax(c.x, d.x), smax(c.y, d.y));
    const float2 dO = mul2(make_float2(Ox.rho[0], Oy.rho[0]), sub2(SO, uO));
    const float2 dN = mul2(make_float2(Bx.rho[0], By.rho[0]), sub2(SN, uN));
    const float2 num = sub2(fma2(dO, uO, sub2(pN, pO)), mul2(dN, uN));
    const float2 dd = sub2(dO, dN);
    const float2 Sc = mul2(num, make_float2(rcpf(dd.x), rcpf(dd.y)));
    const float2 PON =
        mul2(fma2(dN, sub2(Sc, uN), fma2(dO, sub2(Sc, uO), add2(pO, pN))), make_float2(0.5f, 0.5f));
    const bool supX = SO.x >= 0.f, supY = SO.y >= 0.f;
    const bool ownX = supX || Sc.x >= 0.f, ownY = supY || Sc.y >= 0.f;
    const bool stX = !supX && (Sc.x >= 0.f || SN.x > 0.f), stY = !supY && (Sc.y >= 0.f || SN.y > 0.f);
    okx = supX || stX || SN.x <= 0.f;
    oky = supY || stY || SN.y <= 0.f;
    // side K the contact leaves
    const float2 u = sel2(ownX, ownY, uO, uN), S = sel2(ownX, ownY, SO, SN), p = sel2(ownX, ownY, pO, pN);
    const float2 E = sel2(ownX, ownY, make_float2(Ox.E, Oy.E), make_float2(Bx.E, By.E));
    const float2 mn = sel2(ownX, ownY, make_float2(Ox.m[0], Oy.m[1]), make_float2(Bx.m[0], By.m[1]));
    const float2 mt = sel2(ownX, ownY, make_float2(Ox.m[1], Oy.m[0]), make_float2(Bx.m[1], By.m[0]));
    const float2 factor = sub2(S, u);
    const float2 sd = sub2(S, Sc);
    const float2 den = make_float2(stX ? rcpf(sd.x) : 0.f, stY ? rcpf(sd.y) : 0.f);
    const float2 w = make_float2(stX ? S.x : 0.f, stY ? S.y : 0.f);
    const float2 fd = mul2(factor, den);
#pragma unroll
    for (int k = 0; k <= NS; ++k) {
        const float2 r = sel2(ownX, ownY, make_float2(Ox.rho[k], Oy.rho[k]), make_float2(Bx.rho[k], By.rho[k]));
        const float2 f = fma2(w, sub2(mul2(r, fd), r), mul2(r, u));
        Fx.rho[k] = f.x;
        Fy.rho[k] = f.y;
    }
    // normal momentum: mn u + p + w ((mn factor - (p - PON)) den - mn)
    const float2 ms = mul2(sub2(mul2(mn, factor), sub2(p, PON)), den);
    const float2 Fmn = fma2(w, sub2(ms, mn), fma2(mn, u, p));
    // tangential momentum: mt u + w (mt fd - mt)
    const float2 Fmt = fma2(w, sub2(mul2(mt, fd), mt), mul2(mt, u));
    // energy: (E + p) u + w ((E factor - p u + PON Sc) den - E)
    const float2 Es = mul2(fma2(PON, Sc, sub2(mul2(E, factor), mul2(p, u))), den);
    const float2 FE = fma2(w, sub2(Es, E), mul2(add2(E, p), u));
    Fx.m[0] = Fmn.x;
    Fx.m[1] = Fmt.x;
    Fy.m[1] = Fmn.y;
    Fy.m[0] = Fmt.y;
    Fx.E = FE.x;
    Fy.E = FE.y;
}

// Ghost state beyond a boundary patch of a 2D mesh (the ghostState of fv_device.cuh on a lean
// state): fixed-value concentrations / velocity / pressure, slip mirrors the normal velocity.
template <int NS, int EOS>
__device__ __forceinline__ void leanGhost(const LeanMix<NS>& L, const BCParams& bc, int patch, const LeanW<NS>& own,
                                          LeanW<NS>& g) {
    float rho[NS + 1];
    rho[0] = 0.f;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        const float ck = bc.conc[patch][k - 1] == FV_BC_FIXED_CELL ? float(bc.conc_value[patch][k - 1])
                                                                  : own.rho[k] * L.invM[k - 1];
        rho[k] = ck * L.M[k - 1];
        rho[0] += rho[k];
    }
    float v[2] = {own.v[0], own.v[1]};
    const int vt = bc.vel[patch];
    if (vt == FV_BC_FIXED_CELL) {
        v[0] = float(bc.vel_value[patch][0]);
        v[1] = float(bc.vel_value[patch][1]);
    } else if (vt == FV_BC_SLIP) {
        const int axis = (patch == FV_PATCH_TAIL || patch == FV_PATCH_POINT) ? 0 : 1;
        v[axis] = -v[axis];
    }
    const float p = bc.p[patch] == FV_BC_FIXED_CELL ? float(bc.p_value[patch]) : own.p;
#pragma unroll
    for (int k = 0; k <= NS; ++k) g.rho[k] = rho[k];
    g.v[0] = v[0];
    g.v[1] = v[1];
    g.m[0] = v[0] * rho[0];
    g.m[1] = v[1] * rho[0];
    g.p = p;
    // internal energy from the pressure (UvFromp), then E and the sound speed
    float c[NS + 1];
    c[0] = 0.f;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = rho[k] * L.invM[k - 1];
        c[0] += c[k];
    }
    float X[NS], Cvm = 0.f;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        X[k] = c[k + 1] / c[0];
        Cvm += X[k] * L.Cv[k];
    }
    const float g1 = L.R / Cvm;
    float Uv;
    if (EOS == FV_EOS_IDEAL) {
        Uv = p / g1;
    } else {
        float am = 0.f, bm = 0.f;
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                am += X[k] * X[l] * L.a[k][l];
                bm += X[k] * X[l] * L.b[k][l];
            }
        const float acc = am * c[0] * c[0];
        Uv = (p + acc) * (1.f - c[0] * bm) / g1 - acc;
    }
    g.E = Uv + 0.5f * rho[0] * (v[0] * v[0] + v[1] * v[1]);
    float pp, cs2;
    leanEos<NS, EOS>(L, rho, 1.f / rho[0], Uv, pp, cs2);
    g.cs = sqrtf(cs2);
}

template <int NS> __device__ __forceinline__ void shflUp(const LeanW<NS>& a, LeanW<NS>& b) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) b.rho[k] = __shfl_up_sync(0xffffffffu, a.rho[k], 1);
    b.m[0] = __shfl_up_sync(0xffffffffu, a.m[0], 1);
    b.m[1] = __shfl_up_sync(0xffffffffu, a.m[1], 1);
    b.E = __shfl_up_sync(0xffffffffu, a.E, 1);
    b.p = __shfl_up_sync(0xffffffffu, a.p, 1);
    b.cs = __shfl_up_sync(0xffffffffu, a.cs, 1);
    b.v[0] = __shfl_up_sync(0xffffffffu, a.v[0], 1);
    b.v[1] = a.v[1];  // not read by an x face
}

template <int NS> __device__ __forceinline__ void shflDown(const LeanF<NS>& a, LeanF<NS>& b) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) b.rho[k] = __shfl_down_sync(0xffffffffu, a.rho[k], 1);
    b.m[0] = __shfl_down_sync(0xffffffffu, a.m[0], 1);
    b.m[1] = __shfl_down_sync(0xffffffffu, a.m[1], 1);
    b.E = __shfl_down_sync(0xffffffffu, a.E, 1);
}

// A benign state for lanes outside the mesh (their fluxes are never used).
template <int NS> __device__ __forceinline__ void restState(double* d) {
#pragma unroll
    for (int k = 0; k < NS; ++k) d[k] = 1.0;
    d[NS] = double(NS);
    d[NS + 1] = 0.0;
    d[NS + 2] = 0.0;
    d[NS + 3] = 1.0;
}

// Asynchronous 8-byte copies global -> shared (one per lane and field), in groups per row.
__device__ __forceinline__ void cpAsync8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cpAsyncWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Rows a warp keeps in its shared-memory ring (RING mode): the row being updated, the next one
// and two in flight.
constexpr int kWarpRingRows = 4;
template <int NS> __host__ __device__ constexpr int warpRingDoubles() { return kWarpRingRows * (NS + 4) * 32; }

// One strip: columns xs .. xs + 29 (lanes 1..30), rows z0 .. z0 + rows - 1.  Returns the lane's
// CFL signal maximum (-1 when it updated nothing).  Field offsets are 32-bit (the host enables
// this march only when (N + 5) * cells < 2^31).  RING: rows arrive three ahead in the warp's
// shared-memory ring `ring` by asynchronous copies (each lane copies and reads only its own
// column, so no warp synchronisation is needed); otherwise they are loaded one row ahead into
// registers.
template <int NS, int EOS, bool RING>
__device__ __forceinline__ float warpStrip(const StepParams& P, const double* __restrict__ U, double* __restrict__ Un,
                                           DevClock* __restrict__ ck, const LeanMix<NS>& L, double dt,
                                           const double* g, int xs, int z0, int rows, double* ring) {
    constexpr int NF = NS + 4;  // conserved fields carried: rho_1..rho_N, rho, m_x, m_y, E
    const int lane = threadIdx.x & 31;
    const int nx = P.n[0], ny = P.n[1];
    const bool perX = P.periodic[0] != 0, perY = P.periodic[1] != 0;
    const int X = xs - 1 + lane;
    int cx = X;
    bool has = X >= 0 && X < nx;
    if (!has && perX && (X == -1 || X == nx)) {
        cx = X < 0 ? nx - 1 : 0;
        has = true;
    }
    const bool interior = lane >= 1 && lane <= 30 && X < nx;
    const bool xLoPatch = X == 0 && !perX;        // tail patch below this cell
    const bool xHiPatch = X == nx - 1 && !perX;   // point patch above this cell
    const int z1 = min(z0 + rows, ny);
    const int st = (int)P.stride;
    int off[NF];  // field offsets in the state (E follows m_z)
#pragma unroll
    for (int f = 0; f < NF; ++f) off[f] = (f < NF - 1 ? f : NS + 4) * st;
    const float hxf = has ? float(P.geo.h[0][cx]) : 1.f;
    const float Lz = float(P.ext[2]);
    const float gx = float(g[0]), gy = float(g[1]);
    const float dtf = float(dt);
    const float axdt = dtf / hxf;  // dt * (x face area) / volume
    const bool grav = P.gravity != 0;
    const int flux = P.flux;

    auto wrapY = [&](int z, bool& ok) -> int {
        ok = true;
        if (z < 0) { if (perY) return z + ny; ok = false; return 0; }
        if (z >= ny) { if (perY) return z - ny; ok = false; return 0; }
        return z;
    };
    auto load = [&](int z, double* d) {
        bool ok;
        const int zz = wrapY(z, ok);
        if (has && ok) {
            const double* q = U + ((long long)zz * nx + cx);
#pragma unroll
            for (int f = 0; f < NF; ++f) d[f] = __ldg(q + off[f]);
        } else {
            restState<NS>(d);
        }
    };

    // ring slot of row r: rows z0 - 1, z0, z0 + 1, ... cycle through the slots
    auto slotOf = [&](int r) -> double* { return ring + ((r - z0 + 1) & (kWarpRingRows - 1)) * (NF * 32) + lane; };
    auto issue = [&](int r) {  // RING: copy row r into its slot (an empty group when outside)
        bool ok;
        const int zz = wrapY(r, ok);
        if (has && ok && r < z0 + rows + 1) {
            const double* q = U + ((long long)zz * nx + cx);
            double* dst = slotOf(r);
#pragma unroll
            for (int f = 0; f < NF; ++f) cpAsync8(dst + f * 32, q + off[f]);
        }
        cpAsyncCommit();
    };
    auto fetch = [&](int r, double* d) {  // RING: row r from its slot
        bool ok;
        wrapY(r, ok);
        if (has && ok) {
            const double* src = slotOf(r);
#pragma unroll
            for (int f = 0; f < NF; ++f) d[f] = src[f * 32];
        } else {
            restState<NS>(d);
        }
    };

    bool bad = false;
    float localMax = -1.f;
    // Row z with the state of rows z (Wc, dCur) and z + 1 (Wn, dNext to be loaded) and the flux
    // through the face below row z (Gprev); leaves the flux above row z in Gnext.
    auto row = [&](int z, const LeanW<NS>& Wc, LeanW<NS>& Wn, const double* dCur, double* dNext,
                   const LeanF<NS>& Gprev, LeanF<NS>& Gnext) {
        if constexpr (RING) {
            issue(z + 3);         // into the slot of row z - 1, read for the last time a row ago
            cpAsyncWait<2>();     // rows up to z + 1 have landed
            fetch(z + 1, dNext);
        } else {
            load(z + 1, dNext);
        }
        // the low x face of this lane (owner: W of lane - 1, or the tail-patch ghost) and the
        // face above this row (neighbour: W of the next row, or the left-patch ghost)
        LeanW<NS> Ox;
        shflUp<NS>(Wc, Ox);
        if (xLoPatch) leanGhost<NS, EOS>(L, P.bc, FV_PATCH_TAIL, Wc, Ox);
        leanClose<NS, EOS>(L, dNext, Wn);
        bool okN;
        wrapY(z + 1, okN);
        LeanW<NS> By = Wn;
        if (!okN) leanGhost<NS, EOS>(L, P.bc, FV_PATCH_LEFT, Wc, By);
        LeanF<NS> Fx;
        bool okx, oky;
        if (flux == FV_FLUX_HLLC) {
            hllcPair<NS>(Ox, Wc, Wc, By, Fx, Gnext, okx, oky);
        } else {
            okx = leanRiemann<NS, 0>(flux, Ox, Wc, Fx);
            oky = leanRiemann<NS, 1>(flux, Wc, By, Gnext);
        }
        bad |= (!okx && has && lane >= 1) || (!oky && has);
        // high x face: the low face of lane + 1, or the point patch
        LeanF<NS> Fxp;
        shflDown<NS>(Fx, Fxp);
        if (xHiPatch) {
            LeanW<NS> Gs;
            leanGhost<NS, EOS>(L, P.bc, FV_PATCH_POINT, Wc, Gs);
            bad |= !leanRiemann<NS, 0>(flux, Wc, Gs, Fxp);
        }
        if (interior) {
            const float hy = float(P.geo.h[1][z]);
            const float aydt = dtf / hy;
            const float minLS = 1.f / fminf(fminf(hxf, hy), Lz);
            double* q = Un + ((long long)z * nx + cx);
            double dOld[NF];
            if constexpr (RING) {
                fetch(z, dOld);
            } else {
#pragma unroll
                for (int f = 0; f < NF; ++f) dOld[f] = dCur[f];
            }
            // per field in state order (rho_1..rho_N, rho, m_x, m_y, E): FP32 increments
            // dt * div F (+ gravity), two fields per paired instruction
            float fxp[NF], fxm[NF], gn[NF], gp[NF], w0[NF], inc[NF];
            auto flat = [&](const LeanF<NS>& F, float* o) {
#pragma unroll
                for (int k = 1; k <= NS; ++k) o[k - 1] = F.rho[k];
                o[NS] = F.rho[0];
                o[NS + 1] = F.m[0];
                o[NS + 2] = F.m[1];
                o[NS + 3] = F.E;
            };
            flat(Fxp, fxp);
            flat(Fx, fxm);
            flat(Gnext, gn);
            flat(Gprev, gp);
#pragma unroll
            for (int k = 1; k <= NS; ++k) w0[k - 1] = Wc.rho[k];
            w0[NS] = Wc.rho[0];
            w0[NS + 1] = Wc.m[0];
            w0[NS + 2] = Wc.m[1];
            w0[NS + 3] = Wc.E;
            const float2 ax2 = make_float2(axdt, axdt), ay2 = make_float2(aydt, aydt);
#pragma unroll
            for (int f = 0; f + 1 < NF; f += 2) {
                const float2 dx = sub2(make_float2(fxp[f], fxp[f + 1]), make_float2(fxm[f], fxm[f + 1]));
                const float2 dy = sub2(make_float2(gn[f], gn[f + 1]), make_float2(gp[f], gp[f + 1]));
                const float2 i2 = fma2(dx, ax2, mul2(dy, ay2));
                inc[f] = i2.x;
                inc[f + 1] = i2.y;
            }
            if (NF & 1) inc[NF - 1] = (fxp[NF - 1] - fxm[NF - 1]) * axdt + (gn[NF - 1] - gp[NF - 1]) * aydt;
            if (grav) {
                const float r0 = Wc.rho[0] * dtf;
                inc[NS + 1] -= gx * r0;
                inc[NS + 2] -= gy * r0;
                inc[NS + 3] -= r0 * (Wc.v[0] * gx + Wc.v[1] * gy);
            }
            // FP64 accumulation; the FP32 state after the step (for the CFL signal) takes the
            // same increments
            float wn[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                q[off[f]] = dOld[f] - double(inc[f]);
                wn[f] = w0[f] - inc[f];
            }
            float rhoN[NS + 1], mN[2];
#pragma unroll
            for (int k = 1; k <= NS; ++k) rhoN[k] = wn[k - 1];
            rhoN[0] = wn[NS];
            mN[0] = wn[NS + 1];
            mN[1] = wn[NS + 2];
            const float EN = wn[NS + 3];
            localMax = fmaxf(localMax, leanSignal<NS, EOS>(L, rhoN, mN, EN, minLS));
        }
    };

    double dA[NF], dB[NF];
    LeanW<NS> WA, WB;
    LeanF<NS> GA, GB;
    // prologue: the cell below the strip's first row and the flux through the face between
    {
        double dBelow[NF];
        if constexpr (RING) {
            for (int r = z0 - 1; r < z0 + 3; ++r) issue(r);
            cpAsyncWait<2>();
            fetch(z0 - 1, dBelow);
            fetch(z0, dA);
        } else {
            load(z0 - 1, dBelow);
            load(z0, dA);
        }
        LeanW<NS> Wb;
        leanClose<NS, EOS>(L, dBelow, Wb);
        leanClose<NS, EOS>(L, dA, WA);
        bool okB;
        wrapY(z0 - 1, okB);
        if (okB) {
            bad |= !leanRiemann<NS, 1>(flux, Wb, WA, GA);
        } else {
            LeanW<NS> Gs;
            leanGhost<NS, EOS>(L, P.bc, FV_PATCH_RIGHT, WA, Gs);
            bad |= !leanRiemann<NS, 1>(flux, Gs, WA, GA);
        }
    }
    // two rows per iteration with the roles of the A and B registers swapped (no copies)
    int z = z0;
    for (; z + 1 < z1; z += 2) {
        row(z, WA, WB, dA, dB, GA, GB);
        row(z + 1, WB, WA, dB, dA, GB, GA);
    }
    if (z < z1) row(z, WA, WB, dA, dB, GA, GB);
    if constexpr (RING) cpAsyncWait<0>();  // no copy outlives the strip
    if (bad) raise(ck, FV_ERR_RIEMANN);
    return localMax;
}

// CTA = NW independent warps, each on one strip; grid x: strips / NW, grid y: row tiles.
// The warps of a tile are independent to the end: each writes its own CFL partial maximum to
// partials[w] (no CTA barrier).
template <int NS, int EOS, bool RING>
__device__ __forceinline__ void warpTile(const StepParams& P, const double* __restrict__ U, double* __restrict__ Un,
                                         DevClock* __restrict__ ck, double* __restrict__ partials, int rows,
                                         int tileX, int tileZ) {
    extern __shared__ __align__(16) double warpRing[];
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float m = -1.f;
    if (!ck->done) {
        LeanMix<NS> L;
        leanMix<NS, EOS>(P.mix, L);
        const int strip = tileX * nw + w;
        const int xs = strip * kWarpStripCols;
        if (xs < P.n[0])
            m = warpStrip<NS, EOS, RING>(P, U, Un, ck, L, ck->dt, ck->g, xs, tileZ * rows, rows,
                                         RING ? warpRing + w * warpRingDoubles<NS>() : nullptr);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) partials[w] = double(m);
}

template <int NS, int EOS, int NW, int MINB, bool RING>
__global__ void __launch_bounds__(32 * NW, MINB) k_warp2d(const StepParams P, const double* __restrict__ U,
                                                          double* __restrict__ Un, DevClock* __restrict__ ck,
                                                          double* __restrict__ blockMax, int rows) {
    if (ck->done) return;  // uniform over the grid
    warpTile<NS, EOS, RING>(P, U, Un, ck, blockMax + (blockIdx.x + (long long)gridDim.x * blockIdx.y) * NW, rows,
                            blockIdx.x, blockIdx.y);
    if (P.fuseFinalize) {
        const unsigned n = gridDim.x * gridDim.y;
        finalizeIfLast(P, ck, blockMax, (int)(n * NW), n);
    }
}

// Ensemble version: one CTA per tile of any case (the tile list of all cases in order).
template <int NS, int EOS, int NW, int MINB, bool RING>
__global__ void __launch_bounds__(32 * NW, MINB) k_warp2d_batch(const BatchCase* __restrict__ cases, int nCases,
                                                                long long totalTiles, int rows) {
    static_assert(sizeof(StepParams) % 8 == 0, "StepParams is copied in 8-byte words");
    __shared__ StepParams sP;
    const long long t = blockIdx.x;
    if (t >= totalTiles) return;
    int lo = 0, hi = nCases - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cases[mid].tileBase <= t) lo = mid;
        else hi = mid - 1;
    }
    const BatchCase& C = cases[lo];
    if (C.ck->done) return;  // uniform over the CTA
    const long long local = t - C.tileBase;
    const int tx = (int)(local % C.tiles[0]);
    const int tz = (int)(local / C.tiles[0]);
    const bool odd = ((C.ck->steps - C.stepsBase) & 1) != 0;
    const double* Uin = odd ? C.U1 : C.U0;
    double* Uout = odd ? const_cast<double*>(C.U0) : C.U1;
    // the case's parameters in shared memory: read where needed instead of held in registers
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&C.P);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sP);
        for (int i = threadIdx.x; i < (int)(sizeof(StepParams) / 8); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    warpTile<NS, EOS, RING>(sP, Uin, Uout, C.ck, C.blockMax + local * NW, rows, tx, tz);
    if (sP.fuseFinalize) finalizeIfLast(sP, C.ck, C.blockMax, C.nPartials, (unsigned)C.nTiles);
}

}  // namespace fv
