// fv_warp2d64.cuh -- warp-strip march in FP64: the bit-exact 2D step of the fused march (zero-slope
// limiters, two momentum components) laid out like the FP32-flux warp strip of fv_warp2d.cuh.
//
// Each warp owns a strip of 30 columns (lanes 1..30; lanes 0 and 31 are the halo columns on either
// side) and marches along y over `rows` rows.  Per row a lane
//   * builds the predicted face state W of the next row (closure and Hancock round trip of the
//     reference, FP64 without contraction) from its conserved values, which were loaded one row
//     earlier into registers;
//   * takes W of lane - 1 by shuffle and computes the flux through its low x face, and the flux
//     through the face between its row and the next (kept in registers for the next row);
//   * takes the high-x-face flux from lane + 1 by shuffle and updates its cell: the divergence in
//     the reference's face order [x-, x+, y+, y-] divided by the volume, U_new = U - div * dt, the
//     gravity source of Advection.cpp:424-431, and the CFL signal of the updated cell.
// Every expression is the CTA march's (marchTile in fv_kernels.cuh): the same device functions in
// the same order, so the results are the reference's bit for bit.  Warps never wait for one
// another: no shared memory and no CTA barrier; each warp writes its own CFL partial maximum.
#pragma once

#include "fv_kernels.cuh"

namespace fv {

// Resident threads per SM the register budget of the FP64 warp strip is sized for.
#ifndef FV_WARP64_THREADS_PER_SM
#define FV_WARP64_THREADS_PER_SM 384
#endif
constexpr int kWarp64ThreadsPerSM = FV_WARP64_THREADS_PER_SM;

template <int NS> __device__ __forceinline__ void shflUpW(const FaceState<double, NS>& a, FaceState<double, NS>& b) {
    // the fields an x face reads from its owner (riemann along axis 0)
#pragma unroll
    for (int k = 0; k <= NS; ++k) b.rho[k] = __shfl_up_sync(0xffffffffu, a.rho[k], 1);
    b.m[0] = __shfl_up_sync(0xffffffffu, a.m[0], 1);
    b.m[1] = __shfl_up_sync(0xffffffffu, a.m[1], 1);
    b.m[2] = 0.0;
    b.v[0] = __shfl_up_sync(0xffffffffu, a.v[0], 1);
    b.v[1] = 0.0;
    b.v[2] = 0.0;
    b.E = __shfl_up_sync(0xffffffffu, a.E, 1);
    b.p = __shfl_up_sync(0xffffffffu, a.p, 1);
    b.cs = __shfl_up_sync(0xffffffffu, a.cs, 1);
}

template <int NS> __device__ __forceinline__ void shflDownF(const FaceFlux<double, NS>& a, FaceFlux<double, NS>& b) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) b.rho[k] = __shfl_down_sync(0xffffffffu, a.rho[k], 1);
    b.m[0] = __shfl_down_sync(0xffffffffu, a.m[0], 1);
    b.m[1] = __shfl_down_sync(0xffffffffu, a.m[1], 1);
    b.m[2] = 0.0;
    b.E = __shfl_down_sync(0xffffffffu, a.E, 1);
}

// One strip of the FP64 march: columns xs .. xs + 29 (lanes 1..30), rows z0 .. z0 + rows - 1.
// Returns the lane's CFL signal maximum (-1 when it updated nothing).
//
// Primitive cache (pcIn / pcOut, one array per state buffer, N + 7 fields of n_cells doubles:
// c_1..c_N, v_x, v_y, p and the mixture coefficients g1, a, b, M): the epilogue recovers c, v, p and
// the coefficients of the updated cell for its CFL signal, which are exactly what the next step's
// closure recovers again from the same FP64 state (same operations on the same values).  A fused
// step writes them to pcOut and its finalize marks the clock's cache valid; the next step then
// reads them (pcIn) instead of recomputing them.  Any other writer of the state clears the mark.
template <int NS, int EOS>
__device__ __forceinline__ double warpStrip64(const StepParams& P, const double* __restrict__ U,
                                              double* __restrict__ Un, const double* __restrict__ prim,
                                              DevClock* __restrict__ ck, double dt, const double* g, int xs, int z0,
                                              int rows, const double* __restrict__ pcIn, double* __restrict__ pcOut) {
    constexpr int NF = NS + 4;  // rho_1..rho_N, rho, m_x, m_y, E
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
    const bool xLoPatch = X == 0 && !perX;
    const bool xHiPatch = X == nx - 1 && !perX;
    const int z1 = min(z0 + rows, ny);
    const long long st = P.stride;
    const double hx = has ? P.geo.h[0][cx] : 1.0;
    const double Lz = P.ext[2];
    const double gx_ = g[0], gy_ = g[1], gz_ = g[2];

    auto wrapY = [&](int z, bool& ok) -> int {
        ok = true;
        if (z < 0) { if (perY) return z + ny; ok = false; return 0; }
        if (z >= ny) { if (perY) return z - ny; ok = false; return 0; }
        return z;
    };
    // conserved values of row z in slot order (densities, mixture density, m_x, m_y, E)
    auto load = [&](int z, double* d) {
        bool ok;
        const int zz = wrapY(z, ok);
        if (has && ok) {
            const double* q = U + ((long long)zz * nx + cx);
#pragma unroll
            for (int f = 0; f < NF; ++f) d[f] = __ldg(q + (long long)(f < NF - 1 ? f : NS + 4) * st);
        } else {
#pragma unroll
            for (int k = 0; k < NS; ++k) d[k] = 1.0;
            d[NS] = double(NS);
            d[NS + 1] = 0.0;
            d[NS + 2] = 0.0;
            d[NS + 3] = 1.0;
        }
    };
    // predicted face state of the cell in row z from its loaded conserved values; vp: its
    // velocity at the step's start (the gravity source)
    auto state = [&](int z, const double* d, FaceState<double, NS>& W, double* vp) {
        bool ok;
        const int zz = wrapY(z, ok);
        const Src sc{d, 1, NS + 3};
        // a lane outside the mesh works on the benign state of load() (its fluxes are not used)
        // and reads the restart set or the stored concentrations at cell 0
        const long long i = (has && ok) ? (long long)zz * nx + cx : 0;
        double c[NS + 1], v[3], p, r0, rr[NS + 1], mm[3], EE;
        typename Mixture<double, NS, EOS>::Coef kc;
        bool haveK;
        if (pcIn && has && ok) {
            const double* q = pcIn + i;
            c[0] = 0;
#pragma unroll
            for (int k = 1; k <= NS; ++k) {
                c[k] = __ldg(q + (k - 1) * st);
                c[0] += c[k];
            }
            v[0] = __ldg(q + NS * st);
            v[1] = __ldg(q + (NS + 1) * st);
            v[2] = 0.0;
            p = __ldg(q + (NS + 2) * st);
            kc.g1 = __ldg(q + (NS + 3) * st);
            kc.am = __ldg(q + (NS + 4) * st);
            kc.bm = __ldg(q + (NS + 5) * st);
            kc.Mm = __ldg(q + (NS + 6) * st);
            haveK = true;
        } else {
            cellPrimitive<double, NS, EOS, 2>(P, sc, (has && ok) ? prim : nullptr, i, c, v, p, r0, rr, mm, EE, &kc,
                                              &haveK);
        }
        cellFaceState<double, NS, EOS>(P.mix, c, v, p, W, 2, P.hancock != 0, haveK ? &kc : nullptr);
        vp[0] = v[0];
        vp[1] = v[1];
        vp[2] = v[2];
    };

    bool bad = false;
    double localMax = -1;
    FaceState<double, NS> Wc, Wn;
    FaceFlux<double, NS> Gprev, Gnext;
    double GprevSign = -1;
    double vCur[3] = {0, 0, 0}, vNext[3] = {0, 0, 0};
    double dCur[NF], dNext[NF];

    // prologue: W of row z0 and the flux through the face below it
    load(z0, dCur);
    if (z0 < z1) {
        state(z0, dCur, Wc, vCur);
        bool okB;
        wrapY(z0 - 1, okB);
        if (okB) {
            double dB[NF], vb[3];
            load(z0 - 1, dB);
            FaceState<double, NS> Wb;
            state(z0 - 1, dB, Wb, vb);
            bad |= !riemann<double, NS>(P.flux, 1, 1, Wb, Wc, Gprev) && has;
            GprevSign = -1;
        } else {
            // y-min patch (right in 2D); outward normal -e_y
            FaceState<double, NS> Gs;
            ghostState<double, NS, EOS>(P.mix, P.bc, FV_PATCH_RIGHT, 1, -1, Wc, Gs);
            bad |= !riemann<double, NS>(P.flux, 1, -1, Wc, Gs, Gprev) && has;
            GprevSign = 1;
        }
    }
    for (int z = z0; z < z1; ++z) {
        load(z + 1, dNext);
        bool okN;
        wrapY(z + 1, okN);
        // the low x face of this lane: owner W of lane - 1, or (tail patch) the ghost of this cell
        FaceState<double, NS> Wl;
        shflUpW<NS>(Wc, Wl);
        FaceFlux<double, NS> Fx;
        if (xLoPatch) {
            FaceState<double, NS> Gs;
            ghostState<double, NS, EOS>(P.mix, P.bc, FV_PATCH_TAIL, 0, -1, Wc, Gs);
            bad |= !riemann<double, NS>(P.flux, 0, -1, Wc, Gs, Fx) && has;
        } else {
            bad |= !riemann<double, NS>(P.flux, 0, 1, Wl, Wc, Fx) && has && lane >= 1;
        }
        // the face above this row: neighbour W of the next row, or the y-max (left) patch ghost
        if (okN) {
            state(z + 1, dNext, Wn, vNext);
            bad |= !riemann<double, NS>(P.flux, 1, 1, Wc, Wn, Gnext) && has;
        } else {
            FaceState<double, NS> Gs;
            ghostState<double, NS, EOS>(P.mix, P.bc, FV_PATCH_LEFT, 1, 1, Wc, Gs);
            bad |= !riemann<double, NS>(P.flux, 1, 1, Wc, Gs, Gnext) && has;
        }
        // the high x face: the low face of lane + 1, or the point patch
        FaceFlux<double, NS> Fxp;
        shflDownF<NS>(Fx, Fxp);
        if (xHiPatch) {
            FaceState<double, NS> Gs;
            ghostState<double, NS, EOS>(P.mix, P.bc, FV_PATCH_POINT, 0, 1, Wc, Gs);
            bad |= !riemann<double, NS>(P.flux, 0, 1, Wc, Gs, Fxp);
        }
        if (interior) {
            const double sxm = xLoPatch ? 1.0 : -1.0;
            const double hm = P.geo.h[1][z];
            // face areas and volume (mesh.cpp): x faces Lz h_y, y faces h_x Lz, V = h_x h_y Lz
            const double Sx = Lz * hm, Sm = hx * Lz;
            const double V = hx * hm * Lz;
            const double minLS = 1.0 / smin(smin(hx, hm), Lz);
            auto div = [&](auto get) -> double {
                double s = get(Fx) * sxm * Sx;
                s += get(Fxp) * Sx;
                s += get(Gnext) * Sm;
                s += get(Gprev) * GprevSign * Sm;
                return s / V;
            };
            const long long ic = (long long)z * nx + cx;
            const double rho0Old = dCur[NS];
            double Enew = dCur[NS + 3] - div([](const FaceFlux<double, NS>& f) { return f.E; }) * dt;
            double mNew[3] = {0, 0, 0};
            mNew[0] = dCur[NS + 1] - div([](const FaceFlux<double, NS>& f) { return f.m[0]; }) * dt;
            mNew[1] = dCur[NS + 2] - div([](const FaceFlux<double, NS>& f) { return f.m[1]; }) * dt;
            if (P.gravity) {
                // Advection.cpp:424-431 with the old density and velocity
                double vg = 0;
                vg += vCur[0] * gx_;
                vg += vCur[1] * gy_;
                vg += vCur[2] * gz_;
                Enew += (rho0Old * vg) * dt;
                mNew[0] += (gx_ * rho0Old) * dt;
                mNew[1] += (gy_ * rho0Old) * dt;
            }
            double rNew[NS + 1];
            rNew[0] = rho0Old - div([](const FaceFlux<double, NS>& f) { return f.rho[0]; }) * dt;
#pragma unroll
            for (int k = 1; k <= NS; ++k)
                rNew[k] = dCur[k - 1] - div([k](const FaceFlux<double, NS>& f) { return f.rho[k]; }) * dt;
#pragma unroll
            for (int k = 1; k <= NS; ++k) Un[(k - 1) * st + ic] = rNew[k];
            Un[NS * st + ic] = rNew[0];
            Un[(NS + 1) * st + ic] = mNew[0];
            Un[(NS + 2) * st + ic] = mNew[1];
            Un[(NS + 4) * st + ic] = Enew;
            double cN[NS + 1], vN[3], pN;
            typename Mixture<double, NS, EOS>::Coef kN;
            localMax = smax(localMax,
                            cellSignalPrim<double, NS, EOS>(P, rNew, rNew[0], mNew, Enew, minLS, cN, vN, pN, kN));
            if (pcOut) {
                double* q = pcOut + ic;
#pragma unroll
                for (int k = 1; k <= NS; ++k) q[(k - 1) * st] = cN[k];
                q[NS * st] = vN[0];
                q[(NS + 1) * st] = vN[1];
                q[(NS + 2) * st] = pN;
                q[(NS + 3) * st] = kN.g1;
                q[(NS + 4) * st] = kN.am;
                q[(NS + 5) * st] = kN.bm;
                q[(NS + 6) * st] = kN.Mm;
            }
        }
        // roll the marching window
        Gprev = Gnext;
        GprevSign = -1;
        if (okN) {
            Wc = Wn;
            vCur[0] = vNext[0];
            vCur[1] = vNext[1];
            vCur[2] = vNext[2];
#pragma unroll
            for (int f = 0; f < NF; ++f) dCur[f] = dNext[f];
        }
    }
    if (bad) raise(ck, FV_ERR_RIEMANN);
    return localMax;
}

// CTA = NW independent warps, each on one strip; grid x: strips / NW, grid y: row tiles.
template <int NS, int EOS, int NW, int MINB>
__global__ void __launch_bounds__(32 * NW, MINB) k_warp2d64(const StepParams P, const double* __restrict__ U,
                                                            double* __restrict__ Un,
                                                            const double* __restrict__ prim0,
                                                            DevClock* __restrict__ ck, double* __restrict__ blockMax,
                                                            int rows, const double* __restrict__ pcIn,
                                                            double* __restrict__ pcOut) {
    if (ck->done) return;  // uniform over the grid
    const int w = threadIdx.x >> 5;
    const double* prim = ck->first ? prim0 : nullptr;
    // the cache is read when the clock marks it valid (never before the first step, which reads
    // the restart set) and written only by a step that finalizes itself (and so marks it)
    const double* pcUse = (pcIn && ck->pcValid && !ck->first) ? pcIn : nullptr;
    double* pcWrite = P.fuseFinalize ? pcOut : nullptr;
    const int strip = blockIdx.x * NW + w;
    const int xs = strip * kWarpStripCols;
    double m = -1;
    if (xs < P.n[0])
        m = warpStrip64<NS, EOS>(P, U, Un, prim, ck, ck->dt, ck->g, xs, blockIdx.y * rows, rows, pcUse, pcWrite);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = smax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const long long part = (blockIdx.x + (long long)gridDim.x * blockIdx.y) * NW + w;
    if ((threadIdx.x & 31) == 0) blockMax[part] = m;
    if (P.fuseFinalize) {
        const unsigned n = gridDim.x * gridDim.y;
        finalizeIfLast(P, ck, blockMax, (int)(n * NW), n, pcWrite ? 1 : 0);
    }
}

}  // namespace fv
