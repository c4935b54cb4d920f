// fv_generic.cuh -- full MUSCL-Hancock step of the reference with face states in scratch.
//
//   k_prim    cell primitives c_k, v, p (Advection.cpp:455-479, or the restart set at step 1)
//   k_faces   per cell: Gauss gradients (gradient.hpp:19-58 + linearInterpolate.hpp:43-80),
//             r-ratio TVD limiter (TVDLimiter.cpp:12-272, including its [direction][component]
//             neighbour-gradient layout for the velocity tensor), reconstruction at every face
//             of the cell (Advection.cpp:114-235), closure (:237-387), Hancock half step over the
//             cell's own faces (HancockStage.cpp:17-240); SecondOrderRK stages stop after the
//             closure (Advection2dOrder.cpp, no predictor)
//   k_fluxes  per face: ghost neighbour on boundary patches (HancockStage.cpp:324-446) and the
//             Riemann flux
//   k_update  per cell: divergence in the cell's face order, conservative update, gravity,
//             new primitives and the CTA maximum of the CFL signal
//
// Face numbering: faces normal to axis a form a block of (n_a + 1) * prod(n_b, b != a) faces,
// index i_a + (n_a + 1) * (transverse index).  A periodic axis uses face n_a as the wrap face
// (owner n_a - 1, neighbour 0) and leaves face 0 unused, like the reference's face list has
// one face per cell pair.
#pragma once

#include "fv_kernels.cuh"

namespace fv {

struct GenericLayout {
    long long faceBase[3];   // first face of each axis block
    long long nfaces;        // total (including unused periodic slots)
};

// number of face-state fields per side: c[0..NS], rho[0..NS], v[3], m[3], E, Uv, p, cs
template <int NS> __host__ __device__ constexpr int faceFields() { return 2 * (NS + 1) + 10; }

template <typename T, int NS>
__device__ __forceinline__ void storeFace(T* __restrict__ FS, long long nf, int side, long long f, const FaceState<T, NS>& s) {
    constexpr int NF = faceFields<NS>();
    T* b = FS + (long long)side * NF * nf + f;
    int q = 0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) b[(q++) * nf] = s.c[k];
#pragma unroll
    for (int k = 0; k <= NS; ++k) b[(q++) * nf] = s.rho[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) b[(q++) * nf] = s.v[d];
#pragma unroll
    for (int d = 0; d < 3; ++d) b[(q++) * nf] = s.m[d];
    b[(q++) * nf] = s.E;
    b[(q++) * nf] = s.Uv;
    b[(q++) * nf] = s.p;
    b[(q++) * nf] = s.cs;
}

template <typename T, int NS>
__device__ __forceinline__ void loadFace(const T* __restrict__ FS, long long nf, int side, long long f, FaceState<T, NS>& s) {
    constexpr int NF = faceFields<NS>();
    const T* b = FS + (long long)side * NF * nf + f;
    int q = 0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) s.c[k] = b[(q++) * nf];
#pragma unroll
    for (int k = 0; k <= NS; ++k) s.rho[k] = b[(q++) * nf];
#pragma unroll
    for (int d = 0; d < 3; ++d) s.v[d] = b[(q++) * nf];
#pragma unroll
    for (int d = 0; d < 3; ++d) s.m[d] = b[(q++) * nf];
    s.E = b[(q++) * nf];
    s.Uv = b[(q++) * nf];
    s.p = b[(q++) * nf];
    s.cs = b[(q++) * nf];
}

// Geometry of one face of cell (i, j, k): axis a, high (+) or low (-) side.
struct FaceGeo {
    long long f;       // face index
    int own;           // 1 if the cell is the face's owner
    int boundary;      // 1 on a non-periodic patch
    int patch;         // patch of a boundary face
    int sign;          // sign of the face normal N (outward for the owner)
    double rc[3];      // face centre
    double S;          // area
};

__device__ __forceinline__ double extent(const StepParams& P, int a, int idx) {
    return a < P.dims ? P.geo.h[a][idx] : P.ext[a];
}

// Face of cell (ijk) normal to axis a on side hi (0 = low, 1 = high), following mesh.cpp.
__device__ __forceinline__ FaceGeo faceOf(const StepParams& P, const GenericLayout& L, const int* ijk, int a, int hi) {
    FaceGeo g;
    const int n = P.n[a];
    const bool per = P.periodic[a];
    int fi = ijk[a] + hi;                       // face position along the axis, 0..n
    if (per && fi == 0) fi = n;                 // wrap face
    g.boundary = !per && (fi == 0 || fi == n);
    if (g.boundary) {
        g.own = 1;
        g.sign = fi == 0 ? -1 : 1;
        g.patch = a == 0 ? (fi == 0 ? FV_PATCH_TAIL : FV_PATCH_POINT)
                         : a == 1 ? (fi == 0 ? FV_PATCH_RIGHT : FV_PATCH_LEFT)
                                  : (fi == 0 ? FV_PATCH_BOTTOM : FV_PATCH_TOP);
    } else {
        g.own = hi;                             // the low cell owns the face
        g.sign = 1;
        g.patch = -1;
    }
    // transverse index
    long long tr;
    if (a == 0) tr = (long long)ijk[1] + (long long)P.n[1] * ijk[2];
    else if (a == 1) tr = (long long)ijk[0] + (long long)P.n[0] * ijk[2];
    else tr = (long long)ijk[0] + (long long)P.n[0] * ijk[1];
    g.f = L.faceBase[a] + fi + (long long)(n + 1) * tr;
    // centre: own-axis coordinate of the face, transverse coordinates by corner pattern
    const bool bnd_pattern = (a == 1) && (fi == 0 || fi == n);  // y patches (and the periodic y wrap face)
    g.rc[a] = P.geo.fpos[a][fi];
    if (a == 0) {
        g.rc[1] = P.geo.aabb[1][ijk[1]];
        g.rc[2] = P.geo.abab[2][ijk[2]];
    } else if (a == 1) {
        g.rc[0] = bnd_pattern ? P.geo.aabb[0][ijk[0]] : P.geo.abab[0][ijk[0]];
        g.rc[2] = bnd_pattern ? P.geo.abab[2][ijk[2]] : P.geo.aabb[2][ijk[2]];
    } else {
        g.rc[0] = P.geo.abab[0][ijk[0]];
        g.rc[1] = P.geo.aabb[1][ijk[1]];
    }
    // area |rX0 - r00| * |r0Y - r00| (same value for inner and patch faces)
    const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
    g.S = a == 0 ? ez * ey : (a == 1 ? ex * ez : ex * ey);
    return g;
}

// Neighbour cell across a face (periodic wrap included); returns false on a patch.
__device__ __forceinline__ bool neighbourOf(const StepParams& P, const int* ijk, int a, int hi, int* nb, double& shift) {
    nb[0] = ijk[0]; nb[1] = ijk[1]; nb[2] = ijk[2];
    shift = 0;
    const int n = P.n[a];
    int q = ijk[a] + (hi ? 1 : -1);
    if (q < 0 || q >= n) {
        if (!P.periodic[a]) return false;
        shift = q < 0 ? -P.ext[a] : P.ext[a];
        q = q < 0 ? q + n : q - n;
    }
    nb[a] = q;
    return true;
}

// ---------------------------------------------------------------------------- k_prim
template <typename T, int NS, int EOS, int D>
__global__ void k_prim(const StepParams P, const double* __restrict__ U, const double* __restrict__ prim0,
                       DevClock* __restrict__ ck, T* __restrict__ Pc) {
    if (ck->done) return;
    // the restart set at the first step, the primitives of a diffusion stage after one
    const double* prim = ck->first ? prim0 : (ck->stagePrim ? P.stagePrim : nullptr);
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    T c[NS + 1], v[3], p, r0, rr[NS + 1], mm[3], EE;
    cellPrimitive<T, NS, EOS, D>(P, U, prim, i, c, v, p, r0, rr, mm, EE);
    const long long n = P.ncell;
#pragma unroll
    for (int k = 1; k <= NS; ++k) Pc[(k - 1) * n + i] = c[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) Pc[(NS + d) * n + i] = v[d];
    Pc[(NS + 3) * n + i] = p;
}

// scalar primitive q of cell index i: q < NS: c_{q+1}; NS..NS+2: v; NS+3: p
template <typename T, int NS>
__device__ __forceinline__ T primAt(const T* __restrict__ Pc, long long n, int q, long long i) { return Pc[q * n + i]; }

// surface boundary value of a scalar primitive (boundaryConditionValueSurface, :34-66)
template <typename T, int NS>
__device__ __forceinline__ T surfaceScalar(const StepParams& P, int patch, int q, T in) {
    int type;
    double val;
    if (q < NS) { type = P.bc.conc[patch][q]; val = P.bc.conc_value[patch][q]; }
    else { type = P.bc.p[patch]; val = P.bc.p_value[patch]; }
    if (type == FV_BC_FIXED_CELL) return (in + T(val)) * T(0.5);
    if (type == FV_BC_FIXED_SURFACE) return T(val);
    return in;
}
template <typename T, int NS>
__device__ __forceinline__ T cellGhostScalar(const StepParams& P, int patch, int q, T in, bool& bad) {
    int type;
    double val;
    if (q < NS) { type = P.bc.conc[patch][q]; val = P.bc.conc_value[patch][q]; }
    else { type = P.bc.p[patch]; val = P.bc.p_value[patch]; }
    if (type == FV_BC_FIXED_SURFACE) bad = true;
    return type == FV_BC_FIXED_CELL ? T(val) : in;
}
// surface value of the velocity (slip: v - (v & n) n; fixedValueCell: (v + val) * 0.5)
template <typename T>
__device__ __forceinline__ void surfaceVelocity(const StepParams& P, int patch, int a, int sign, const T* in, T* out) {
    const int type = P.bc.vel[patch];
    if (type == FV_BC_FIXED_CELL) {
        for (int d = 0; d < 3; ++d) out[d] = (in[d] + T(P.bc.vel_value[patch][d])) * T(0.5);
    } else if (type == FV_BC_FIXED_SURFACE) {
        for (int d = 0; d < 3; ++d) out[d] = T(P.bc.vel_value[patch][d]);
    } else if (type == FV_BC_SLIP) {
        T n[3] = {T(0), T(0), T(0)};
        n[a] = T(sign);
        T vn = 0;
        vn += in[0] * n[0];
        vn += in[1] * n[1];
        vn += in[2] * n[2];
        for (int d = 0; d < 3; ++d) out[d] = in[d] - n[d] * vn;
    } else {
        for (int d = 0; d < 3; ++d) out[d] = in[d];
    }
}

template <typename T>
__device__ __forceinline__ T mag3d(T x, T y, T z) { return mag3<T>(x, y, z); }

// ---------------------------------------------------------------------------- k_faces
template <typename T, int NS, int EOS, int D>
__global__ void k_faces(const StepParams P, const GenericLayout L, const T* __restrict__ Pc, DevClock* __restrict__ ck,
                        T* __restrict__ FS) {
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long n = P.ncell;
    const double halfTimestep = 0.5 * ck->dt;
    const int nx = P.n[0], ny = P.n[1];
    int ijk[3];
    ijk[0] = (int)(i % nx);
    ijk[1] = D >= 2 ? (int)((i / nx) % ny) : 0;
    ijk[2] = D >= 3 ? (int)(i / ((long long)nx * ny)) : 0;
    const T rc[3] = {T(P.geo.cc[0][ijk[0]]), T(P.geo.cc[1][ijk[1]]), T(P.geo.cc[2][ijk[2]])};
    const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
    const T V = T(ex * ey * ez);
    bool bad = false;

    // faces of the cell in mesh.cpp order: [x-, x+, y+, y-, z-, z+]
    constexpr int NFC = 2 * D;
    int fa[NFC], fh[NFC];
    {
        int q = 0;
        fa[q] = 0; fh[q++] = 0;
        fa[q] = 0; fh[q++] = 1;
        if (D >= 2) { fa[q] = 1; fh[q++] = 1; fa[q] = 1; fh[q++] = 0; }
        if (D >= 3) { fa[q] = 2; fh[q++] = 0; fa[q] = 2; fh[q++] = 1; }
    }
    FaceGeo fg[NFC];
#pragma unroll
    for (int q = 0; q < NFC; ++q) fg[q] = faceOf(P, L, ijk, fa[q], fh[q]);

    // neighbours in mesh.cpp order [x-, x+, y-, y+, z-, z+]
    long long nbIdx[NFC];
    bool nbOk[NFC];
    T nbC[NFC][3];      // neighbour centre (unshifted)
    T nbSh[NFC];        // periodic shift of the neighbour along the face axis
    T nbD[NFC][3];      // rC_nb (+ periodic shift) - rC_i
#pragma unroll
    for (int q = 0; q < NFC; ++q) {
        const int a = q >> 1, hi = q & 1;
        int nb[3];
        double sh;
        nbOk[q] = neighbourOf(P, ijk, a, hi, nb, sh);
        if (nbOk[q]) {
            nbIdx[q] = cellIndex(P, nb[0], nb[1], nb[2]);
            nbSh[q] = T(sh);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                nbC[q][d] = T(P.geo.cc[d][nb[d]]);
                nbD[q][d] = d == a ? (nbC[q][d] + nbSh[q]) - rc[d] : nbC[q][d] - rc[d];
            }
        }
    }

    // limited gradients: scalar fields q in [0, NS) and p (q = NS+3) -> Lg[s][3];
    // velocity tensor -> Lv[9] ([3*component + direction])
    constexpr int NSC = NS + 1;
    T Lg[NSC][3];
    T Lv[9];
    T prim_i[NS + 4];
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) prim_i[q] = primAt<T, NS>(Pc, n, q, i);

    // face interpolation value of primitive q at face slot s
    auto faceValue = [&](int q, int s) -> T {
        const FaceGeo& g = fg[s];
        if (g.boundary) {
            if (q >= NS && q < NS + 3) {
                T vin[3] = {prim_i[NS], prim_i[NS + 1], prim_i[NS + 2]}, vout[3];
                surfaceVelocity<T>(P, g.patch, fa[s], g.sign, vin, vout);
                return vout[q - NS];
            }
            return surfaceScalar<T, NS>(P, g.patch, q, prim_i[q]);
        }
        // inner face: owner * wOwn + neighbour * wNei, weights from the centre distances
        const int a = fa[s];
        const int slot = (a << 1) | fh[s];
        const long long j = nbIdx[slot];
        const T vj = primAt<T, NS>(Pc, n, q, j);
        // distances |rC_f - rC_own|, |rC_f - rC_nei| (mesh.cpp:55-86); across a periodic wrap
        // face the neighbour-side cell sits one period further along the axis
        T dOwn[3], dNei[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T fc = T(g.rc[d]);
            T ownP, neiP;
            if (g.own) {
                ownP = rc[d];
                neiP = d == a ? nbC[slot][d] + nbSh[slot] : nbC[slot][d];
            } else {
                ownP = nbC[slot][d];
                neiP = d == a ? rc[d] - nbSh[slot] : rc[d];
            }
            dOwn[d] = fc - ownP;
            dNei[d] = fc - neiP;
        }
        const T ownR = mag3<T>(dOwn[0], dOwn[1], dOwn[2]);
        const T neiR = mag3<T>(dNei[0], dNei[1], dNei[2]);
        const T sumR = ownR + neiR;
        const T wOwn = neiR / sumR, wNei = ownR / sumR;
        const T vown = g.own ? prim_i[q] : vj, vnei = g.own ? vj : prim_i[q];
        return vown * wOwn + vnei * wNei;
    };
    (void)faceValue;

    // gradient of primitive q: [direction]
    auto gradient = [&](int q, T* gr) {
        T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int s = 0; s < NFC; ++s) {
            const T fv = faceValue(q, s);
            const int a = fa[s];
            const T nsgn = fg[s].own ? T(fg[s].sign) : T(-fg[s].sign);
            // (n * phi) * S with n = nsgn * e_a; the transverse components are (+-0 * phi) * S
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[d] += (d == a ? nsgn * fv : T(0) * fv) * T(fg[s].S);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) gr[d] = acc[d] / V;
    };

    // ghost-gradient deltas for boundary faces: d = (rC_f - rC_i) * 2
    // scalars
    const int lim = P.limiter;
#pragma unroll 1
    for (int s2 = 0; s2 < NSC; ++s2) {
        const int q = s2 < NS ? s2 : NS + 3;
        T gr[3];
        gradient(q, gr);
        T mn[3], mx[3];
        bool firstEntry = true;
        auto push = [&](const T* g) {
            if (firstEntry) {
#pragma unroll
                for (int d = 0; d < 3; ++d) { mn[d] = g[d]; mx[d] = g[d]; }
                firstEntry = false;
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) { mn[d] = smin(mn[d], g[d]); mx[d] = smax(mx[d], g[d]); }
            }
        };
#pragma unroll
        for (int slot = 0; slot < NFC; ++slot) {
            if (!nbOk[slot]) continue;
            const T* d3 = nbD[slot];
            const T dm = mag3<T>(d3[0], d3[1], d3[2]);
            const T dn[3] = {d3[0] / dm, d3[1] / dm, d3[2] / dm};
            const T diff = primAt<T, NS>(Pc, n, q, nbIdx[slot]) - prim_i[q];
            T g[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) g[d] = diff / dm * dn[d];
            push(g);
        }
#pragma unroll
        for (int s = 0; s < NFC; ++s) {
            if (!fg[s].boundary) continue;
            T d3[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) d3[d] = (T(fg[s].rc[d]) - rc[d]) * T(2);
            const T dm = mag3<T>(d3[0], d3[1], d3[2]);
            const T dn[3] = {d3[0] / dm, d3[1] / dm, d3[2] / dm};
            const T b = cellGhostScalar<T, NS>(P, fg[s].patch, q, prim_i[q], bad);
            T g[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) g[d] = (b - prim_i[q]) / dm * dn[d];
            push(g);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T r = mn[d] / (mx[d] + Num<T>::stab());
            T lg = limiterPhi<T>(lim, r, T(2) / (T(1) + r)) * gr[d];
            if (lim == FV_LIM_ZERO) lg = T(0);
            if (lim == FV_LIM_LINEAR) lg = gr[d];
            Lg[s2][d] = lg;
        }
    }
    // velocity tensor
    {
        T gr[9];  // [3*component + direction]
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T g3[3];
            gradient(NS + c, g3);
#pragma unroll
            for (int d = 0; d < 3; ++d) gr[3 * c + d] = g3[d];
        }
        T mn[9], mx[9];
        bool firstEntry = true;
        auto push = [&](const T* dv, const T* dn, T dm) {
            // neighbour gradient stored as [3*direction + component]
            T g[9];
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int c = 0; c < 3; ++c) g[3 * j + c] = dv[c] / dm * dn[j];
            if (firstEntry) {
#pragma unroll
                for (int m = 0; m < 9; ++m) { mn[m] = g[m]; mx[m] = g[m]; }
                firstEntry = false;
            } else {
#pragma unroll
                for (int m = 0; m < 9; ++m) { mn[m] = smin(mn[m], g[m]); mx[m] = smax(mx[m], g[m]); }
            }
        };
        const T vi[3] = {prim_i[NS], prim_i[NS + 1], prim_i[NS + 2]};
#pragma unroll
        for (int slot = 0; slot < NFC; ++slot) {
            if (!nbOk[slot]) continue;
            const T* d3 = nbD[slot];
            const T dm = mag3<T>(d3[0], d3[1], d3[2]);
            const T dn[3] = {d3[0] / dm, d3[1] / dm, d3[2] / dm};
            T dv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) dv[c] = primAt<T, NS>(Pc, n, NS + c, nbIdx[slot]) - vi[c];
            push(dv, dn, dm);
        }
#pragma unroll
        for (int s = 0; s < NFC; ++s) {
            if (!fg[s].boundary) continue;
            T d3[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) d3[d] = (T(fg[s].rc[d]) - rc[d]) * T(2);
            const T dm = mag3<T>(d3[0], d3[1], d3[2]);
            const T dn[3] = {d3[0] / dm, d3[1] / dm, d3[2] / dm};
            T gv[3];
            ghostVelocity<T>(P.bc.vel[fg[s].patch], P.bc.vel_value[fg[s].patch], fa[s], fg[s].sign, vi, gv);
            if (P.bc.vel[fg[s].patch] == FV_BC_FIXED_SURFACE) bad = true;
            T dv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) dv[c] = gv[c] - vi[c];
            push(dv, dn, dm);
        }
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            const T r = mn[m] / (mx[m] + Num<T>::stab());
            T lv = limiterPhi<T>(lim, r, T(2) / (T(1) + r)) * gr[m];
            if (lim == FV_LIM_ZERO) lv = T(0);
            if (lim == FV_LIM_LINEAR) lv = gr[m];
            Lv[m] = lv;
        }
    }
    if (bad) raise(ck, FV_ERR_BOUNDARY);

    // reconstruction + closure at every face, Hancock divergence over the cell's faces
    T divR[NS + 1], divM[3], divE = T(0);
#pragma unroll
    for (int k = 0; k <= NS; ++k) divR[k] = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) divM[d] = T(0);
    const long long nf = L.nfaces;
#pragma unroll
    for (int s = 0; s < NFC; ++s) {
        const FaceGeo& g = fg[s];
        T delta[3];
        {
            const int a = fa[s];
            const int slot = (a << 1) | fh[s];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const T self = (!g.own && !g.boundary && d == a) ? rc[d] - nbSh[slot] : rc[d];
                delta[d] = T(g.rc[d]) - self;
            }
        }
        FaceState<T, NS> st;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            T dot = T(0);
            dot += Lg[k - 1][0] * delta[0];
            dot += Lg[k - 1][1] * delta[1];
            dot += Lg[k - 1][2] * delta[2];
            st.c[k] = dot + prim_i[k - 1];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
            st.v[c] = prim_i[NS + c] + (Lv[3 * c] * delta[0] + Lv[3 * c + 1] * delta[1] + Lv[3 * c + 2] * delta[2]);
        {
            T dot = T(0);
            dot += Lg[NS][0] * delta[0];
            dot += Lg[NS][1] * delta[1];
            dot += Lg[NS][2] * delta[2];
            st.p = dot + prim_i[NS + 3];
        }
        closeFromPrimitive<T, NS, EOS>(P.mix, st);
        if (!P.hancock) {
            // SecondOrderRK stage (Advection2dOrder.cpp): the closed reconstruction is the face state
            soundSpeed<T, NS, EOS>(P.mix, st);
            storeFace<T, NS>(FS, L.nfaces, g.own ? 0 : 1, g.f, st);
            continue;
        }
        const int a = fa[s];
        const T nsg = g.own ? T(g.sign) : T(-g.sign);
        const T S = T(g.S);
#pragma unroll
        for (int k = 0; k <= NS; ++k) divR[k] += (st.v[a] * st.rho[k]) * nsg * S;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            T t = (st.m[d] * st.v[a]) * nsg;
            if (d == a) t = t + nsg * (st.p + T(0));
            divM[d] += t * S;
        }
        divE += ((st.v[a] * st.E) * nsg + (st.v[a] * (st.p + T(0))) * nsg) * S;
        storeFace<T, NS>(FS, nf, g.own ? 0 : 1, g.f, st);
    }
    if (!P.hancock) return;
#pragma unroll
    for (int k = 0; k <= NS; ++k) divR[k] /= V;
#pragma unroll
    for (int d = 0; d < 3; ++d) divM[d] /= V;
    divE /= V;
#pragma unroll
    for (int s = 0; s < NFC; ++s) {
        const FaceGeo& g = fg[s];
        FaceState<T, NS> st;
        loadFace<T, NS>(FS, nf, g.own ? 0 : 1, g.f, st);
#pragma unroll
        for (int k = 0; k <= NS; ++k) st.rho[k] -= divR[k] * T(halfTimestep);
#pragma unroll
        for (int d = 0; d < 3; ++d) st.m[d] -= divM[d] * T(halfTimestep);
        st.E -= divE * T(halfTimestep);
        closeFromConserved<T, NS, EOS>(P.mix, st);
        soundSpeed<T, NS, EOS>(P.mix, st);
        storeFace<T, NS>(FS, nf, g.own ? 0 : 1, g.f, st);
    }
}

// ---------------------------------------------------------------------------- k_faces3
// ThirdOrder reconstruction (Advection3dOrder.cpp:56-235 with templates/thirdOrderLimiter.hpp):
// surface gradients at every face of the cell (gradient.hpp:96-168: inner faces
// (phi_N - phi_O) / |d|^2 * d, patches (ghost - phi_O) / |dR| * dR / |dR| with dR = 2 (r_f - r_O)),
// for each face the limited gradient against the cell's farthest other face, component by
// component 0.5 ((1 - 1/3) phi(r) g_far + (1 + 1/3) phi(1 / (r + eps)) g_face) with
// r = g_face / (g_far + eps) and the limiter without its xi bound, then the face value
// phi_i + g . delta, closure and sound speed (no predictor).

// <Name>LimiterCalculation(r) of src/limiters/*.cpp (calculateNoRSLimit); linear: 1.
template <typename T> __device__ __forceinline__ T limiterPhiNoRS(int lim, T r) {
    const T one = 1, two = 2;
    switch (lim) {
    case FV_LIM_ZERO: return 0;
    case FV_LIM_MINMOD: return r <= T(0) ? T(0) : (r <= one ? r : one);
    case FV_LIM_VANLEER: return r < T(0) ? T(0) : two * r / (one + r);
    case FV_LIM_LINEAR: return one;
    case FV_LIM_VANALBADA: return r <= T(0) ? T(0) : (r * r + r) / (one + r * r);
    case FV_LIM_HQUICK: return r <= T(0) ? T(0) : T(4) * r / (T(3) + r);
    case FV_LIM_VANLEER2: {
        if (r <= T(0)) return 0;
        const T denom = one + r;
        return T(4) * r / (denom * denom);
    }
    case FV_LIM_SUPERBEE:
        if (r <= T(0)) return 0;
        if (r <= T(0.5)) return two * r;
        if (r <= one) return r;
        return smin(r, two);
    case FV_LIM_VANALBADA2: return r <= T(0) ? T(0) : two * r / (one + r * r);
    case FV_LIM_MINMOD2: return r <= T(0) ? T(0) : smin(one, T(4) * r / (one + r));
    case FV_LIM_SWEBY: {
        const T b = 2;
        return r <= T(0) ? T(0) : smin(smin(one, b * r), smin(b, r));
    }
    case FV_LIM_KOREN: return r <= T(0) ? T(0) : smin(smin(two * r, (one + two * r) / T(3)), two);
    case FV_LIM_KOREN2: {
        const T tt = T(2. / 3.);
        if (r <= T(0)) return smin(T(0), smax(-tt, (one + two * r) / T(3)));
        return smin(two * tt * r, smin((one + two * r) / T(3), two));
    }
    case FV_LIM_UTCDFS:
        if (r < T(-1)) return r * (r + one) / (r * r + one);
        if ((r >= T(-1)) && (r < T(0))) return 0;
        if ((r >= T(0)) && (r < T(0.5))) return r * r * r - two * (r * r) + two * r;
        if ((r >= T(0.5)) && (r < two)) return T(0.75) * r + T(0.25);
        return (two * (r * r) - two * r - T(9.0 / 4.0)) / (r * r - r - one);
    case FV_LIM_SCHMIDTMANN: {
        const T alpha = 1, beta = 2, gamma = 1.5;
        const T phiO3 = (two + r) / T(3);
        return smax(T(0), smin(phiO3, smax(-alpha * r, smin(smin(beta * r, phiO3), gamma))));
    }
    }
    return 0;
}

template <typename T> __device__ __forceinline__ T thirdOrderComponent(int lim, T g1, T g2) {
    const T r = g1 / (g2 + Num<T>::stab());
    const T retr = T(1) / (r + Num<T>::stab());
    T limGrad, limOpp;
    if (lim == FV_LIM_ZERO) {
        limGrad = T(0);
        limOpp = T(0);
    } else if (lim == FV_LIM_LINEAR) {
        limGrad = g1;
        limOpp = g2;
    } else {
        limGrad = limiterPhiNoRS<T>(lim, retr) * g1;
        limOpp = limiterPhiNoRS<T>(lim, r) * g2;
    }
    return T(0.5) * ((T(1) - T(1. / 3.)) * limOpp + (T(1) + T(1. / 3.)) * limGrad);
}

// thirdOrderLimiterCada (templates/thirdOrderLimiterCada.hpp:19-133) for one face and the
// cell's farthest face, NC gradient components in storage order: dx2 = (1 / minLS)^2 with minLS
// the cell's 1 / min edge (Schemi.cpp:648-662), eta = (dx2 (gN & gN) + dx2 (gO & gO)) /
// (sqrt(5/2) (8 pi)^2 dx2); below 1 - 1e-6 the unlimited 0.5 ((1 - 1/3) gO + (1 + 1/3) gN),
// above 1 + 1e-6 thirdOrderComponent, in between 0.5 ((1 - e) unlimited + (1 + e) limited) with
// e = (eta - 1) / 1e-6.
template <typename T, int NC>
__device__ __forceinline__ void cadaLimit(int lim, const T* gN, const T* gO, T minLS, T* out) {
    const T pi8 = T(8) * T(3.14159265358979323846);
    const T alpha = pi8 * pi8, eps = T(1E-6);
    const T inv = T(1) / minLS;
    const T dx2 = inv * inv;
    T sN = T(0), sO = T(0);
#pragma unroll
    for (int q = 0; q < NC; ++q) sN += gN[q] * gN[q];
#pragma unroll
    for (int q = 0; q < NC; ++q) sO += gO[q] * gO[q];
    const T delta2Near = dx2 * sN, delta2Oppose = dx2 * sO;
    const T eta = (delta2Near + delta2Oppose) / (sqrt(T(5.0 / 2.0)) * alpha * dx2);
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const T unlimited = T(0.5) * ((T(1) - T(1. / 3.)) * gO[q] + (T(1) + T(1. / 3.)) * gN[q]);
        if (eta < (T(1) - eps)) {
            out[q] = unlimited;
        } else {
            const T limited = thirdOrderComponent<T>(lim, gN[q], gO[q]);
            if (eta > (T(1) + eps)) {
                out[q] = limited;
            } else {
                const T eta1eps = (eta - T(1)) / eps;
                out[q] = T(0.5) * ((T(1) - eta1eps) * unlimited + (T(1) + eta1eps) * limited);
            }
        }
    }
}

template <typename T, int NS, int EOS, int D>
__global__ void k_faces3(const StepParams P, const GenericLayout L, const T* __restrict__ Pc, DevClock* __restrict__ ck,
                         T* __restrict__ FS) {
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long n = P.ncell;
    const int nx = P.n[0], ny = P.n[1];
    int ijk[3];
    ijk[0] = (int)(i % nx);
    ijk[1] = D >= 2 ? (int)((i / nx) % ny) : 0;
    ijk[2] = D >= 3 ? (int)(i / ((long long)nx * ny)) : 0;
    const T rc[3] = {T(P.geo.cc[0][ijk[0]]), T(P.geo.cc[1][ijk[1]]), T(P.geo.cc[2][ijk[2]])};
    bool bad = false;
    const int lim = P.limiter;
    const bool cada = P.cada != 0;
    // the cell's minimal length scale (1 / min edge) of the Cada switch
    const T minLS = T(1) / smin(smin(T(extent(P, 0, ijk[0])), T(extent(P, 1, ijk[1]))), T(extent(P, 2, ijk[2])));

    // faces of the cell in mesh.cpp order: [x-, x+, y+, y-, z-, z+]
    constexpr int NFC = 2 * D;
    int fa[NFC], fh[NFC];
    {
        int q = 0;
        fa[q] = 0; fh[q++] = 0;
        fa[q] = 0; fh[q++] = 1;
        if (D >= 2) { fa[q] = 1; fh[q++] = 1; fa[q] = 1; fh[q++] = 0; }
        if (D >= 3) { fa[q] = 2; fh[q++] = 0; fa[q] = 2; fh[q++] = 1; }
    }
    FaceGeo fg[NFC];
    long long nbIdx[NFC];
    T nbSh[NFC];     // periodic shift of the neighbour across face s along its axis
    T fc[NFC][3];    // face centre seen from this cell
#pragma unroll
    for (int s = 0; s < NFC; ++s) {
        fg[s] = faceOf(P, L, ijk, fa[s], fh[s]);
        int nb[3];
        double sh = 0;
        nbIdx[s] = -1;
        nbSh[s] = T(0);
        if (!fg[s].boundary && neighbourOf(P, ijk, fa[s], fh[s], nb, sh)) {
            nbIdx[s] = cellIndex(P, nb[0], nb[1], nb[2]);
            nbSh[s] = T(sh);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d)
            fc[s][d] = (!fg[s].own && !fg[s].boundary && d == fa[s]) ? T(fg[s].rc[d]) + nbSh[s] : T(fg[s].rc[d]);
    }
    T prim_i[NS + 4];
#pragma unroll
    for (int q = 0; q < NS + 4; ++q) prim_i[q] = primAt<T, NS>(Pc, n, q, i);

    // surface gradients: scalars (c_1..c_N, p) sgS[s][j][3], velocity sgV[s][9] ([3*component + direction])
    constexpr int NSC = NS + 1;
    T sgS[NFC][NSC][3];
    T sgV[NFC][9];
#pragma unroll
    for (int s = 0; s < NFC; ++s) {
        const FaceGeo& g = fg[s];
        const int a = fa[s];
        if (g.boundary) {
            T d3[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) d3[d] = (T(g.rc[d]) - rc[d]) * T(2);
            const T dm = mag3<T>(d3[0], d3[1], d3[2]);
            const T dn[3] = {d3[0] / dm, d3[1] / dm, d3[2] / dm};
#pragma unroll
            for (int j = 0; j < NSC; ++j) {
                const int q = j < NS ? j : NS + 3;
                const T b = cellGhostScalar<T, NS>(P, g.patch, q, prim_i[q], bad);
                const T qv = (b - prim_i[q]) / dm;
#pragma unroll
                for (int d = 0; d < 3; ++d) sgS[s][j][d] = qv * dn[d];
            }
            const T vi[3] = {prim_i[NS], prim_i[NS + 1], prim_i[NS + 2]};
            T gv[3];
            ghostVelocity<T>(P.bc.vel[g.patch], P.bc.vel_value[g.patch], a, g.sign, vi, gv);
            if (P.bc.vel[g.patch] == FV_BC_FIXED_SURFACE) bad = true;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T qv = (gv[c] - vi[c]) / dm;
#pragma unroll
                for (int d = 0; d < 3; ++d) sgV[s][3 * c + d] = qv * dn[d];
            }
        } else {
            // the face's owner and neighbour cells; the neighbour centre shifted by one period
            // across a wrap face
            const long long j = nbIdx[s];
            const int nbAxis = fh[s] ? ijk[a] + 1 : ijk[a] - 1;
            const int na = P.n[a];
            const int nbA = nbAxis < 0 ? nbAxis + na : (nbAxis >= na ? nbAxis - na : nbAxis);
            T dvec[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const T cNb = d == a ? T(P.geo.cc[a][nbA]) : rc[d];
                const T cOwn = g.own ? rc[d] : cNb;
                const T cNei = g.own ? cNb : rc[d];
                const T shift = d == a ? (g.own ? nbSh[s] : -nbSh[s]) : T(0);
                dvec[d] = (cNei + shift) - cOwn;
            }
            const T m = mag3<T>(dvec[0], dvec[1], dvec[2]);
            const T m2 = m * m;
            const long long iOwn = g.own ? i : j, iNei = g.own ? j : i;
#pragma unroll
            for (int jj = 0; jj < NSC; ++jj) {
                const int q = jj < NS ? jj : NS + 3;
                const T qv = (primAt<T, NS>(Pc, n, q, iNei) - primAt<T, NS>(Pc, n, q, iOwn)) / m2;
#pragma unroll
                for (int d = 0; d < 3; ++d) sgS[s][jj][d] = qv * dvec[d];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T qv = (primAt<T, NS>(Pc, n, NS + c, iNei) - primAt<T, NS>(Pc, n, NS + c, iOwn)) / m2;
#pragma unroll
                for (int d = 0; d < 3; ++d) sgV[s][3 * c + d] = qv * dvec[d];
            }
        }
    }
    if (bad) raise(ck, FV_ERR_BOUNDARY);

#pragma unroll
    for (int s = 0; s < NFC; ++s) {
        // farthest other face of the cell (first of equals)
        int far = 0;
        T best = T(0);
#pragma unroll
        for (int s2 = 0; s2 < NFC; ++s2) {
            if (s2 == s) continue;
            const T dist = mag3<T>(fc[s2][0] - fc[s][0], fc[s2][1] - fc[s][1], fc[s2][2] - fc[s][2]);
            if (best < dist) {
                best = dist;
                far = s2;
            }
        }
        const FaceGeo& g = fg[s];
        const int a = fa[s];
        T delta[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T self = (!g.own && !g.boundary && d == a) ? rc[d] - nbSh[s] : rc[d];
            delta[d] = T(g.rc[d]) - self;
        }
        FaceState<T, NS> st;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            T lg[3];
            if (cada) {
                cadaLimit<T, 3>(lim, sgS[s][k - 1], sgS[far][k - 1], minLS, lg);
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) lg[d] = thirdOrderComponent<T>(lim, sgS[s][k - 1][d], sgS[far][k - 1][d]);
            }
            T dot = T(0);
            dot += lg[0] * delta[0];
            dot += lg[1] * delta[1];
            dot += lg[2] * delta[2];
            st.c[k] = dot + prim_i[k - 1];
        }
        T lv[9];
        if (cada) {
            cadaLimit<T, 9>(lim, sgV[s], sgV[far], minLS, lv);
        } else {
#pragma unroll
            for (int m = 0; m < 9; ++m) lv[m] = thirdOrderComponent<T>(lim, sgV[s][m], sgV[far][m]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
            st.v[c] = prim_i[NS + c] + (lv[3 * c] * delta[0] + lv[3 * c + 1] * delta[1] + lv[3 * c + 2] * delta[2]);
        {
            T lp[3];
            if (cada) {
                cadaLimit<T, 3>(lim, sgS[s][NS], sgS[far][NS], minLS, lp);
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) lp[d] = thirdOrderComponent<T>(lim, sgS[s][NS][d], sgS[far][NS][d]);
            }
            T dot = T(0);
            dot += lp[0] * delta[0];
            dot += lp[1] * delta[1];
            dot += lp[2] * delta[2];
            st.p = dot + prim_i[NS + 3];
        }
        closeFromPrimitive<T, NS, EOS>(P.mix, st);
        soundSpeed<T, NS, EOS>(P.mix, st);
        storeFace<T, NS>(FS, L.nfaces, g.own ? 0 : 1, g.f, st);
    }
}

// ---------------------------------------------------------------------------- k_fluxes
template <typename T, int NS, int EOS, int D>
__global__ void k_fluxes(const StepParams P, const GenericLayout L, const T* __restrict__ FS, DevClock* __restrict__ ck,
                         T* __restrict__ FL) {
    if (ck->done) return;
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= L.nfaces) return;
    int a = 0;
    while (a + 1 < D && f >= L.faceBase[a + 1]) ++a;
    const long long local = f - L.faceBase[a];
    const int n = P.n[a];
    const int fi = (int)(local % (n + 1));
    if (P.periodic[a] && fi == 0) return;  // unused slot
    const long long nf = L.nfaces;
    FaceState<T, NS> O, B;
    loadFace<T, NS>(FS, nf, 0, f, O);
    const bool boundary = !P.periodic[a] && (fi == 0 || fi == n);
    FaceFlux<T, NS> F;
    bool ok;
    T sv[3], sp = T(0);
    T* svp = P.starV ? sv : nullptr;
    T* spp = P.starP ? &sp : nullptr;
    if (boundary) {
        const int sign = fi == 0 ? -1 : 1;
        const int patch = a == 0 ? (fi == 0 ? FV_PATCH_TAIL : FV_PATCH_POINT)
                                 : a == 1 ? (fi == 0 ? FV_PATCH_RIGHT : FV_PATCH_LEFT)
                                          : (fi == 0 ? FV_PATCH_BOTTOM : FV_PATCH_TOP);
        ghostState<T, NS, EOS>(P.mix, P.bc, patch, a, sign, O, B);
        ok = riemann<T, NS, EOS>(P.flux, a, sign, O, B, F, svp, spp, &P.mix);
    } else {
        loadFace<T, NS>(FS, nf, 1, f, B);
        ok = riemann<T, NS, EOS>(P.flux, a, 1, O, B, F, svp, spp, &P.mix);
    }
    if (!ok) raise(ck, FV_ERR_RIEMANN);
    if (P.starV) {
#pragma unroll
        for (int d = 0; d < 3; ++d) P.starV[d * nf + f] = double(sv[d]);
    }
    if (P.starP) P.starP[f] = double(sp);
    int q = 0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) FL[(q++) * nf + f] = F.rho[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) FL[(q++) * nf + f] = F.m[d];
    FL[(q++) * nf + f] = F.E;
}

// ---------------------------------------------------------------------------- k_update
template <typename T, int NS, int EOS, int D>
__global__ void k_update(const StepParams P, const GenericLayout L, const double* __restrict__ U,
                         double* __restrict__ Un, const T* __restrict__ Pc, const T* __restrict__ FL,
                         DevClock* __restrict__ ck, double* __restrict__ blockMax) {
    __shared__ T red[32];
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    T localMax = T(-1);
    if (i < P.ncell) {
        const double dt = ck->dt;
        const long long n = P.ncell, st = P.stride, nf = L.nfaces;
        int ijk[3];
        ijk[0] = (int)(i % P.n[0]);
        ijk[1] = D >= 2 ? (int)((i / P.n[0]) % P.n[1]) : 0;
        ijk[2] = D >= 3 ? (int)(i / ((long long)P.n[0] * P.n[1])) : 0;
        const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
        const T V = T(ex * ey * ez);
        const T minLS = T(1) / smin(smin(T(ex), T(ey)), T(ez));
        constexpr int NFC = 2 * D;
        int fa[NFC], fh[NFC];
        {
            int q = 0;
            fa[q] = 0; fh[q++] = 0;
            fa[q] = 0; fh[q++] = 1;
            if (D >= 2) { fa[q] = 1; fh[q++] = 1; fa[q] = 1; fh[q++] = 0; }
            if (D >= 3) { fa[q] = 2; fh[q++] = 0; fa[q] = 2; fh[q++] = 1; }
        }
        constexpr int NQ = NS + 1 + 3 + 1;
        T acc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = T(0);
#pragma unroll
        for (int s = 0; s < NFC; ++s) {
            const FaceGeo g = faceOf(P, L, ijk, fa[s], fh[s]);
            const T sg = g.own ? T(1) : T(-1);
            const T S = T(g.S);
#pragma unroll
            for (int q = 0; q < NQ; ++q) acc[q] += FL[q * nf + g.f] * sg * S;
        }
        // acc order: rho[0..NS], m[0..2], E
        const T vOld[3] = {Pc[(NS + 0) * n + i], Pc[(NS + 1) * n + i], Pc[(NS + 2) * n + i]};
        const T rho0Old = T(U[NS * st + i]);
        double Enew = U[(NS + 4) * st + i] - double(acc[NS + 4] / V) * dt;
        double mNew[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d < P.nmom) mNew[d] = U[(NS + 1 + d) * st + i] - double(acc[NS + 1 + d] / V) * dt;
        if (P.gravity) {
            T vg = 0;
            vg += vOld[0] * T(ck->g[0]);
            vg += vOld[1] * T(ck->g[1]);
            vg += vOld[2] * T(ck->g[2]);
            Enew += double(rho0Old * vg) * dt;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (d < P.nmom) mNew[d] += double(T(ck->g[d]) * rho0Old) * dt;
        }
        double rNew[NS + 1];
#pragma unroll
        for (int k = 0; k <= NS; ++k) rNew[k] = U[(k == 0 ? NS : k - 1) * st + i] - double(acc[k] / V) * dt;
#pragma unroll
        for (int k = 1; k <= NS; ++k) Un[(k - 1) * st + i] = rNew[k];
        Un[NS * st + i] = rNew[0];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d < P.nmom) Un[(NS + 1 + d) * st + i] = mNew[d];
        Un[(NS + 4) * st + i] = Enew;
        T rhoN[NS + 1], mN[3];
#pragma unroll
        for (int k = 0; k <= NS; ++k) rhoN[k] = T(rNew[k]);
#pragma unroll
        for (int d = 0; d < 3; ++d) mN[d] = T(mNew[d]);
        localMax = cellSignal<T, NS, EOS, D>(P, rhoN, rhoN[0], mN, T(Enew), minLS);
    }
    const T bm = blockMaxReduce<T>(localMax, red);
    if (threadIdx.x == 0) blockMax[blockIdx.x] = double(bm);
    // the advected state's primitives follow from its conserved variables again (k_prim of this
    // step has read the flag)
    if (i == 0) ck->stagePrim = 0;
    if (P.fuseFinalize) finalizeIfLast(P, ck, blockMax, (int)gridDim.x, gridDim.x);
}

}  // namespace fv
