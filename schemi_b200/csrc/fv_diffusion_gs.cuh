// fv_diffusion_gs.cuh -- the diffusion stage with the Gauss-Seidel solver (#Type_of_SLE_solver_flag
// GaussSeidel): the implicit matrices of SLEMatrix::generateDTimeLaplacian (SLEMatrix.cpp:410-546,
// 706-907) and GaussSeidelSolver::algorithm (GaussSeidelSolver.cpp:12-82), FP64 in the
// reference's operation order.
//
// Matrix of a field phi with face coefficient D_f: diagonal rNew / dt + sum over the cell's faces
// (in its face order) of D_f / |d| (n S / V & d / |d|), free term rOld / dt plus, on a patch, that
// coefficient times the ghost value; the neighbour of an inner face gets -D_f / |d| (...).  On
// this mesh n = +-e_a and an inner face's d lies along a, so the product is n_a S / V d_a / |d|
// (the other terms add zeros); a patch's d = 2 (r_f - r_C) enters through |d| and d_a / |d|.
//
// The solver sweeps forward, then backward, until 100 max |(new - old) / (|new| + eps)| < 1e-12 or
// the iteration limit.  The backward sweep recomputes every cell from the old iterate of its lower
// neighbours and the new one of its upper neighbours, so the forward sweep's values are never
// read and the iterate is the backward sweep's alone.  Cells with the same i + j + k depend on
// none of each other in that sweep: k_gs_solve runs it as wavefronts of decreasing i + j + k in
// one CTA (the order of every cell's own operations is the reference's), a 1D mesh on one thread.
// Without a periodic axis the lower neighbours of cell (i, j, k) in its face order are x-, y-, z-
// and the upper ones x+, y+, z+.
#pragma once

#include "fv_diffusion.cuh"

namespace fv {
namespace diff {

// geometry of face slot s of cell ijk: the neighbour (or -1 on a patch), |d| and (n S / V)_a d_a / |d|
struct FaceCoef {
    long long nb;
    double m, dot;
    FaceGeo g;
};
template <int D>
__device__ __forceinline__ FaceCoef faceCoef(const StepParams& P, const GenericLayout& L, const int* ijk, int a, int hi,
                                             const double* rc, double V) {
    FaceCoef c;
    c.g = faceOf(P, L, ijk, a, hi);
    double dR[3];
    double onA;
    if (!c.g.boundary) {
        int nbc[3];
        double sh;
        neighbourOf(P, ijk, a, hi, nbc, sh);
        c.nb = cellIndex(P, nbc[0], nbc[1], nbc[2]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double cn = P.geo.cc[d][nbc[d]];
            dR[d] = (d == a ? cn + sh : cn) - rc[d];
        }
        onA = c.g.own ? (1.0 * c.g.S) / V : ((1.0 * c.g.S) / V) * -1;
    } else {
        c.nb = -1;
#pragma unroll
        for (int d = 0; d < 3; ++d) dR[d] = (c.g.rc[d] - rc[d]) * 2;
        onA = (double(c.g.sign) * c.g.S) / V;
    }
    c.m = mag3<double>(dR[0], dR[1], dR[2]);
    c.dot = onA * (dR[a] / c.m);
    return c;
}

template <int D> __device__ __forceinline__ void faceOrder(int* fa, int* fh) {
    int q = 0;
    fa[q] = 0; fh[q++] = 0;
    fa[q] = 0; fh[q++] = 1;
    if (D >= 2) { fa[q] = 1; fh[q++] = 1; fa[q] = 1; fh[q++] = 0; }
    if (D >= 3) { fa[q] = 2; fh[q++] = 0; fa[q] = 2; fh[q++] = 1; }
}

// ----------------------------------------------------------------------------- k_gs_wmat
// the mass fractions' matrices (coefficient rho D_k of the face) and the molar-mass correction
// distributed into them (Diffusion.cpp:321-339, 396-412)
template <int NS, int EOS, int D>
__global__ void k_gs_wmat(const StepParams P, const GenericLayout L, const DiffParams X, const double* __restrict__ U,
                          DevClock* __restrict__ ck) {
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long st = P.stride, nf = L.nfaces;
    const double rt = 1 / ck->dt;
    int ijk[3];
    cellAxisCoords(P, i, D, ijk);
    const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
    const double V = ex * ey * ez;
    const double rc[3] = {P.geo.cc[0][ijk[0]], P.geo.cc[1][ijk[1]], P.geo.cc[2][ijk[2]]};
    const double* cp = X.cellPrim;
    const double* F = X.face;
    const double rho0 = U[NS * st + i];
    double c[NS + 1], w[NS];
    c[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = cp[(k - 1) * st + i];
        c[0] += c[k];
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) w[k] = cp[(NS + 5 + k) * st + i];
    // the patch's concentrations as cell values (calculatedMassFraction's ghosts)
    double diag[NS], free[NS], divC[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        diag[k] = rho0 * rt;
        free[k] = (w[k] * rho0) * rt;
        divC[k] = 0;
    }
    bool bad = false;
    constexpr int NFC = 2 * D;
    int fa[NFC], fh[NFC];
    faceOrder<D>(fa, fh);
#pragma unroll
    for (int s = 0; s < NFC; ++s) {
        const FaceCoef fc = faceCoef<D>(P, L, ijk, fa[s], fh[s], rc, V);
        const long long f = fc.g.f;
        const double sRho = F[slotRho<NS>() * nf + f];
        double cB[NS + 1], sum = 0;
        if (fc.nb < 0) {
            cB[0] = 0;
#pragma unroll
            for (int k = 1; k <= NS; ++k) {
                cB[k] = cellGhostScalar<double, NS>(P, fc.g.patch, k - 1, c[k], bad);
                cB[0] += cB[k];
            }
#pragma unroll
            for (int q = 1; q <= NS; ++q) sum += cB[q] * P.mix.M[q - 1];
        }
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const double rhoD = sRho * F[slotDs<NS>(k) * nf + f];
            const double coef = rhoD / fc.m * fc.dot;
            diag[k] += coef;
            if (fc.nb >= 0) {
                X.wOff[(k * 6 + s) * st + i] = -rhoD / fc.m * fc.dot;
            } else {
                X.wOff[(k * 6 + s) * st + i] = 0;
                free[k] += coef * ((cB[k + 1] * P.mix.M[k]) / sum);
            }
        }
        if (X.molmass) {
            const double nsg = fc.g.own ? double(fc.g.sign) : double(-fc.g.sign);
#pragma unroll
            for (int k = 0; k < NS; ++k) divC[k] += F[slotCorr<NS>(k) * nf + f] * nsg * fc.g.S;
        }
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double dk = diag[k], fk = free[k];
        if (X.molmass) {
            const double s = (divC[k] / V) * (-1.0);
            if (s >= 0.) fk += s;
            else dk -= s / (w[k] + Num<double>::stab());
        }
        X.wDiag[k * st + i] = dk;
        X.wFree[k * st + i] = fk;
        X.sol[k * st + i] = w[k];  // the solve's start: the current mass fraction
    }
    if (bad) raise(ck, FV_ERR_BOUNDARY);
}


// ----------------------------------------------------------------------------- k_gs_solve
// One CTA solves diag x + off x = free for the field in x (start in, solution out): backward
// sweeps as wavefronts of decreasing i + j (+ k), the convergence test of each sweep over all
// cells.  Each cell computes, in the reference's order, x = free / diag - sum of off x / diag over
// the lower neighbours in reverse face order (z-, y-, x-: the old iterate) and then the upper ones
// (z+, y+, x+: this sweep's new values).
constexpr int kGsThreads = 1024;
// the two iterates (and in split mode the helpers' slots) in shared memory up to this many bytes
// (else the iterates in global memory)
constexpr int kGsSmemBytes = 200 * 1024;
// split mode: per column 2 slots of the lower part and 2 x 4 coefficients
constexpr int kGsRoleDoubles = 2 + 8;

// one cell's coefficients: 1 / diag (the same value each sweep, formed once per solve), free, the
// off-diagonal per face slot
struct GsCoef {
    double aii, free, o[6];
};
template <int D>
__device__ __forceinline__ void gsLoad(const StepParams& P, long long i, const double* aiiI,
                                       const double* __restrict__ free, const double* __restrict__ off, GsCoef& c) {
    const long long st = P.stride;
    c.aii = aiiI[i];
    c.free = free[i];
#pragma unroll
    for (int s = 0; s < 2 * D; ++s) c.o[s] = off[s * st + i];
}
// free / diag less the lower neighbours' terms (the old iterate: known before the sweep reaches
// the cell), then the upper neighbours' (this sweep's new values)
template <int D>
__device__ __forceinline__ double gsLower(const StepParams& P, long long i, const int* ijk, const GsCoef& c,
                                          const double* oldI) {
    const double aii = c.aii;
    double x = c.free * aii;
    const long long sy = P.n[0], sz = (long long)P.n[0] * P.n[1];
    if (D >= 3 && ijk[2] > 0) x -= c.o[4] * oldI[i - sz] * aii;
    if (D >= 2 && ijk[1] > 0) x -= c.o[3] * oldI[i - sy] * aii;
    if (ijk[0] > 0) x -= c.o[0] * oldI[i - 1] * aii;
    return x;
}
template <int D>
__device__ __forceinline__ double gsUpper(const StepParams& P, long long i, const int* ijk, const GsCoef& c,
                                          double x, const double* newI) {
    const double aii = c.aii;
    const long long sy = P.n[0], sz = (long long)P.n[0] * P.n[1];
    if (D >= 3 && ijk[2] < P.n[2] - 1) x -= c.o[5] * newI[i + sz] * aii;
    if (D >= 2 && ijk[1] < P.n[1] - 1) x -= c.o[2] * newI[i + sy] * aii;
    if (ijk[0] < P.n[0] - 1) x -= c.o[1] * newI[i + 1] * aii;
    return x;
}
template <int D>
__device__ __forceinline__ double gsUpdate(const StepParams& P, long long i, const int* ijk, const GsCoef& c,
                                           const double* oldI, const double* newI) {
    return gsUpper<D>(P, i, ijk, c, gsLower<D>(P, i, ijk, c, oldI), newI);
}
// the reference loop's convergence measure of one cell, as a test: 100 max_i r_i < 1e-12 holds
// exactly when no cell has 100 r_i >= 1e-12 (the rounded product is monotone in r), a NaN at the
// first cell failing it (its value is taken as it is) and elsewhere passed over (taken only when
// larger)
__device__ __forceinline__ bool gsFails(long long i, double v, double old) {
    const double r = fabs((v - old) / (fabs(v) + Num<double>::stab()));
    return i == 0 ? !(100. * r < 1e-12) : (100. * r >= 1e-12);
}

// The sweep's cells of one wavefront are one per column (2D: the cells of one x; 3D: of one
// (x, y)), so a thread keeps its columns over the whole solve and walks down each.  With at most
// one column per thread the work between two barriers is pipelined: the thread applies to its
// cell only the upper neighbours' terms (the values of the wavefront just computed), and then
// forms its next cell's lower part (free / diag and the old iterate's terms, whose coefficients
// it loaded a wavefront earlier) and loads the coefficients of the cell after that; the
// convergence test runs over all cells after the sweep.  The iterates live in shared memory when
// both fit (useSmem), else in work[0..2); 1 / diag in work[2] (work[0] with useSmem).
template <int D>
__global__ void __launch_bounds__(kGsThreads) k_gs_solve(const StepParams P, const double* __restrict__ diag,
                                                          const double* __restrict__ free,
                                                          const double* __restrict__ off, double* __restrict__ x,
                                                          double* __restrict__ work, int maxIt, int useSmem,
                                                          DevClock* __restrict__ ck) {
    extern __shared__ double gsSmem[];
    if (ck->done) return;
    const long long n = P.ncell, rs = P.stride;
    // split mode (2D / 3D, at most 512 columns, launched with two threads per column rounded to
    // warps): the first W threads apply each column's upper terms, the other W prepare the next
    // cell's lower part and coefficients, in shared memory ahead of the iterates
    const int ncolAll = D == 1 ? 1 : (D == 2 ? P.n[0] : P.n[0] * P.n[1]);
    const int W = (ncolAll + 31) / 32 * 32;
    const bool split = D >= 2 && (int)blockDim.x == 2 * W;
    const int roleOff = split ? kGsRoleDoubles * W : 0;
    double* oldI = useSmem ? gsSmem + roleOff : work;
    double* newI = useSmem ? gsSmem + roleOff + n : work + rs;
    double* aiiI = useSmem ? work : work + 2 * rs;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) aiiI[i] = 1. / diag[i];
    __syncthreads();
    if constexpr (D == 1) {
        // a 1D wavefront is one cell: one thread sweeps
        if (threadIdx.x == 0) {
            for (long long i = 0; i < n; ++i) oldI[i] = x[i];
            for (int it = 1;; ++it) {
                bool failed = false;
                GsCoef c;
                gsLoad<D>(P, n - 1, aiiI, free, off, c);
                for (long long i = n - 1; i >= 0; --i) {
                    GsCoef cn;
                    if (i > 0) gsLoad<D>(P, i - 1, aiiI, free, off, cn);
                    const int ijk[3] = {(int)i, 0, 0};
                    const double v = gsUpdate<D>(P, i, ijk, c, oldI, newI);
                    newI[i] = v;
                    failed |= gsFails(i, v, oldI[i]);
                    c = cn;
                }
                if (!failed || it >= maxIt) break;
                double* t = oldI;
                oldI = newI;
                newI = t;
            }
            for (long long i = 0; i < n; ++i) {
                double v = newI[i];
                if (fabs(v) < 2.220446049250313e-16) v = 0;
                x[i] = v;
            }
        }
        return;
    }
    const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
    const int dmax = (nx - 1) + (ny - 1) + (D >= 3 ? nz - 1 : 0);
    const int ncol = D == 2 ? nx : nx * ny;
    const int hmax = D == 2 ? ny : nz;  // cells per column
    for (long long i = threadIdx.x; i < n; i += blockDim.x) oldI[i] = x[i];
    __syncthreads();
    if (split) {
        // slot (phase & 1): lowerS[slot][col], coefS[slot][q][col] with q = 1/diag, z+, y+, x+
        double* lowerS = gsSmem;
        double* coefS = gsSmem + 2 * W;
        const bool helper = (int)threadIdx.x >= W;
        const int col = helper ? (int)threadIdx.x - W : (int)threadIdx.x;
        const bool has = col < ncol;
        const int cx = D == 2 ? col : col % nx, cy = D == 2 ? 0 : col / nx;
        const int base = D == 2 ? cx : cx + cy;
        const long long sy = nx, sz = (long long)nx * ny;
        auto cellOf = [&](int hh) -> long long {
            return D == 2 ? cx + (long long)nx * hh : cx + (long long)nx * (cy + (long long)ny * hh);
        };
        // the helper's preparation of its column's cell at wavefront dd into slot sl, from the
        // coefficients cq already loaded
        auto prepare = [&](int dd, int sl, const GsCoef& cq) {
            const int h = dd - base;
            int ijk[3] = {cx, D == 2 ? h : cy, D == 2 ? 0 : h};
            lowerS[sl * W + col] = gsLower<D>(P, cellOf(h), ijk, cq, oldI);
            coefS[(sl * 4 + 0) * W + col] = cq.aii;
            coefS[(sl * 4 + 1) * W + col] = cq.o[5];
            coefS[(sl * 4 + 2) * W + col] = cq.o[2];
            coefS[(sl * 4 + 3) * W + col] = cq.o[1];
        };
        auto valid = [&](int dd) { return has && dd - base >= 0 && dd - base < hmax; };
        for (int it = 1;; ++it) {
            GsCoef cpre{};  // helper: the coefficients of its next cell to prepare
            if (helper) {
                if (valid(dmax)) {
                    GsCoef c0{};
                    gsLoad<D>(P, cellOf(dmax - base), aiiI, free, off, c0);
                    prepare(dmax, 0, c0);
                }
                if (valid(dmax - 1)) gsLoad<D>(P, cellOf(dmax - 1 - base), aiiI, free, off, cpre);
            }
            __syncthreads();
            for (int d = dmax; d >= 0; --d) {
                const int p = dmax - d, sl = p & 1;
                if (!helper) {
                    if (valid(d)) {
                        const int h = d - base;
                        const long long i = cellOf(h);
                        const double aii = coefS[(sl * 4 + 0) * W + col];
                        double v = lowerS[sl * W + col];
                        if (D >= 3 && h < nz - 1) v -= coefS[(sl * 4 + 1) * W + col] * newI[i + sz] * aii;
                        if (D >= 2 && (D == 2 ? h : cy) < ny - 1) v -= coefS[(sl * 4 + 2) * W + col] * newI[i + sy] * aii;
                        if (cx < nx - 1) v -= coefS[(sl * 4 + 3) * W + col] * newI[i + 1] * aii;
                        newI[i] = v;
                    }
                } else {
                    // the cell of the next wavefront from the coefficients loaded a wavefront ago,
                    // then the load for the one after (a column's first cell included)
                    if (valid(d - 1)) prepare(d - 1, sl ^ 1, cpre);
                    if (valid(d - 2)) gsLoad<D>(P, cellOf(d - 2 - base), aiiI, free, off, cpre);
                }
                __syncthreads();
            }
            bool failed = false;
            for (long long i = threadIdx.x; i < n; i += blockDim.x) failed |= gsFails(i, newI[i], oldI[i]);
            const int anyFailed = __syncthreads_or(failed);
            if (!anyFailed || it >= maxIt) break;
            double* t = oldI;
            oldI = newI;
            newI = t;
        }
        for (long long i = threadIdx.x; i < n; i += blockDim.x) {
            double v = newI[i];
            if (fabs(v) < 2.220446049250313e-16) v = 0;
            x[i] = v;
        }
        return;
    }
    const bool single = ncol <= (int)blockDim.x;
    // this thread's column (single): its x (and y) and the wavefront index of its lowest cell
    const int col = threadIdx.x;
    const int cx = D == 2 ? col : col % nx, cy = D == 2 ? 0 : col / nx;
    const int base = D == 2 ? cx : cx + cy;  // d of the column's cell at height 0
    const bool mine = single && col < ncol;
    auto cellOf = [&](int hh) -> long long {
        return D == 2 ? cx + (long long)nx * hh : cx + (long long)nx * (cy + (long long)ny * hh);
    };
    auto ijkOf = [&](int hh, int* ijk) {
        ijk[0] = cx;
        ijk[1] = D == 2 ? hh : cy;
        ijk[2] = D == 2 ? 0 : hh;
    };
    for (int it = 1;; ++it) {
        bool failed = false;
        int h = hmax - 1;  // height of this thread's next cell (y in 2D, z in 3D)
        GsCoef c{}, cn{};  // the coefficients of cells h and h - 1
        double lower = 0;  // the lower part of cell h
        if (mine) {
            int ijk[3];
            ijkOf(h, ijk);
            gsLoad<D>(P, cellOf(h), aiiI, free, off, c);
            lower = gsLower<D>(P, cellOf(h), ijk, c, oldI);
            if (h > 0) gsLoad<D>(P, cellOf(h - 1), aiiI, free, off, cn);
        }
        for (int d = dmax; d >= 0; --d) {
            if (single) {
                if (mine && h >= 0 && d == base + h) {
                    const long long i = cellOf(h);
                    int ijk[3];
                    ijkOf(h, ijk);
                    const double v = gsUpper<D>(P, i, ijk, c, lower, newI);
                    newI[i] = v;
                    // off the path to the next barrier's readers: the next cell's lower part and
                    // the loads of the one after it
                    if (h > 0) {
                        int ijn[3];
                        ijkOf(h - 1, ijn);
                        c = cn;
                        lower = gsLower<D>(P, cellOf(h - 1), ijn, c, oldI);
                        if (h > 1) gsLoad<D>(P, cellOf(h - 2), aiiI, free, off, cn);
                    }
                    --h;
                }
            } else {
                for (int q = threadIdx.x; q < ncol; q += blockDim.x) {
                    const int qx = D == 2 ? q : q % nx, qy = D == 2 ? 0 : q / nx;
                    const int hh = d - (D == 2 ? qx : qx + qy);
                    if (hh < 0 || hh >= hmax) continue;
                    const long long i = D == 2 ? qx + (long long)nx * hh : qx + (long long)nx * (qy + (long long)ny * hh);
                    GsCoef cq;
                    gsLoad<D>(P, i, aiiI, free, off, cq);
                    const int ijk[3] = {qx, D == 2 ? hh : qy, D == 2 ? 0 : hh};
                    newI[i] = gsUpdate<D>(P, i, ijk, cq, oldI, newI);
                }
            }
            __syncthreads();
        }
        for (long long i = threadIdx.x; i < n; i += blockDim.x) failed |= gsFails(i, newI[i], oldI[i]);
        const int anyFailed = __syncthreads_or(failed);
        if (!anyFailed || it >= maxIt) break;
        double* t = oldI;
        oldI = newI;
        newI = t;
    }
    // normalize, and the solution into x
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        double v = newI[i];
        if (fabs(v) < 2.220446049250313e-16) v = 0;
        x[i] = v;
    }
}


// ----------------------------------------------------------------------------- k_jacobi_solve
// JacobiSolver::algorithm (JacobiSolver.cpp:9-86) in one CTA: every row from the old iterate
// alone, (free + rowSum) / diag with rowSum the negated terms of the lower then the upper
// neighbours, each list in reverse (z-, y-, x-, then z+, y+, x+: the backward pass, whose values
// are the reference's iterate), all cells of an iteration at once; the convergence test over all
// cells after each iteration (gsFails).  Iterates in shared memory when they fit, else in work.
template <int D>
__global__ void __launch_bounds__(kGsThreads) k_jacobi_solve(const StepParams P, const double* __restrict__ diag,
                                                              const double* __restrict__ free,
                                                              const double* __restrict__ off, double* __restrict__ x,
                                                              double* __restrict__ work, int maxIt, int useSmem,
                                                              DevClock* __restrict__ ck) {
    extern __shared__ double gsSmem[];
    if (ck->done) return;
    const long long n = P.ncell, rs = P.stride;
    double* oldI = useSmem ? gsSmem : work;
    double* newI = useSmem ? gsSmem + n : work + rs;
    const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
    const long long sy = nx, sz = (long long)nx * ny;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) oldI[i] = x[i];
    __syncthreads();
    for (int it = 1;; ++it) {
        bool failed = false;
        for (long long i = threadIdx.x; i < n; i += blockDim.x) {
            const int cx = (int)(i % nx);
            const int cy = D >= 2 ? (int)((i / nx) % ny) : 0;
            const int cz = D >= 3 ? (int)(i / sz) : 0;
            const double aii = 1. / diag[i];
            double rowSum = 0;
            if (D >= 3 && cz > 0) rowSum -= off[4 * rs + i] * oldI[i - sz];
            if (D >= 2 && cy > 0) rowSum -= off[3 * rs + i] * oldI[i - sy];
            if (cx > 0) rowSum -= off[0 * rs + i] * oldI[i - 1];
            if (D >= 3 && cz < nz - 1) rowSum -= off[5 * rs + i] * oldI[i + sz];
            if (D >= 2 && cy < ny - 1) rowSum -= off[2 * rs + i] * oldI[i + sy];
            if (cx < nx - 1) rowSum -= off[1 * rs + i] * oldI[i + 1];
            const double v = (free[i] + rowSum) * aii;
            newI[i] = v;
            failed |= gsFails(i, v, oldI[i]);
        }
        const int anyFailed = __syncthreads_or(failed);
        if (!anyFailed || it >= maxIt) break;
        double* t = oldI;
        oldI = newI;
        newI = t;
    }
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        double v = newI[i];
        if (fabs(v) < 2.220446049250313e-16) v = 0;
        x[i] = v;
    }
}

// ----------------------------------------------------------------------------- k_thomas_solve
// ThomasSolver::algorithm (ThomasSolver.cpp:9-52), a 1D mesh on one thread: P_i = -u_i / (d_i +
// l_i P_{i-1}), Q_i = (f_i - l_i Q_{i-1}) / (the same denominator), x from the last row down as
// P_i x_{i+1} + Q_i, then normalize.  l_i, u_i are the x- and x+ slots of the off-diagonal.
__global__ void k_thomas_solve(const StepParams P, const double* __restrict__ diag, const double* __restrict__ free,
                               const double* __restrict__ off, double* __restrict__ x, double* __restrict__ work,
                               DevClock* __restrict__ ck) {
    if (ck->done || threadIdx.x != 0) return;
    const long long N = P.ncell, rs = P.stride;
    double* Pp = work;
    double* Qq = work + rs;
    Pp[0] = -off[1 * rs + 0] / diag[0];
    Qq[0] = free[0] / diag[0];
    for (long long i = 1; i < N - 1; ++i) {
        const double l = off[0 * rs + i];
        const double den = diag[i] + l * Pp[i - 1];
        Pp[i] = -off[1 * rs + i] / den;
        Qq[i] = (free[i] - l * Qq[i - 1]) / den;
    }
    Pp[N - 1] = 0;
    {
        const double l = off[0 * rs + N - 1];
        Qq[N - 1] = (free[N - 1] - l * Qq[N - 2]) / (diag[N - 1] + l * Pp[N - 2]);
    }
    double xn = Qq[N - 1];
    x[N - 1] = fabs(xn) < 2.220446049250313e-16 ? 0.0 : xn;
    for (long long i = N - 2; i >= 0; --i) {
        const double v = Pp[i] * xn + Qq[i];  // from the unnormalized x_{i+1}
        xn = v;
        x[i] = fabs(v) < 2.220446049250313e-16 ? 0.0 : v;
    }
}


// ----------------------------------------------------------------------------- k_cg_solve
// conjugateGradientSovler / JacobiConjugateGradientSolver / biConjugateGradientSovler::algorithm
// (conjugateGradientSolver.cpp:10-53, JacobiConjugateGradientSolver.cpp:10-83,
// biConjugateGradientSolver.cpp:10-75) in one CTA.  The matrix products take each row's terms in
// the reference's order (diag v_i, the lower entries x-, y-, z-, the upper x+, y+, z+; the
// transposed matrix's rows as SLEMatrixStorage::transpose leaves them: z-, y-, x-, then x+, y+,
// z+, each entry the transposed row's); the dot products are sums over the CTA in a fixed order,
// not the reference's serial order, so the iterates agree with it to rounding.  Stop when the
// absolute residual max |r| is below 1e-12 after the first iteration, or at the limit.
// KIND: 0 CG, 1 Jacobi-preconditioned CG, 2 BiCG.  work holds [7][stride] vectors.
__device__ __forceinline__ double blockSum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0;
    for (int w = 0; w < nw; ++w) s += red[w];  // every thread, in warp order
    return s;
}

template <int D, bool TRANSPOSED>
__device__ __forceinline__ double cgRow(const StepParams& P, long long i, const double* __restrict__ diag,
                                        const double* __restrict__ off, const double* v) {
    const long long rs = P.stride;
    const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
    const long long sy = nx, sz = (long long)nx * ny;
    const int cx = (int)(i % nx);
    const int cy = D >= 2 ? (int)((i / nx) % ny) : 0;
    const int cz = D >= 3 ? (int)(i / sz) : 0;
    double acc = diag[i] * v[i];
    if (!TRANSPOSED) {
        // row i's own entries: off slots [x-, x+, y+, y-, z-, z+] = 0, 1, 2, 3, 4, 5
        if (cx > 0) acc += off[0 * rs + i] * v[i - 1];
        if (D >= 2 && cy > 0) acc += off[3 * rs + i] * v[i - sy];
        if (D >= 3 && cz > 0) acc += off[4 * rs + i] * v[i - sz];
        if (cx < nx - 1) acc += off[1 * rs + i] * v[i + 1];
        if (D >= 2 && cy < ny - 1) acc += off[2 * rs + i] * v[i + sy];
        if (D >= 3 && cz < nz - 1) acc += off[5 * rs + i] * v[i + sz];
    } else {
        // column i: the entries of the rows that reach cell i, lower ones from the lowest row up
        if (D >= 3 && cz > 0) acc += off[5 * rs + i - sz] * v[i - sz];
        if (D >= 2 && cy > 0) acc += off[2 * rs + i - sy] * v[i - sy];
        if (cx > 0) acc += off[1 * rs + i - 1] * v[i - 1];
        if (cx < nx - 1) acc += off[0 * rs + i + 1] * v[i + 1];
        if (D >= 2 && cy < ny - 1) acc += off[3 * rs + i + sy] * v[i + sy];
        if (D >= 3 && cz < nz - 1) acc += off[4 * rs + i + sz] * v[i + sz];
    }
    return acc;
}

// the Jacobi preconditioner's product: (1 / diag) v plus a zero for each off-diagonal entry
template <int D>
__device__ __forceinline__ double cgPrecond(const StepParams& P, long long i, const double* __restrict__ diag,
                                            const double* v) {
    const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
    const long long sy = nx, sz = (long long)nx * ny;
    const int cx = (int)(i % nx);
    const int cy = D >= 2 ? (int)((i / nx) % ny) : 0;
    const int cz = D >= 3 ? (int)(i / sz) : 0;
    double acc = (1. / diag[i]) * v[i];
    if (cx > 0) acc += 0 * v[i - 1];
    if (D >= 2 && cy > 0) acc += 0 * v[i - sy];
    if (D >= 3 && cz > 0) acc += 0 * v[i - sz];
    if (cx < nx - 1) acc += 0 * v[i + 1];
    if (D >= 2 && cy < ny - 1) acc += 0 * v[i + sy];
    if (D >= 3 && cz < nz - 1) acc += 0 * v[i + sz];
    return acc;
}

template <int D, int KIND>
__global__ void __launch_bounds__(kGsThreads) k_cg_solve(const StepParams P, const double* __restrict__ diag,
                                                          const double* __restrict__ free,
                                                          const double* __restrict__ off, double* __restrict__ x,
                                                          double* __restrict__ work, int maxIt,
                                                          DevClock* __restrict__ ck) {
    __shared__ double red[32];
    if (ck->done) return;
    const long long n = P.ncell, rs = P.stride;
    double* r = work;
    double* d = work + rs;
    double* Ad = work + 2 * rs;
    double* z = work + 3 * rs;   // JCG: the preconditioned residual
    double* ro = work + 4 * rs;  // BiCG: the shadow residual and direction, A^T do
    double* dO = work + 5 * rs;
    double* ATd = work + 6 * rs;
    const int tid = threadIdx.x, bd = blockDim.x;
    for (long long i = tid; i < n; i += bd) r[i] = free[i] - cgRow<D, false>(P, i, diag, off, x);
    __syncthreads();
    for (long long i = tid; i < n; i += bd) {
        d[i] = KIND == 1 ? cgPrecond<D>(P, i, diag, r) : r[i];
        if (KIND == 2) ro[i] = dO[i] = r[i];
    }
    __syncthreads();
    for (int it = 1;; ++it) {
        double mx = -1.0;  // max |r| (a NaN passed over)
        for (long long i = tid; i < n; i += bd) mx = smax(mx, fabs(r[i]));
        mx = blockMaxReduce<double>(mx, red);
        __syncthreads();
        if (tid == 0) red[0] = mx;
        __syncthreads();
        mx = red[0];
        if ((mx < 1e-12 && it > 1) || it >= maxIt) break;
        double p1 = 0, p2 = 0;
        for (long long i = tid; i < n; i += bd) {
            const double a = cgRow<D, false>(P, i, diag, off, d);
            Ad[i] = a;
            if (KIND == 0) p1 += r[i] * r[i];
            else if (KIND == 1) p1 += r[i] * cgPrecond<D>(P, i, diag, r);
            else p1 += ro[i] * r[i];
            p2 += (KIND == 2 ? dO[i] : d[i]) * a;
        }
        const double rz = blockSum(p1, red);
        const double alpha = rz / (blockSum(p2, red) + Num<double>::stab());
        __syncthreads();
        if (KIND == 2)
            for (long long i = tid; i < n; i += bd) ATd[i] = cgRow<D, true>(P, i, diag, off, dO);
        double p3 = 0;
        for (long long i = tid; i < n; i += bd) {
            x[i] += alpha * d[i];
            const double r1 = r[i] - alpha * Ad[i];
            r[i] = r1;
            if (KIND == 2) {
                const double ro1 = ro[i] - alpha * ATd[i];
                ro[i] = ro1;
                p3 += ro1 * r1;
            } else if (KIND == 0) {
                p3 += r1 * r1;
            }
        }
        __syncthreads();
        if (KIND == 1) {
            for (long long i = tid; i < n; i += bd) {
                const double z1 = cgPrecond<D>(P, i, diag, r);
                z[i] = z1;
                p3 += r[i] * z1;
            }
        }
        const double beta = blockSum(p3, red) / (rz + Num<double>::stab());
        for (long long i = tid; i < n; i += bd) {
            d[i] = (KIND == 1 ? z[i] : r[i]) + beta * d[i];
            if (KIND == 2) dO[i] = ro[i] + beta * dO[i];
        }
        __syncthreads();
    }
    for (long long i = tid; i < n; i += bd)
        if (fabs(x[i]) < 2.220446049250313e-16) x[i] = 0;
}


// ----------------------------------------------------------------------------- k_gs_post1
// new mass fractions (clipped at 0, renormalised), concentrations, CCV and the old energy
// (Diffusion.cpp:443-478)
template <int NS, int EOS, int D>
__global__ void k_gs_post1(const StepParams P, const DiffParams X, const double* __restrict__ U,
                           DevClock* __restrict__ ck) {
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P.ncell) return;
    const long long st = P.stride;
    const double* cp = X.cellPrim;
    const double rho0 = U[NS * st + i];
    double wNew[NS], sum = 0.;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double x = X.sol[k * st + i];
        if (x < 0.) x = 0.0;
        wNew[k] = x;
        sum += x;
    }
    double c[NS + 1], cN[NS + 1];
    c[0] = 0;
    cN[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = cp[(k - 1) * st + i];
        c[0] += c[k];
        cN[k] = wNew[k - 1] / sum * rho0 / P.mix.M[k - 1];
        cN[0] += cN[k];
    }
    const double T = cp[(NS + 4) * st + i];
    const double CCVOld = c[0] * mixCv<NS, EOS>(P.mix, c);
    const double CCVNew = mixCv<NS, EOS>(P.mix, cN) * cN[0];
    const double oldEnergy = CCVOld * T + nonIdeality<NS, EOS>(P.mix, c) - nonIdeality<NS, EOS>(P.mix, cN);
#pragma unroll
    for (int k = 0; k <= NS; ++k) X.cNew[k * st + i] = cN[k];
    X.cNew[(NS + 1) * st + i] = CCVNew;
    X.cNew[(NS + 2) * st + i] = oldEnergy;
}

// ----------------------------------------------------------------------------- k_gs_afdif
// the enthalpy flow again with the new concentrations (their interpolation, molar fractions and
// Maxwell-Stefan fluxes; the patches' molar fractions still those of the phase) and its 0.5
// average with the first, then the product with the face temperature (Diffusion.cpp:618-690)
template <int NS, int EOS, int D>
__global__ void k_gs_afdif(const StepParams P, const GenericLayout L, const DiffParams X, DevClock* __restrict__ ck) {
    if (ck->done) return;
    const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (f >= L.nfaces) return;
    int a = 0;
    while (a + 1 < D && f >= L.faceBase[a + 1]) ++a;
    const long long local = f - L.faceBase[a];
    const int n = P.n[a];
    const int fi = (int)(local % (n + 1));
    if (P.periodic[a] && fi == 0) return;
    const long long tr = local / (n + 1);
    int ijk[3];
    if (a == 0) { ijk[1] = D >= 2 ? (int)(tr % P.n[1]) : 0; ijk[2] = D >= 3 ? (int)(tr / P.n[1]) : 0; }
    else if (a == 1) { ijk[0] = (int)(tr % P.n[0]); ijk[2] = D >= 3 ? (int)(tr / P.n[0]) : 0; }
    else { ijk[0] = (int)(tr % P.n[0]); ijk[1] = (int)(tr / P.n[0]); }
    const bool boundary = !P.periodic[a] && (fi == 0 || fi == n);
    ijk[a] = fi == 0 ? 0 : fi - 1;
    const int hi = (boundary && fi == 0) ? 0 : 1;
    const FaceGeo g = faceOf(P, L, ijk, a, hi);
    const long long o = cellIndex(P, ijk[0], ijk[1], ijk[2]);
    const long long st = P.stride, nf = L.nfaces;
    const double rO[3] = {P.geo.cc[0][ijk[0]], P.geo.cc[1][ijk[1]], P.geo.cc[2][ijk[2]]};
    bool bad = false;
    long long nb = -1;
    double dA = 0, m2 = 0, dnA = 0, dmag = 0, wOwn = 0, wNei = 0;
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
        const double ownR = mag3<double>(dOwn[0], dOwn[1], dOwn[2]);
        const double neiR = mag3<double>(dNei[0], dNei[1], dNei[2]);
        const double sumR = ownR + neiR;
        wOwn = neiR / sumR;
        wNei = ownR / sumR;
    } else {
        double dR[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) dR[d] = (g.rc[d] - rO[d]) * 2.;
        dmag = mag3<double>(dR[0], dR[1], dR[2]);
        dnA = dR[a] / dmag;
    }
    auto sgrad = [&](double phiO, double other) {
        if (!boundary) return ((other - phiO) / m2) * dA;
        return ((other - phiO) / dmag) * dnA;
    };
    const double* cn = X.cNew;
    double cO[NS + 1], cNb[NS + 1], sc[NS + 1];
    sc[0] = 0.0;
#pragma unroll
    for (int k = 0; k <= NS; ++k) {
        cO[k] = cn[k * st + o];
        cNb[k] = boundary ? 0.0 : cn[k * st + nb];
    }
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        sc[k] = boundary ? surfaceScalar<double, NS>(P, g.patch, k - 1, cO[k]) : cO[k] * wOwn + cNb[k] * wNei;
        sc[0] += sc[k];
    }
    const double* F = X.face;
    const double sT = F[slotTs<NS>() * nf + f];
    double flowW[NS], corr[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        flowW[k] = F[slotW<NS>(k) * nf + f];
        corr[k] = 0;
    }
    if (X.molmass && NS == 1) corr[0] = 0 - flowW[0];  // no Maxwell-Stefan flux for one species
    if (X.molmass && NS > 1) {
        // the patch's molar fractions from the phase's concentrations (calculatedMolarFraction)
        double cB[NS + 1];
        if (boundary) {
            const double* cp = X.cellPrim;
            cB[0] = 0;
#pragma unroll
            for (int k = 1; k <= NS; ++k) {
                cB[k] = cellGhostScalar<double, NS>(P, g.patch, k - 1, cp[(k - 1) * st + o], bad);
                cB[0] += cB[k];
            }
        }
        double gX[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            const double xO = cO[k + 1] / cO[0];
            double other;
            if (boundary) {
                double sum = 0;
#pragma unroll
                for (int q = 1; q <= NS; ++q) sum += cB[q];
                other = cB[k + 1] / sum;
            } else {
                other = cNb[k + 1] / cNb[0];
            }
            gX[k] = sgrad(xO, other);
        }
        // the face's binary coefficients of the first pass (they depend on T and p alone)
        double Dm[NS][NS], DF[NS];
        pointDm<NS>(X, P.mix.M, sT, X.starP[f], Dm);
        maxwellStefan<NS>(sc, P.mix.M, Dm, gX, DF);
#pragma unroll
        for (int k = 0; k < NS; ++k) corr[k] = DF[k] - flowW[k];
    }
    double af = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const double h = hkT<EOS>(P.mix, sc[k + 1], sT, k);
        af = af + (corr[k] + flowW[k]) * h / P.mix.M[k];
    }
    const double raw = F[slotEnt<NS>() * nf + f];
    const double avg = af * 0.5 + raw * (1 - 0.5);
    X.face[slotEnt<NS>() * nf + f] = X.enthImplicit ? avg : avg * sT;  // the implicit flow enters without T
    if (bad) raise(ck, FV_ERR_BOUNDARY);
}


// ----------------------------------------------------------------------------- k_gs_vtmat
// the velocity matrices (coefficient mu; the explicit deviatoric stress in their free terms) and
// the temperature matrix (coefficient kappa; the explicit enthalpy flow distributed into it, its
// time-step limit's partial minima, the viscous heating) (Diffusion.cpp:480-500, 600-709)
template <int NS, int EOS, int D>
__global__ void k_gs_vtmat(const StepParams P, const GenericLayout L, const DiffParams X, const double* __restrict__ U,
                           DevClock* __restrict__ ck) {
    __shared__ double red[32];
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double minE = 1.0 / 0.0;
    if (i < P.ncell) {
        const long long st = P.stride, nf = L.nfaces;
        const double rt = 1 / ck->dt;
        int ijk[3];
        cellAxisCoords(P, i, D, ijk);
        const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
        const double V = ex * ey * ez;
        const double rc[3] = {P.geo.cc[0][ijk[0]], P.geo.cc[1][ijk[1]], P.geo.cc[2][ijk[2]]};
        const double* cp = X.cellPrim;
        const double* F = X.face;
        const double rho0 = U[NS * st + i];
        double c[NS + 1], v[3];
        c[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            c[k] = cp[(k - 1) * st + i];
            c[0] += c[k];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = cp[(NS + d) * st + i];
        const double p = cp[(NS + 3) * st + i], T = cp[(NS + 4) * st + i];
        const double CCVNew = X.cNew[(NS + 1) * st + i], oldEnergy = X.cNew[(NS + 2) * st + i];
        double vdiag = rho0 * rt, vfree[3], tdiag = CCVNew * rt, tfree = oldEnergy * rt;
#pragma unroll
        for (int d = 0; d < 3; ++d) vfree[d] = (v[d] * rho0) * rt;
        double divDev[3] = {0, 0, 0}, divE = 0, gradV[9], divV = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) gradV[q] = 0;
        bool bad = false;
        constexpr int NFC = 2 * D;
        int fa[NFC], fh[NFC];
        faceOrder<D>(fa, fh);
#pragma unroll
        for (int s = 0; s < NFC; ++s) {
            const int a = fa[s];
            const FaceCoef fc = faceCoef<D>(P, L, ijk, a, fh[s], rc, V);
            const long long f = fc.g.f;
            const double muF = F[slotMu<NS>() * nf + f], kappaF = F[slotKappa<NS>() * nf + f];
            const double coefV = muF / fc.m * fc.dot, coefT = kappaF / fc.m * fc.dot;
            vdiag += coefV;
            tdiag += coefT;
            if (fc.nb >= 0) {
                X.vOff[s * st + i] = -muF / fc.m * fc.dot;
                X.tOff[s * st + i] = -kappaF / fc.m * fc.dot;
            } else {
                X.vOff[s * st + i] = 0;
                X.tOff[s * st + i] = 0;
                double gv[3];
                if (P.bc.vel[fc.g.patch] == FV_BC_FIXED_SURFACE) bad = true;
                ghostVelocity<double>(P.bc.vel[fc.g.patch], P.bc.vel_value[fc.g.patch], a, fc.g.sign, v, gv);
#pragma unroll
                for (int d = 0; d < 3; ++d) vfree[d] += coefV * gv[d];
                tfree += coefT * boundaryT<NS, EOS>(P, fc.g.patch, c, p, true, bad);
            }
            const double nsg = fc.g.own ? double(fc.g.sign) : double(-fc.g.sign);
            const double S = fc.g.S;
#pragma unroll
            for (int d = 0; d < 3; ++d) divDev[d] += F[slotDev<NS>(d) * nf + f] * nsg * S;
            if (X.enthalpy && !X.enthImplicit) divE += F[slotEnt<NS>() * nf + f] * nsg * S;
            double sv[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) sv[d] = X.starV[d * nf + f];
#pragma unroll
            for (int d = 0; d < 3; ++d) gradV[3 * d + a] += sv[d] * nsg * S;
            divV += sv[a] * nsg * S;
        }
        divE /= V;
        divV /= V;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            divDev[d] /= V;
            vfree[d] += divDev[d];
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) gradV[q] /= V;
        if (X.enthalpy && !X.enthImplicit) {
            const double CCVOld = c[0] * mixCv<NS, EOS>(P.mix, c);
            minE = CCVOld * T / fabs(divE + Num<double>::stab());
            const double s = divE * -1;
            if (s >= 0.) tfree += s;
            else tdiag -= s / (T + Num<double>::stab());
        }
        {
            // the viscous heating with the cell's viscosity (Diffusion.cpp:130-132,506)
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
            tfree += dd;
        }
        if (X.enthImplicit) {
            // SLEMatrix::addNabla (SLEMatrix.cpp:291-401) of the enthalpy flow, after every other
            // term (Diffusion.cpp:820-822): F & (n S / V), n outward, onto the diagonal when
            // outgoing, else onto the neighbour's entry or, on a patch, times the temperature's
            // cell-variant ghost off the free term (the flow's other components meet zeros of n)
#pragma unroll
            for (int s = 0; s < NFC; ++s) {
                const FaceGeo g = faceOf(P, L, ijk, fa[s], fh[s]);
                const double on = g.boundary ? (double(g.sign) * g.S) / V
                                             : (g.own ? (1.0 * g.S) / V : ((1.0 * g.S) / V) * -1);
                const double val = F[slotEnt<NS>() * nf + g.f] * on;
                if (val > 0) tdiag += val;
                else if (!g.boundary) X.tOff[s * st + i] += val;
                else tfree -= val * boundaryT<NS, EOS>(P, g.patch, c, p, true, bad);
            }
        }
        X.vDiag[i] = vdiag;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            X.vFree[d * st + i] = vfree[d];
            X.sol[(NS + d) * st + i] = v[d];
        }
        X.tDiag[i] = tdiag;
        X.tFree[i] = tfree;
        X.sol[(NS + 3) * st + i] = T;
        if (bad) raise(ck, FV_ERR_BOUNDARY);
    }
    const double bE = blockMinReduce(minE, red);
    if (threadIdx.x == 0) X.partMin[blockIdx.x] = bE;
}


// ----------------------------------------------------------------------------- k_gs_final
// the recomputed phase from the solved velocity and temperature (Diffusion.cpp:965-1025), its CFL
// signal and the diffusion limit's partial minima (as k_diff_cells)
template <int NS, int EOS, int D>
__global__ void k_gs_final(const StepParams P, const GenericLayout L, const DiffParams X, double* __restrict__ U,
                           DevClock* __restrict__ ck, double* __restrict__ blockMax) {
    __shared__ double red[32];
    if (ck->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double localMax = -1, minD = 1.0 / 0.0;
    if (i < P.ncell) {
        const long long st = P.stride, nf = L.nfaces;
        int ijk[3];
        cellAxisCoords(P, i, D, ijk);
        const double ex = extent(P, 0, ijk[0]), ey = extent(P, 1, ijk[1]), ez = extent(P, 2, ijk[2]);
        const double minLS = 1.0 / smin(smin(ex, ey), ez);
        const double rc[3] = {P.geo.cc[0][ijk[0]], P.geo.cc[1][ijk[1]], P.geo.cc[2][ijk[2]]};
        const double rho0 = U[NS * st + i];
        double cNew[NS + 1], vNew[3];
#pragma unroll
        for (int k = 0; k <= NS; ++k) cNew[k] = X.cNew[k * st + i];
#pragma unroll
        for (int d = 0; d < 3; ++d) vNew[d] = d < P.nmom ? X.sol[(NS + d) * st + i] : 0.0;
        const double Tn = X.sol[(NS + 3) * st + i];
        if (Tn < 0.) raise(ck, FV_ERR_NEGATIVE_T);
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
        const double sonic = sqrt(Mixture<double, NS, EOS>::sqSonic(Mixture<double, NS, EOS>::coef(P.mix, cNew), cNew,
                                                                     rho0, Uv, p));
        localMax = (mag3<double>(vNew[0], vNew[1], vNew[2]) + sonic) * minLS;
        if (X.dtDiff) {
            constexpr int NFC = 2 * D;
            int fa[NFC], fh[NFC];
            faceOrder<D>(fa, fh);
            double dist[NFC], sumDist = 0, vol = 0;
#pragma unroll
            for (int s = 0; s < NFC; ++s) {
                const FaceGeo g = faceOf(P, L, ijk, fa[s], fh[s]);
                double dr[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double fc = g.rc[d];
                    if (d == fa[s] && !g.own && !g.boundary && ijk[fa[s]] == 0) fc -= P.ext[fa[s]];
                    dr[d] = fc - rc[d];
                }
                dist[s] = mag3<double>(dr[0], dr[1], dr[2]);
                sumDist += dist[s];
            }
#pragma unroll
            for (int s = 0; s < NFC; ++s) {
                const FaceGeo g = faceOf(P, L, ijk, fa[s], fh[s]);
                vol += X.face[slotMax<NS>() * nf + g.f] * (1 - dist[s] / sumDist);
            }
            minD = vol * minLS * minLS;
        }
    }
    const double bm = blockMaxReduce<double>(localMax, red);
    __syncthreads();
    const double bD = blockMinReduce(minD, red);
    if (threadIdx.x == 0) {
        blockMax[blockIdx.x] = bm;
        X.partMin[gridDim.x + blockIdx.x] = bD;
    }
    if (i == 0) ck->stagePrim = 1;
}

}  // namespace diff
}  // namespace fv
