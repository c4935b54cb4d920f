// fv_kernels.cuh -- CUDA kernels of the explicit finite-volume step (sm_100a).
//
// Storage: the conserved state is structure-of-arrays FP64, field f of cell i at
// U[f * stride + i] with cells in the reference's order (x fastest, then y, then z).
// Fields: rho_1..rho_N, rho (mixture density, evolved with its own flux as
// Advection.cpp:433-435 does), m_x, m_y, m_z, E.  The reference carries all three momentum
// components in every dimension (a transverse component is advected passively); a case whose
// transverse velocities are all zero keeps them zero, and the kernels then touch only the first
// `nmom` = dims momentum fields.
//
// Two step paths:
//  * k_march  -- fused single-pass step for 2D/3D meshes whose limiter gives zero slopes on a
//                multi-dimensional structured mesh (limiterZeroForNonPositiveR).  Then every face
//                of a cell carries the same predicted state W (closure of Advection.cpp:237-303
//                followed by the Hancock round trip of HancockStage.cpp:174-240, whose
//                divergence cancels exactly face pair by face pair), so W is computed once per
//                cell.  A CTA owns a tile of columns (x, or x-y in 3D) plus a one-cell halo ring
//                and marches along the last axis; in-plane neighbours' W and fluxes are exchanged
//                through shared memory, the marching-axis flux stays in registers.  The epilogue
//                recovers the new primitives and reduces the CFL signal speed per CTA.
//  * generic  -- k_prim / k_faces / k_fluxes / k_update: the full MUSCL-Hancock of the reference
//                (Gauss gradient, r-ratio TVD limiter, reconstruction, Hancock predictor,
//                Riemann flux, update) with face states in global scratch.  Used in 1D and for
//                the limiters whose phi(r <= 0) is not zero.
// Both end with k_finalize, which reduces the per-CTA maxima to the next time step exactly as
// the CFL block of Schemi.cpp:807-833 and advances the device-resident clock.
#pragma once

#include "fv_device.cuh"

namespace fv {

struct Geometry {
    const double* h[3];     // cell edge along axis a (n_a entries)
    const double* cc[3];    // cell-centre coordinate along axis a
    const double* fpos[3];  // own-axis coordinate of face i (n_a + 1 entries)
    const double* aabb[3];  // transverse face-centre coordinate, corner pattern a,a,b,b
    const double* abab[3];  // transverse face-centre coordinate, corner pattern a,b,a,b
};

struct StepParams {
    int dims;
    int n[3];
    int periodic[3];
    long long ncell;
    long long stride;       // distance between fields of U
    int nmom;               // momentum components carried (dims, or 3 when a transverse velocity is non-zero)
    int tma;                // 1: stage state rows into shared memory with bulk async copies (nx even)
    int warp2d;             // 1: FP32-flux 2D steps use the warp-strip march (k_warp2d) when nmom == 2
    int hancock;            // 1: MUSCL-Hancock (SecondOrder); 0: no predictor (SecondOrderRK / ThirdOrder stages)
    int third;              // 1: ThirdOrder reconstruction (per-face limited surface gradients, k_faces3)
    int cada;               // 1: with third, the smoothness-switched limiter of ThirdOrderCada
    const double* conc;     // stored concentrations c_0..c_N (stride apart), read instead of rho_k / M_k
                            // when not null and the restart set is not in use (SecondOrderRK)
    int limiter;
    int flux;
    int gravity;
    int courant_only;
    double courant;
    double min_dt;
    double const_dt;     // > 0: constant time step (main skips its CFL block)
    double ext[3];          // parallelepiped extents (the transverse sizes of 1D / 2D cells)
    int fuseFinalize;       // 1: the step kernel's last CTA runs the CFL finalize (no k_finalize launch)
    int pad0;
    double* starV;          // not null: k_fluxes stores each face's Riemann star velocity here
                            // ([3][faces], HLLCSolver.cpp:399) for the diffusion stage
    double* starP;          // not null: and its star pressure ([faces], :400), which the transport
                            // models' face coefficients read
    const double* stagePrim;  // primitives a diffusion stage left (c_1..c_N, v, p, Uv, T; stride
                              // apart): the next step reads them when the clock's stagePrim is set
    MixParams mix;
    BCParams bc;
    Geometry geo;
};

// Device-resident clock of one case (main's Time / mesh timestep / gravity vector).
struct DevClock {
    double time;
    double dt;          // step to take next
    double dt_used;     // step taken last
    double t_end;       // clamp target (+inf for single steps)
    double dt_free;     // CFL step before the end-time clamp
    double g[3];
    double g_delta[3];
    long long steps;
    int done;           // time >= t_end: further steps are no-ops
    int err;            // fv_error_code raised by a kernel
    int first;          // 1 until the first step: primitives come from the uploaded restart set
    unsigned ticket;    // CTAs of the running step that have written their CFL partials (fused
                        // finalize); the last one resets it to 0
    int flag;           // scratch word of host-side checks (the transverse-velocity test of an upload)
    int pcValid;        // 1: the primitive cache of the buffer to read holds this state's primitives
                        // (written by the last FP64 warp-strip step; every other writer clears it)
    int stagePrim;      // 1: the state's primitives are those a diffusion stage set (P.stagePrim),
                        // not the ones its conserved variables give; cleared by the next advection
    double dtSource;    // mesh::timestepSource: the limit a diffusion stage sets for the next step;
                        // 0 stands for the reference's initial and reset value (veryBig), so that a
                        // zeroed clock holds it; main's CFL block takes it and resets it
    double dtSourceLast;  // the limit the last CFL block took (same encoding)
};

__host__ __device__ inline double sourceTimestep(const DevClock* ck) {
    return ck->dtSource > 0 ? ck->dtSource : kVeryBigD();
}

__device__ __forceinline__ void raise(DevClock* ck, int code) { atomicCAS(&ck->err, 0, code); }

// Interior columns of a march tile of `bx` threads: the warp-strip march gives each warp 30 of
// its 32 lanes (one halo lane per side), the CTA march shares one halo column per side.
constexpr int kWarpStripCols = 30;
__host__ __device__ inline bool warpStripMarch(const StepParams& P) {
    return P.warp2d != 0 && P.dims == 2 && P.nmom == 2;
}
__host__ __device__ inline int marchTileColumns(const StepParams& P, int bx) {
    return warpStripMarch(P) ? kWarpStripCols * (bx / 32) : bx - 2;
}
// CFL partial maxima per tile: the warp-strip march writes one per warp (no CTA barrier).
__host__ __device__ inline int marchPartialsPerTile(const StepParams& P, int bx) {
    return warpStripMarch(P) ? bx / 32 : 1;
}

// Index helpers
__device__ __forceinline__ long long cellIndex(const StepParams& P, int i, int j, int k) {
    return (long long)i + (long long)P.n[0] * ((long long)j + (long long)P.n[1] * k);
}

// Where a cell's conserved values are read from: its element of field slot 0 and the distance
// between slots.  Slots 0..N are the densities, N+1.. the carried momenta, `eSlot` the energy
// (global memory: N+4; a staged row in shared memory: N+1+nmom).
struct Src {
    const double* p;
    long long fs;
    int eSlot;
};

__device__ __forceinline__ Src globalSrc(const StepParams& P, const double* __restrict__ U, long long i) {
    return Src{U + i, P.stride, P.mix.ns + 4};
}

// Primitive recovery of a cell from its conserved state (Advection.cpp:455-479), or the
// uploaded restart primitives before the first step (phaseInitialization keeps them as read).
// `kc` (optional) receives the mixture coefficients of c when c is computed here from the
// densities (its c_0 then being the sum that closeFromPrimitive forms again); *haveK says so.
template <typename T, int NS, int EOS, int D>
__device__ __forceinline__ void cellPrimitive(const StepParams& P, const Src& sc, const double* __restrict__ prim,
                                              long long i, T* c, T* v, T& p, T& rho0, T* rho, T* m, T& E,
                                              typename Mixture<T, NS, EOS>::Coef* kc = nullptr,
                                              bool* haveK = nullptr) {
    if (haveK) *haveK = false;
    const long long s = P.stride;
#pragma unroll
    for (int k = 1; k <= NS; ++k) rho[k] = T(sc.p[(k - 1) * sc.fs]);
    rho0 = T(sc.p[NS * sc.fs]);
    rho[0] = rho0;
#pragma unroll
    for (int d = 0; d < 3; ++d) m[d] = d < P.nmom ? T(sc.p[(NS + 1 + d) * sc.fs]) : T(0);
    E = T(sc.p[sc.eSlot * sc.fs]);
    if (prim) {
        c[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            c[k] = T(prim[(k - 1) * s + i]);
            c[0] += c[k];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = T(prim[(NS + d) * s + i]);
        p = T(prim[(NS + 3) * s + i]);
        return;
    }
    if (P.conc) {
        // concentrations of the step's start state (averaged by the previous SecondOrderRK step)
#pragma unroll
        for (int k = 0; k <= NS; ++k) c[k] = T(P.conc[k * s + i]);
    } else {
        c[0] = 0;
#pragma unroll
        for (int k = 1; k <= NS; ++k) {
            c[k] = rho[k] / T(P.mix.M[k - 1]);
            c[0] += c[k];
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = d < P.nmom ? m[d] / rho0 : T(0);
    T v2 = 0;
    v2 += v[0] * v[0];
    v2 += v[1] * v[1];
    v2 += v[2] * v[2];
    const T Uv = E - rho0 * v2 * T(0.5) - T(0);
    const typename Mixture<T, NS, EOS>::Coef k = Mixture<T, NS, EOS>::coef(P.mix, c);
    p = Mixture<T, NS, EOS>::pFromUv(k, c, Uv);
    if (kc && !P.conc) {
        *kc = k;
        *haveK = true;
    }
}

template <typename T, int NS, int EOS, int D>
__device__ __forceinline__ void cellPrimitive(const StepParams& P, const double* __restrict__ U,
                                              const double* __restrict__ prim, long long i, T* c, T* v, T& p,
                                              T& rho0, T* rho, T* m, T& E) {
    cellPrimitive<T, NS, EOS, D>(P, globalSrc(P, U, i), prim, i, c, v, p, rho0, rho, m, E);
}

// Face state of a cell whose slopes vanish: closure, then (MUSCL-Hancock) the zero Hancock
// divergence and the recalculation from conserved values, sound speed.
// known: the mixture coefficients of c (with c_0 the sum of c_1..c_N), when the caller has them.
template <typename T, int NS, int EOS>
__device__ __forceinline__ void cellFaceState(const MixParams& mp, const T* c, const T* v, T p, FaceState<T, NS>& W,
                                              int nmom = 3, bool hancock = true,
                                              const typename Mixture<T, NS, EOS>::Coef* known = nullptr) {
#pragma unroll
    for (int k = 1; k <= NS; ++k) W.c[k] = c[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) W.v[d] = v[d];
    W.p = p;
    closeFromPrimitive<T, NS, EOS>(mp, W, known);
    if (hancock) {
        typename Mixture<T, NS, EOS>::Coef k2;
        closeFromConserved<T, NS, EOS>(mp, W, nmom, &k2);
        soundSpeed<T, NS, EOS>(k2, W);
    } else if (known) {
        soundSpeed<T, NS, EOS>(*known, W);
    } else {
        soundSpeed<T, NS, EOS>(mp, W);
    }
}

// FP32-flux predicted state: the closure / Hancock round trip is an identity up to rounding, so
// the face state is the cell state itself (densities, momenta and energy as stored, primitives
// recovered once with reciprocals).  Accuracy is bounded by the FP32 tolerance of this mode.
template <int NS, int EOS>
__device__ __forceinline__ void cellStateLean(const StepParams& P, const Src& sc, FaceState<float, NS>& W) {
#pragma unroll
    for (int k = 1; k <= NS; ++k) W.rho[k] = float(sc.p[(k - 1) * sc.fs]);
    W.rho[0] = float(sc.p[NS * sc.fs]);
#pragma unroll
    for (int d = 0; d < 3; ++d) W.m[d] = d < P.nmom ? float(sc.p[(NS + 1 + d) * sc.fs]) : 0.f;
    W.E = float(sc.p[sc.eSlot * sc.fs]);
    const float inv = 1.f / W.rho[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) W.v[d] = W.m[d] * inv;
    const float v2 = W.v[0] * W.v[0] + W.v[1] * W.v[1] + W.v[2] * W.v[2];
    W.Uv = W.E - 0.5f * W.rho[0] * v2;
    W.c[0] = 0.f;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        W.c[k] = W.rho[k] * float(P.mix.invM[k - 1]);
        W.c[0] += W.c[k];
    }
    const float ic0 = 1.f / W.c[0];
    float Cvm = 0.f, Mm = 0.f, am = 0.f, bm = 0.f;
    float X[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        X[k] = W.c[k + 1] * ic0;
        Cvm += X[k] * float(P.mix.Cv[k]);
        Mm += X[k] * float(P.mix.M[k]);
    }
    const float g1 = float(P.mix.R) / Cvm;
    if (EOS == FV_EOS_IDEAL) {
        W.p = g1 * W.Uv;
        W.cs = sqrtf(g1 * (W.Uv + W.p) * inv);
    } else {
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                am += X[k] * X[l] * float(P.mix.a[k][l]);
                bm += X[k] * X[l] * float(P.mix.b[k][l]);
            }
        const float c0 = W.c[0];
        const float acc = am * c0 * c0;
        const float m_cb = 1.f - c0 * bm;
        const float im = 1.f / m_cb;
        W.p = g1 * (W.Uv + acc) * im - acc;
        const float ac = am * c0;
        const float dpdrho = (g1 * (2.f * ac * im - bm * (W.Uv + ac * c0) * im * im) - 2.f * ac) / Mm;
        W.cs = sqrtf(dpdrho + g1 * im * (W.Uv + W.p) * inv);
    }
}

// FP32-flux CFL signal (|v| + c) / minEdge of an updated cell.
template <int NS, int EOS>
__device__ __forceinline__ float cellSignalLean(const StepParams& P, const float* rho, const float* m, float E,
                                                float minLS) {
    FaceState<float, NS> W;
    (void)W;
    const float inv = 1.f / rho[0];
    const float v0 = m[0] * inv, v1 = m[1] * inv, v2c = m[2] * inv;
    const float vv = v0 * v0 + v1 * v1 + v2c * v2c;
    const float Uv = E - 0.5f * rho[0] * vv;
    float c[NS + 1];
    c[0] = 0.f;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = rho[k] * float(P.mix.invM[k - 1]);
        c[0] += c[k];
    }
    const float ic0 = 1.f / c[0];
    float Cvm = 0.f, Mm = 0.f, am = 0.f, bm = 0.f, X[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        X[k] = c[k + 1] * ic0;
        Cvm += X[k] * float(P.mix.Cv[k]);
        Mm += X[k] * float(P.mix.M[k]);
    }
    const float g1 = float(P.mix.R) / Cvm;
    float cs2;
    if (EOS == FV_EOS_IDEAL) {
        const float p = g1 * Uv;
        cs2 = g1 * (Uv + p) * inv;
    } else {
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int l = 0; l < NS; ++l) {
                am += X[k] * X[l] * float(P.mix.a[k][l]);
                bm += X[k] * X[l] * float(P.mix.b[k][l]);
            }
        const float c0 = c[0];
        const float acc = am * c0 * c0;
        const float im = 1.f / (1.f - c0 * bm);
        const float p = g1 * (Uv + acc) * im - acc;
        const float ac = am * c0;
        const float dpdrho = (g1 * (2.f * ac * im - bm * (Uv + ac * c0) * im * im) - 2.f * ac) / Mm;
        cs2 = dpdrho + g1 * im * (Uv + p) * inv;
    }
    return (sqrtf(vv) + sqrtf(cs2)) * minLS;
}

// Compact part of W shared with in-plane neighbours for a face normal to `axis`.
template <typename T, int NS>
struct SharedW {
    T rho[NS + 1];
    T m[3];
    T E, p, cs;
    T vn[2];  // velocity along the two in-plane axes
};

template <typename T, int NS>
__device__ __forceinline__ void toShared(const FaceState<T, NS>& W, SharedW<T, NS>& s) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) s.rho[k] = W.rho[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) s.m[d] = W.m[d];
    s.E = W.E;
    s.p = W.p;
    s.cs = W.cs;
    s.vn[0] = W.v[0];
    s.vn[1] = W.v[1];
}

template <typename T, int NS>
__device__ __forceinline__ void fromShared(const SharedW<T, NS>& s, FaceState<T, NS>& W) {
#pragma unroll
    for (int k = 0; k <= NS; ++k) W.rho[k] = s.rho[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) W.m[d] = s.m[d];
    W.E = s.E;
    W.p = s.p;
    W.cs = s.cs;
    W.v[0] = s.vn[0];
    W.v[1] = s.vn[1];
    W.v[2] = T(0);
}

template <typename T> __device__ __forceinline__ T blockMaxReduce(T v, T* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    const int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nw ? red[lane] : T(-1);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// CFL signal of a cell: (|v| + c) / min edge (Schemi.cpp:807-828), from its concentrations
// c_0..c_N and conserved density, momentum and energy.
template <typename T, int NS, int EOS, int D>
__device__ __forceinline__ T cellSignalC(const StepParams& P, const T* c, T rho0, const T* m, T E, T minLS) {
    T v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = d < P.nmom ? m[d] / rho0 : T(0);
    T v2 = 0;
    v2 += v[0] * v[0];
    v2 += v[1] * v[1];
    v2 += v[2] * v[2];
    const T Uv = E - rho0 * v2 * T(0.5) - T(0);
    const typename Mixture<T, NS, EOS>::Coef k = Mixture<T, NS, EOS>::coef(P.mix, c);
    const T p = Mixture<T, NS, EOS>::pFromUv(k, c, Uv);
    const T sonic = Num<T>::sqrt_(Mixture<T, NS, EOS>::sqSonic(k, c, rho0, Uv, p));
    T s = (P.nmom == 3 ? mag3<T>(v[0], v[1], v[2]) : mag2z<T>(v[0], v[1])) + sonic;
    s *= minLS;
    return s;
}

// CFL signal of a cell from its conserved values (c_k = rho_k / M_k) that also returns the
// primitives it recovers on the way (c, v, p and the mixture coefficients of c): exactly what
// cellPrimitive computes from the same state.
template <typename T, int NS, int EOS>
__device__ __forceinline__ T cellSignalPrim(const StepParams& P, const T* rho, T rho0, const T* m, T E, T minLS,
                                            T* c, T* v, T& p, typename Mixture<T, NS, EOS>::Coef& k) {
    c[0] = 0;
#pragma unroll
    for (int q = 1; q <= NS; ++q) {
        c[q] = rho[q] / T(P.mix.M[q - 1]);
        c[0] += c[q];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = d < P.nmom ? m[d] / rho0 : T(0);
    T v2 = 0;
    v2 += v[0] * v[0];
    v2 += v[1] * v[1];
    v2 += v[2] * v[2];
    const T Uv = E - rho0 * v2 * T(0.5) - T(0);
    k = Mixture<T, NS, EOS>::coef(P.mix, c);
    p = Mixture<T, NS, EOS>::pFromUv(k, c, Uv);
    const T sonic = Num<T>::sqrt_(Mixture<T, NS, EOS>::sqSonic(k, c, rho0, Uv, p));
    T s = (P.nmom == 3 ? mag3<T>(v[0], v[1], v[2]) : mag2z<T>(v[0], v[1])) + sonic;
    s *= minLS;
    return s;
}

// The same from conserved values (c_k = rho_k / M_k).
template <typename T, int NS, int EOS, int D>
__device__ __forceinline__ T cellSignal(const StepParams& P, const T* rho, T rho0, const T* m, T E, T minLS) {
    T c[NS + 1];
    c[0] = 0;
#pragma unroll
    for (int k = 1; k <= NS; ++k) {
        c[k] = rho[k] / T(P.mix.M[k - 1]);
        c[0] += c[k];
    }
    return cellSignalC<T, NS, EOS, D>(P, c, rho0, m, E, minLS);
}

// ============================================================================ finalize
// dt = Courant / max signal; dt = min(dt, dtSource) unless Courant-only; dt = max(dt, minTime);
// time += dt_used; g += g_delta * dt_used; clamp to t_end (Schemi.cpp:802-835, 933-935).
// Executed by one CTA.
__device__ __forceinline__ void finalizeCase(const StepParams& P, DevClock* ck, const double* __restrict__ blockMax,
                                             int nblocks, int pcValidAfter = 0) {
    __shared__ double red[32];
    if (ck->done) return;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    double m = -1;
    // L2 loads: the partials may have been written by other CTAs of the same launch
    for (int b = tid; b < nblocks; b += nthr) m = smax(m, __ldcg(blockMax + b));
    m = blockMaxReduce<double>(m, red);
    if (tid != 0) return;
    const double dtUsed = ck->dt;
    double dtn = P.courant / m;
    ck->dtSourceLast = ck->dtSource;
    if (!P.courant_only) dtn = smin(dtn, sourceTimestep(ck));
    dtn = smax(dtn, P.min_dt);
    if (P.const_dt > 0) dtn = P.const_dt;  // Schemi.cpp:807: no CFL block with a constant step
    else ck->dtSource = 0;                  // Schemi.cpp:833 (veryBig)
    if (P.gravity) {
        for (int d = 0; d < 3; ++d) ck->g[d] += ck->g_delta[d] * dtUsed;
    }
    ck->time += dtUsed;
    ck->steps += 1;
    ck->first = 0;
    ck->dt_used = dtUsed;
    ck->dt_free = dtn;
    if ((ck->time + dtn) > ck->t_end) dtn = ck->t_end - ck->time;
    ck->dt = dtn;
    ck->pcValid = pcValidAfter;
    if (!(ck->time < ck->t_end) || ck->err) ck->done = 1;
}

// Fused finalize at the end of a step kernel (all threads of the CTA, after its CFL partials are
// written): each CTA takes a ticket; the CTA that takes the last of `nCtas` has every partial
// of the step visible and runs finalizeCase, then returns the ticket counter to zero for the
// next step.  Every CTA has read the clock before it takes its ticket, so the last one may
// advance it.
__device__ __forceinline__ void finalizeIfLast(const StepParams& P, DevClock* ck, const double* __restrict__ blockMax,
                                               int nPartials, unsigned nCtas, int pcValidAfter = 0) {
    __shared__ int isLast;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        isLast = atomicAdd(&ck->ticket, 1u) == nCtas - 1u;
    }
    __syncthreads();
    if (!isLast) return;
    __threadfence();
    finalizeCase(P, ck, blockMax, nPartials, pcValidAfter);
    if (threadIdx.x == 0 && threadIdx.y == 0) ck->ticket = 0u;
}

// ============================================================================ bulk async copies
// Rows of the state are staged into shared memory by the TMA unit's untiled bulk copies
// (cp.async.bulk, 16-byte aligned source, destination and size), completing on an mbarrier
// that carries the expected byte count.
__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(bar)) : "memory");
}
__device__ __forceinline__ void mbarInval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smemAddr(bar)) : "memory");
}
__device__ __forceinline__ void fenceBarrierInit() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbarArriveExpect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}
__device__ __forceinline__ void bulkCopyG2S(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smemAddr(dst)), "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for a phase with a time limit of about a second; false on timeout.
__device__ __forceinline__ bool mbarWaitBounded(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbarTryWait(bar, parity))
        if (clock64() - t0 > 2000000000LL) return false;
    return true;
}

// Ring of staged rows: stages along the marching axis, each holding NS+5 field slots of BY
// in-plane rows of BX+2 doubles (a segment starting two columns left of the tile).
template <int D> __host__ __device__ constexpr int ringStages() { return D == 3 ? 3 : 4; }
template <int NS, int D, int BX, int BY> __host__ __device__ constexpr size_t ringBytes() {
    return (size_t)ringStages<D>() * (NS + 5) * (D == 3 ? BY : 1) * (BX + 2) * sizeof(double);
}
template <typename T, int NS, int BX, int BY> __host__ __device__ constexpr size_t marchArraysBytes() {
    return ((sizeof(SharedW<T, NS>) + 2 * sizeof(FaceFlux<T, NS>)) * BX * BY + 127) / 128 * 128;
}
template <typename T, int NS, int D, int BX, int BY> __host__ __device__ constexpr size_t marchSmemBytes() {
    return marchArraysBytes<T, NS, BX, BY>() + ringBytes<NS, D, BX, BY>();
}

// ============================================================================ fused march
// Block: BX x BY threads (BY = 1 in 2D).  Thread (tx, ty) owns in-plane column
// (x0 - 1 + tx, y0 - 1 + ty); the outer ring of the block is halo.  D = 2 marches along y,
// D = 3 along z.  Rows per block along the marching axis: `rows`.  MINB: CTAs per SM the
// register budget is sized for.
template <typename T, int NS, int EOS, int D, int BX, int BY>
__device__ __forceinline__ void marchTile(const StepParams& P, const double* __restrict__ U, double* __restrict__ Un,
                                          const double* __restrict__ prim0, DevClock* __restrict__ ck,
                                          double* __restrict__ blockMaxOut, int rows, int tileX, int tileY,
                                          int tileZ) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto sW = reinterpret_cast<SharedW<T, NS>(*)[BX]>(smem_raw);
    auto sFx = reinterpret_cast<FaceFlux<T, NS>(*)[BX]>(smem_raw + sizeof(SharedW<T, NS>) * BX * BY);
    auto sFy = reinterpret_cast<FaceFlux<T, NS>(*)[BX]>(smem_raw + (sizeof(SharedW<T, NS>) + sizeof(FaceFlux<T, NS>)) * BX * BY);
    double* ring = reinterpret_cast<double*>(smem_raw + marchArraysBytes<T, NS, BX, BY>());
    constexpr int S = ringStages<D>();
    constexpr int BXL = BX + 2;
    constexpr int BYR = D == 3 ? BY : 1;
    __shared__ __align__(8) uint64_t mbar[S];
    __shared__ T red[32];
    constexpr bool LEAN = sizeof(T) == 4;  // FP32-flux arithmetic

    if (ck->done) return;  // uniform over the CTA
    const double dt = ck->dt;
    const double* __restrict__ prim = (!LEAN && ck->first) ? prim0 : nullptr;
    const double gx_ = ck->g[0], gy_ = ck->g[1], gz_ = ck->g[2];

    constexpr int MA = D - 1;  // marching axis
    const int nx = P.n[0], ny = P.n[1];
    const int nm = P.n[MA];
    const int nmom = P.nmom;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int X = tileX * (BX - 2) - 1 + tx;
    const int Y = (D == 3) ? tileY * (BY - 2) - 1 + ty : 0;
    const int z0 = tileZ * rows;
    const int z1 = min(z0 + rows, nm);
    const bool perX = P.periodic[0], perY = (D == 3) && P.periodic[1], perM = P.periodic[MA];

    // in-plane cell of this thread (wrapped for periodic axes)
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
    const bool interior = tx >= 1 && tx <= BX - 2 && X < nx && (D == 2 || (ty >= 1 && ty <= BY - 2 && Y < ny));

    // geometry of the column
    const double hxv = has ? P.geo.h[0][cx] : 1.0;
    const double hyv = D == 3 ? (has ? P.geo.h[1][cy] : 1.0) : 0.0;
    const double Lz = P.ext[2];

    auto cellAt = [&](int zm) -> long long {
        return D == 2 ? cellIndex(P, cx, zm, 0) : cellIndex(P, cx, cy, zm);
    };
    auto wrapM = [&](int zm, bool& ok) -> int {
        ok = true;
        if (zm < 0) { if (perM) return zm + nm; ok = false; return 0; }
        if (zm >= nm) { if (perM) return zm - nm; ok = false; return 0; }
        return zm;
    };

    // ---- staged rows.  Ring position q = 0 .. nq-1 holds row z0 - 1 + q of the marching axis
    // in stage q % S; its k-th use completes phase k of mbar[q % S].
    const bool tma = P.tma != 0;
    const int nfl = NS + 2 + nmom;                 // field slots staged: densities, momenta, energy
    const int x0m2 = tileX * (BX - 2) - 2;         // even: start of the staged segment
    const int segStart = max(x0m2, 0), segEnd = min(x0m2 + BXL, nx);
    const int nq = (z1 - z0) + 2;
    const int lane = (tx + ty * BX) & 31, warpId = (tx + ty * BX) >> 5;
    auto slotField = [&](int f) { return f <= NS + nmom ? f : NS + 4; };  // slot -> global field
    auto rowOf = [&](int q, int& rr) -> bool {
        bool ok2;
        rr = wrapM(z0 - 1 + q, ok2);
        return ok2;
    };
    // in-plane rows staged per plane (3D): y = y0 - 1 + j, wrapped when periodic
    auto planeRow = [&](int j, int& yy) -> bool {
        if (D == 2) { yy = 0; return true; }
        const int y = tileY * (BY - 2) - 1 + j;
        if (y >= 0 && y < ny) { yy = y; return true; }
        if (perY && y >= -1 && y <= ny) { yy = y < 0 ? y + ny : y - ny; return true; }
        return false;
    };
    auto issue = [&](int q) {  // warp 0
        const int stg = q % S;
        int rr;
        const bool rowOk = rowOf(q, rr);
        int validRows = 0;
        for (int j = 0; j < BYR; ++j) {
            int yy;
            validRows += planeRow(j, yy) ? 1 : 0;
        }
        const uint32_t bytes = rowOk ? (uint32_t)(nfl * validRows * (segEnd - segStart) * (int)sizeof(double)) : 0u;
        if (lane == 0) {
            if (bytes) mbarArriveExpect(&mbar[stg], bytes);
            else mbarArrive(&mbar[stg]);
        }
        __syncwarp();
        if (!rowOk) return;
        for (int job = lane; job < nfl * BYR; job += 32) {
            const int f = job / BYR, j = job % BYR;
            int yy;
            if (!planeRow(j, yy)) continue;
            const long long rowBase = D == 2 ? (long long)rr * nx : ((long long)rr * ny + yy) * nx;
            const double* src = U + (long long)slotField(f) * P.stride + rowBase + segStart;
            double* dst = ring + (((long long)stg * nfl + f) * BYR + j) * BXL + (segStart - x0m2);
            bulkCopyG2S(dst, src, (uint32_t)((segEnd - segStart) * sizeof(double)), &mbar[stg]);
        }
    };
    bool abortTile = false;
    int qIssued = 0;   // ring positions [0, qIssued) have been armed (same value in every thread)
    int qWaited = -1;  // highest position waited for successfully
    auto waitRow = [&](int q) {  // all threads; uniform
        int rr;
        if (!rowOf(q, rr)) return;
        const bool ok2 = mbarWaitBounded(&mbar[q % S], (uint32_t)((q / S) & 1));
        if (__syncthreads_or(!ok2)) abortTile = true;
        else qWaited = q;
    };
    // source of this thread's cell in row q: staged shared memory, or global memory for a column
    // outside the staged segment (a periodic wrap column)
    const bool fromRing = tma && has && cx == X && X >= segStart && X < segEnd;
    auto srcOf = [&](int q, long long cell) -> Src {
        if (fromRing)
            return Src{ring + ((long long)(q % S) * nfl * BYR + (D == 3 ? ty : 0)) * BXL + (X - x0m2),
                       (long long)BYR * BXL, NS + 1 + nmom};
        return globalSrc(P, U, cell);
    };
    // predicted face state of a cell and its step-start velocity (for the gravity source)
    auto stateOf = [&](const Src& sc, long long cell, FaceState<T, NS>& W, T* vp) {
        if constexpr (LEAN) {
            (void)cell;
            cellStateLean<NS, EOS>(P, sc, W);
#pragma unroll
            for (int d = 0; d < 3; ++d) vp[d] = W.v[d];
        } else {
            T c[NS + 1], v[3], p, r0, rr2[NS + 1], mm[3], EE;
            typename Mixture<T, NS, EOS>::Coef kc;
            bool haveK;
            cellPrimitive<T, NS, EOS, D>(P, sc, prim, cell, c, v, p, r0, rr2, mm, EE, &kc, &haveK);
            cellFaceState<T, NS, EOS>(P.mix, c, v, p, W, nmom, P.hancock != 0, haveK ? &kc : nullptr);
#pragma unroll
            for (int d = 0; d < 3; ++d) vp[d] = v[d];
        }
    };
    if (tma) {
        if (tx == 0 && ty == 0) {
            for (int s2 = 0; s2 < S; ++s2) mbarInit(&mbar[s2]);
            fenceBarrierInit();
        }
        __syncthreads();
        if (warpId == 0)
            for (int q = 0; q < S && q < nq; ++q) issue(q);
        qIssued = min(S, nq);
    }

    FaceState<T, NS> Wc, Wn;
    T vCur[3] = {T(0), T(0), T(0)}, vNext[3] = {T(0), T(0), T(0)};
    FaceFlux<T, NS> Gprev;
    T GprevSign = T(-1);
    T localMax = T(-1);
    bool ok;

    // ---- prologue: W(z0) and the flux of the face below z0
    if (tma) {
        waitRow(0);
        waitRow(1);
    }
    if (has && z0 < z1 && !abortTile) {
        stateOf(srcOf(1, cellAt(z0)), cellAt(z0), Wc, vCur);
        const int zb = wrapM(z0 - 1, ok);
        if (ok) {
            FaceState<T, NS> Wb;
            T vb[3];
            stateOf(srcOf(0, cellAt(zb)), cellAt(zb), Wb, vb);
            if (!riemann<T, NS>(P.flux, MA, 1, Wb, Wc, Gprev)) raise(ck, FV_ERR_RIEMANN);
            GprevSign = T(-1);
        } else {
            // boundary patch below: right (y-min) in 2D, bottom (z-min) in 3D; outward normal -e
            const int patch = D == 2 ? FV_PATCH_RIGHT : FV_PATCH_BOTTOM;
            FaceState<T, NS> Gs;
            ghostState<T, NS, EOS>(P.mix, P.bc, patch, MA, -1, Wc, Gs);
            if (!riemann<T, NS>(P.flux, MA, -1, Wc, Gs, Gprev)) raise(ck, FV_ERR_RIEMANN);
            GprevSign = T(1);
        }
    }

    for (int z = z0; z < z1 && !abortTile; ++z) {
        const int qc = z - z0 + 1;  // ring position of row z
        // W of the next row
        if (tma) {
            waitRow(qc + 1);
            if (abortTile) break;
        }
        const int zn = wrapM(z + 1, ok);
        const bool hasNext = has && ok;
        if (hasNext) stateOf(srcOf(qc + 1, cellAt(zn)), cellAt(zn), Wn, vNext);
        if (has) toShared<T, NS>(Wc, sW[ty][tx]);
        __syncthreads();
        // the stage of row z - 1 is free: refill it two rows ahead of its next reader
        if (tma && qc - 1 + S < nq) {
            if (warpId == 0) {
                fenceProxyAsync();  // generic reads of the stage before its asynchronous refill
                issue(qc - 1 + S);
            }
            qIssued = qc + S;
        }
        // in-plane fluxes through the low faces of this column
        if (has && tx >= 1) {
            FaceState<T, NS> Wl;
            if (X == 0 && !perX) {
                FaceState<T, NS> Gs;
                ghostState<T, NS, EOS>(P.mix, P.bc, FV_PATCH_TAIL, 0, -1, Wc, Gs);
                if (!riemann<T, NS>(P.flux, 0, -1, Wc, Gs, sFx[ty][tx])) raise(ck, FV_ERR_RIEMANN);
            } else {
                fromShared<T, NS>(sW[ty][tx - 1], Wl);
                if (!riemann<T, NS>(P.flux, 0, 1, Wl, Wc, sFx[ty][tx])) raise(ck, FV_ERR_RIEMANN);
            }
        }
        if (D == 3 && has && ty >= 1) {
            FaceState<T, NS> Wl;
            if (Y == 0 && !perY) {
                FaceState<T, NS> Gs;
                ghostState<T, NS, EOS>(P.mix, P.bc, FV_PATCH_RIGHT, 1, -1, Wc, Gs);
                if (!riemann<T, NS>(P.flux, 1, -1, Wc, Gs, sFy[ty][tx])) raise(ck, FV_ERR_RIEMANN);
            } else {
                fromShared<T, NS>(sW[ty - 1][tx], Wl);
                if (!riemann<T, NS>(P.flux, 1, 1, Wl, Wc, sFy[ty][tx])) raise(ck, FV_ERR_RIEMANN);
            }
        }
        // marching-axis flux through the high face of this cell
        FaceFlux<T, NS> Gnext;
        if (has) {
            if (hasNext) {
                if (!riemann<T, NS>(P.flux, MA, 1, Wc, Wn, Gnext)) raise(ck, FV_ERR_RIEMANN);
            } else {
                const int patch = D == 2 ? FV_PATCH_LEFT : FV_PATCH_TOP;
                FaceState<T, NS> Gs;
                ghostState<T, NS, EOS>(P.mix, P.bc, patch, MA, 1, Wc, Gs);
                if (!riemann<T, NS>(P.flux, MA, 1, Wc, Gs, Gnext)) raise(ck, FV_ERR_RIEMANN);
            }
        }
        __syncthreads();
        if (interior) {
            // x-high face: inner (flux of the right neighbour's low face) or the point patch
            FaceFlux<T, NS> Fxp;
            if (X == nx - 1 && !perX) {
                FaceState<T, NS> Gs;
                ghostState<T, NS, EOS>(P.mix, P.bc, FV_PATCH_POINT, 0, 1, Wc, Gs);
                if (!riemann<T, NS>(P.flux, 0, 1, Wc, Gs, Fxp)) raise(ck, FV_ERR_RIEMANN);
            } else {
                Fxp = sFx[ty][tx + 1];
            }
            const T sxm = (X == 0 && !perX) ? T(1) : T(-1);
            FaceFlux<T, NS> Fyp;
            T sym = T(-1);
            if (D == 3) {
                if (Y == ny - 1 && !perY) {
                    FaceState<T, NS> Gs;
                    ghostState<T, NS, EOS>(P.mix, P.bc, FV_PATCH_LEFT, 1, 1, Wc, Gs);
                    if (!riemann<T, NS>(P.flux, 1, 1, Wc, Gs, Fyp)) raise(ck, FV_ERR_RIEMANN);
                } else {
                    Fyp = sFy[ty + 1][tx];
                }
                sym = (Y == 0 && !perY) ? T(1) : T(-1);
            }
            const FaceFlux<T, NS>& Fxm = sFx[ty][tx];
            // face areas and volume (mesh.cpp: S = |rX0 - r00| * |r0Y - r00|, V = e1 * e2 * e3)
            const T hx = T(hxv);
            const T hm = T(P.geo.h[MA][z]);
            T Sx, Sy, Sm, V, minLS;
            if (D == 2) {
                Sx = T(Lz) * hm;          // x faces: Lz * h_y
                Sm = hx * T(Lz);          // y faces: h_x * Lz
                Sy = T(0);
                V = hx * hm * T(Lz);
                minLS = T(1) / smin(smin(hx, hm), T(Lz));
            } else {
                const T hy = T(hyv);
                Sx = hm * hy;             // x faces: h_z * h_y
                Sy = hx * hm;             // y faces: h_x * h_z
                Sm = hx * hy;             // z faces: h_x * h_y
                V = hx * hy * hm;
                minLS = T(1) / smin(smin(hx, hy), hm);
            }
            const T invV = LEAN ? T(1) / V : T(0);
            // divergence in the face order of mesh.cpp: 2D [x-, x+, y+, y-], 3D [x-, x+, y+, y-, z-, z+]
            auto div = [&](auto get) -> T {
                T s = get(Fxm) * sxm * Sx;
                s += get(Fxp) * Sx;
                if (D == 2) {
                    s += get(Gnext) * Sm;
                    s += get(Gprev) * GprevSign * Sm;
                } else {
                    s += get(Fyp) * Sy;
                    s += get(sFy[ty][tx]) * sym * Sy;
                    s += get(Gprev) * GprevSign * Sm;
                    s += get(Gnext) * Sm;
                }
                return LEAN ? s * invV : s / V;
            };
            const long long ic = cellAt(z);
            const long long st = P.stride;
            const Src so = srcOf(qc, ic);
            // FP64 accumulation of the conserved update: U_new = U - div * dt
            const double rho0Old = so.p[NS * so.fs];
            double Enew = so.p[so.eSlot * so.fs] - double(div([](const FaceFlux<T, NS>& f) { return f.E; })) * dt;
            double mNew[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (d < nmom)
                    mNew[d] = so.p[(NS + 1 + d) * so.fs] - double(div([d](const FaceFlux<T, NS>& f) { return f.m[d]; })) * dt;
            if (P.gravity) {
                // Advection.cpp:424-431 with the old density and velocity
                const T r0 = T(rho0Old);
                T vg = 0;
                vg += vCur[0] * T(gx_);
                vg += vCur[1] * T(gy_);
                vg += vCur[2] * T(gz_);
                const T gvec[3] = {T(gx_), T(gy_), T(gz_)};
                Enew += double(r0 * vg) * dt;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if (d < nmom) mNew[d] += double(gvec[d] * r0) * dt;
            }
            double rNew[NS + 1];
            rNew[0] = rho0Old - double(div([](const FaceFlux<T, NS>& f) { return f.rho[0]; })) * dt;
#pragma unroll
            for (int k = 1; k <= NS; ++k)
                rNew[k] = so.p[(k - 1) * so.fs] - double(div([k](const FaceFlux<T, NS>& f) { return f.rho[k]; })) * dt;
            // store
#pragma unroll
            for (int k = 1; k <= NS; ++k) Un[(k - 1) * st + ic] = rNew[k];
            Un[NS * st + ic] = rNew[0];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (d < nmom) Un[(NS + 1 + d) * st + ic] = mNew[d];
            Un[(NS + 4) * st + ic] = Enew;
            // CFL signal of the updated cell
            T rhoN[NS + 1], mN[3];
#pragma unroll
            for (int k = 0; k <= NS; ++k) rhoN[k] = T(rNew[k]);
#pragma unroll
            for (int d = 0; d < 3; ++d) mN[d] = T(mNew[d]);
            T s;
            if constexpr (LEAN) s = cellSignalLean<NS, EOS>(P, rhoN, mN, T(Enew), minLS);
            else s = cellSignal<T, NS, EOS, D>(P, rhoN, rhoN[0], mN, T(Enew), minLS);
            localMax = smax(localMax, s);
        }
        // roll the marching window
        if (has) {
            Gprev = Gnext;
            GprevSign = T(-1);
            if (hasNext) {
                Wc = Wn;
#pragma unroll
                for (int d = 0; d < 3; ++d) vCur[d] = vNext[d];
            }
        }
    }
    if (tma) {
        // every issued stage was waited for (or completed without copies); a timed-out wait
        // drains the remaining phases with the same time limit before the barriers are dropped
        if (abortTile) {
            if (tx == 0 && ty == 0) raise(ck, FV_ERR_SYSTEM);
            for (int q = qWaited + 1; q < qIssued; ++q) {
                int rr;
                if (rowOf(q, rr)) mbarWaitBounded(&mbar[q % S], (uint32_t)((q / S) & 1));
            }
        }
        __syncthreads();
        if (tx == 0 && ty == 0)
            for (int s2 = 0; s2 < S; ++s2) mbarInval(&mbar[s2]);
    }
    const T bm = blockMaxReduce<T>(localMax, red);
    if (threadIdx.x == 0 && threadIdx.y == 0) *blockMaxOut = double(bm);
}

// Single-case step: one CTA per tile.
template <typename T, int NS, int EOS, int D, int BX, int BY, int MINB>
__global__ void __launch_bounds__(BX* BY, MINB) k_march(const StepParams P, const double* __restrict__ U,
                                                        double* __restrict__ Un, const double* __restrict__ prim0,
                                                        DevClock* __restrict__ ck, double* __restrict__ blockMax,
                                                        int rows) {
    if (ck->done) return;  // uniform over the grid
    const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    if (D == 2)
        marchTile<T, NS, EOS, D, BX, BY>(P, U, Un, prim0, ck, blockMax + b, rows, blockIdx.x, 0, blockIdx.y);
    else
        marchTile<T, NS, EOS, D, BX, BY>(P, U, Un, prim0, ck, blockMax + b, rows, blockIdx.x, blockIdx.y, blockIdx.z);
    if (P.fuseFinalize) {
        const unsigned n = gridDim.x * gridDim.y * gridDim.z;
        finalizeIfLast(P, ck, blockMax, (int)n, n);
    }
}

// One case of a batched ensemble (device-side case table).
struct BatchCase {
    StepParams P;
    const double* U0;      // state buffer read at even step counts (relative to stepsBase)
    double* U1;            // the other buffer
    const double* prim0;
    DevClock* ck;
    double* blockMax;      // this case's CTA partials
    long long stepsBase;   // clock step count when the run started
    int tiles[3];          // tiles along x, y (3D), marching axis
    int nTiles;
    int nPartials;         // CFL partial maxima the step writes (one per CTA, or per warp)
    long long tileBase;    // first tile of this case in the ensemble's tile list
};

// Ensemble step: a persistent grid strides over the tiles of all cases; each case picks its
// read/write buffers from the parity of its own step count, so cases advance independently.
template <typename T, int NS, int EOS, int D, int BX, int BY, int MINB>
__global__ void __launch_bounds__(BX* BY, MINB) k_march_batch(const BatchCase* __restrict__ cases, int nCases,
                                                              long long totalTiles, int rows) {
    for (long long t = blockIdx.x; t < totalTiles; t += gridDim.x) {
        // case of tile t: binary search over tileBase
        int lo = 0, hi = nCases - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cases[mid].tileBase <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchCase& C = cases[lo];
        const DevClock* ck = C.ck;
        if (ck->done) continue;
        const long long local = t - C.tileBase;
        const int tx = (int)(local % C.tiles[0]);
        const long long rest = local / C.tiles[0];
        const int tyy = D == 3 ? (int)(rest % C.tiles[1]) : 0;
        const int tz = D == 3 ? (int)(rest / C.tiles[1]) : (int)rest;
        const bool odd = ((ck->steps - C.stepsBase) & 1) != 0;
        const double* Uin = odd ? C.U1 : C.U0;
        double* Uout = odd ? const_cast<double*>(C.U0) : C.U1;
        marchTile<T, NS, EOS, D, BX, BY>(C.P, Uin, Uout, C.prim0, C.ck, C.blockMax + local, rows, tx, tyy, tz);
        __syncthreads();  // shared memory is reused by the next tile
        if (C.P.fuseFinalize) finalizeIfLast(C.P, C.ck, C.blockMax, C.nPartials, (unsigned)C.nTiles);
    }
}

// CTAs per SM the register budget of k_march is sized for.
template <typename T, int BX, int BY> constexpr int marchMinBlocks() {
    return sizeof(T) == 8 ? (384 / (BX * BY) > 0 ? 384 / (BX * BY) : 1) : (512 / (BX * BY) > 0 ? 512 / (BX * BY) : 1);
}

__global__ void k_finalize(const StepParams P, DevClock* ck, const double* __restrict__ blockMax, int nblocks);

// One CTA per case of an ensemble.
__global__ void k_finalize_batch(const BatchCase* __restrict__ cases, int nCases);

}  // namespace fv
