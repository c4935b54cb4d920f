// fv_noalloc.cu -- one explicit finite-volume step that allocates nothing.
//
// Some hosts cannot call cudaMalloc on the step's path: a solver embedded in an application whose
// device memory is owned by a pooling allocator that forbids driver allocations, or a time loop
// that must not take the implicit device synchronisation a cudaMalloc / cudaFree can cause.  For
// them fv_step_noalloc runs the full MUSCL-Hancock step (the generic path of fv_generic.cuh) on
// caller-owned state buffers, and keeps every intermediate -- primitives, face states, face
// fluxes, geometry tables, CTA maxima and the clock -- in one file-scope device array of
// FV_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds until the process exits.
//
// Built with --fmad=false like the other FP64 units.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>

#include "../../include/fvstep.h"
#include "fv_launch.cuh"
#include "fv_validate.h"

using namespace fv;

namespace {

// Scratch layout for at most FV_NOALLOC_MAX_CELLS cells (any dimension, up to 4 species):
//   primitives  (N + 4) * cells
//   face states 2 * (2N + 12) * faces, faces <= 2 * dims * cells
//   face fluxes (N + 5) * faces
//   geometry    5 tables per axis, at most cells + 1 entries each
//   CTA maxima  cells / 128 + 1
// in doubles, plus the clock.
constexpr long long kMaxCells = FV_NOALLOC_MAX_CELLS;
constexpr long long kMaxFaces = 2LL * 3 * kMaxCells;
constexpr long long kPrimD = (FV_MAX_SPECIES + 4) * kMaxCells;
constexpr long long kFaceD = 2LL * (2 * FV_MAX_SPECIES + 12) * kMaxFaces;
constexpr long long kFluxD = (FV_MAX_SPECIES + 5) * kMaxFaces;
constexpr long long kGeoD = 3LL * 5 * (kMaxCells + 1);
constexpr long long kMaxD = kMaxCells / 128 + 1;
constexpr long long kDoubles = kPrimD + kFaceD + kFluxD + kGeoD + kMaxD;
constexpr size_t kClockOff = (size_t)((kDoubles * sizeof(double) + 255) / 256 * 256);
constexpr size_t kScratchBytes = kClockOff + sizeof(DevClock);
static_assert(kScratchBytes <= (size_t)FV_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the documented size");

static __device__ __align__(256) unsigned char g_fv_noalloc_scratch[FV_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array, looked up once per device.  In host code the array's name
// is only a stand-in; cudaGetSymbolAddress, called with the device current, gives the address.
constexpr int kMaxDevices = 64;
unsigned char* g_scratchAddr[kMaxDevices] = {};
std::mutex g_setupMutex;

cudaError_t scratchAddress(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchAddr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_fv_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratchAddr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratchAddr[dev];
    return cudaSuccess;
}

// Geometry tables of the mesh generator (node 0 + d*i, 8-corner cell centres, 4-corner face
// centres), written into the scratch by one thread per axis entry; same arithmetic as the
// handle-based path builds on the host.
__global__ void k_geometry(int dims, int n0, int n1, int n2, double L0, double L1, double L2, double* geo,
                           long long stride) {
    const int a = blockIdx.y;
    const int n = a == 0 ? n0 : (a == 1 ? n1 : n2);
    const double L = a == 0 ? L0 : (a == 1 ? L1 : L2);
    const bool used = a < dims;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    const double d = L / n;
    auto node = [&](int q) -> double {
        if (used) return 0.0 + d * (double)(size_t)q;
        return q == 0 ? 0.0 : L;
    };
    double* base = geo + (long long)a * 5 * stride;
    if (i < n) {
        const double A = node(i), B = node(i + 1);
        base[0 * stride + i] = fabs(B - A);
        double seq[8];
        for (int q = 0; q < 8; ++q) {
            const int bit = a == 0 ? (q & 1) : (a == 1 ? ((q >> 1) & 1) : ((q >> 2) & 1));
            seq[q] = bit ? B : A;
        }
        double s = seq[0] + seq[1];
        for (int q = 2; q < 8; ++q) s = s + seq[q];
        base[1 * stride + i] = s / 8.;
        double t = A + A;
        t = t + B;
        t = t + B;
        base[3 * stride + i] = t / 4.;
        double u = A + B;
        u = u + A;
        u = u + B;
        base[4 * stride + i] = u / 4.;
    }
    double X;
    if (i == 0) X = 0.0 + 0.;
    else if (i == n) X = 0.0 + L;
    else X = node(i);
    double s = X + X;
    s = s + X;
    s = s + X;
    base[2 * stride + i] = s / 4.;
}

__global__ void k_clock(DevClock* ck, double dt, double g0, double g1, double g2) {
    DevClock c;
    memset(&c, 0, sizeof(c));
    c.dt = dt;
    c.dt_free = dt;
    c.t_end = CUDART_INF;
    c.g[0] = g0;
    c.g[1] = g1;
    c.g[2] = g2;
    *ck = c;
}

// Step parameters of a configuration fv_create accepts (checked by fvValidateConfig first) and
// that this entry point runs: the SecondOrder step solver, one MUSCL-Hancock stage.
bool buildParams(const fv_config& c, StepParams& P, std::string& e) {
    if (!fvValidateConfig(c, e)) return false;
    if (c.order != FV_ORDER_SECOND) {
        e = "only the SecondOrder step solver (one MUSCL-Hancock stage) runs without allocation";
        return false;
    }
    memset(&P, 0, sizeof(P));
    P.hancock = 1;
    P.dims = c.dims;
    for (int a = 0; a < 3; ++a) {
        P.n[a] = a < c.dims ? c.n[a] : 1;
        P.ext[a] = c.L[a];
    }
    P.periodic[0] = c.bc_vel[FV_PATCH_TAIL] == FV_BC_PERIODIC;
    P.periodic[1] = c.dims >= 2 && c.bc_vel[FV_PATCH_RIGHT] == FV_BC_PERIODIC;
    P.periodic[2] = c.dims >= 3 && c.bc_vel[FV_PATCH_BOTTOM] == FV_BC_PERIODIC;
    P.ncell = (long long)P.n[0] * P.n[1] * P.n[2];
    P.stride = P.ncell;
    P.nmom = 3;
    P.limiter = c.limiter;
    P.flux = c.flux;
    P.gravity = c.gravity;
    P.courant_only = c.courant_only;
    P.courant = c.courant;
    P.min_dt = c.min_timestep;
    P.const_dt = c.const_timestep;
    fvMixParams(c, P.mix);
    for (int p = 0; p < 6; ++p) {
        for (int k = 0; k < FV_MAX_SPECIES; ++k) {
            P.bc.conc[p][k] = c.bc_conc[p][k];
            P.bc.conc_value[p][k] = c.bc_conc_value[p][k];
        }
        P.bc.vel[p] = c.bc_vel[p];
        for (int d = 0; d < 3; ++d) P.bc.vel_value[p][d] = c.bc_vel_value[p][d];
        P.bc.p[p] = c.bc_p[p];
        P.bc.p_value[p] = c.bc_p_value[p];
    }
    return true;
}

}  // namespace

extern "C" fv_status fv_step_noalloc(const fv_config* cfg, const double* state_in, double* state_out, double dt,
                                     double* dt_next, void* stream) {
    if (!cfg || !state_in || !state_out) return FV_ERR_INIT;
    if (cfg->chemistry != FV_CHEM_NONE) {
        fprintf(stderr, "fv_step_noalloc: the step without device allocation has no chemistry pass\n");
        return FV_ERR_INIT;
    }
    if (cfg->diffusion) {
        fprintf(stderr, "fv_step_noalloc: the step without device allocation has no diffusion stage\n");
        return FV_ERR_INIT;
    }
    StepParams P;
    std::string why;
    if (!buildParams(*cfg, P, why)) {
        fprintf(stderr, "fv_step_noalloc: invalid configuration: %s\n", why.c_str());
        return FV_ERR_INIT;
    }
    if (P.ncell > kMaxCells) {
        fprintf(stderr, "fv_step_noalloc: %lld cells exceed the maximum of %lld cells of the static scratch\n",
                P.ncell, kMaxCells);
        return FV_ERR_INIT;
    }
    {
        // the step reads every cell of state_in while it writes state_out: the two must not overlap
        const size_t bytes = (size_t)(cfg->n_species + 5) * (size_t)P.ncell * sizeof(double);
        const char* a = reinterpret_cast<const char*>(state_in);
        const char* b = reinterpret_cast<const char*>(state_out);
        if (a < b + bytes && b < a + bytes) {
            fprintf(stderr, "fv_step_noalloc: state_in and state_out overlap; pass two separate arrays\n");
            return FV_ERR_INIT;
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = nullptr;
    cudaError_t e = scratchAddress(&scratch);
    if (e != cudaSuccess) {
        fprintf(stderr, "fv_step_noalloc: scratch set-up failed: %s\n", cudaGetErrorString(e));
        return FV_ERR_SYSTEM;
    }
    // carve the scratch
    double* base = reinterpret_cast<double*>(scratch);
    const int ns = cfg->n_species;
    GenericLayout L{};
    long long fb = 0;
    for (int a = 0; a < 3; ++a) {
        L.faceBase[a] = fb;
        if (a < P.dims) {
            long long cnt = P.n[a] + 1;
            for (int b = 0; b < 3; ++b)
                if (b != a) cnt *= P.n[b];
            fb += cnt;
        }
    }
    L.nfaces = fb;
    double* Pc = base;
    double* FS = Pc + (long long)(ns + 4) * P.ncell;
    double* FL = FS + 2LL * (2 * ns + 12) * L.nfaces;
    const long long gstride = std::max(std::max(P.n[0], P.n[1]), P.n[2]) + 1;
    double* geo = FL + (long long)(ns + 5) * L.nfaces;
    double* blockMax = geo + 15 * gstride;
    DevClock* ck = reinterpret_cast<DevClock*>(scratch + kClockOff);
    for (int a = 0; a < 3; ++a) {
        double* t = geo + (long long)a * 5 * gstride;
        P.geo.h[a] = t;
        P.geo.cc[a] = t + gstride;
        P.geo.fpos[a] = t + 2 * gstride;
        P.geo.aabb[a] = t + 3 * gstride;
        P.geo.abab[a] = t + 4 * gstride;
    }
    {
        const int maxn = (int)gstride;
        dim3 grid((maxn + 127) / 128, 3);
        k_geometry<<<grid, 128, 0, st>>>(P.dims, P.n[0], P.n[1], P.n[2], P.ext[0], P.ext[1], P.ext[2], geo, gstride);
        k_clock<<<1, 1, 0, st>>>(ck, dt, cfg->g[0], cfg->g[1], cfg->g[2]);
    }
    StepBuffers B{};
    B.U = state_in;
    B.Un = state_out;
    B.prim0 = nullptr;
    B.ck = ck;
    B.blockMax = blockMax;
    B.blockMaxCap = kMaxD;
    B.Pc = Pc;
    B.FS = FS;
    B.FL = FL;
    B.L = L;
    const MarchShape none{0, 0, 0};
    e = cfg->precision == FV_PREC_F64 ? launchStepF64(P, B, PATH_GENERIC, none, st)
                                      : launchStepF32(P, B, PATH_GENERIC, none, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "fv_step_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return FV_ERR_SYSTEM;
    }
    k_finalize<<<1, 1024, 0, st>>>(P, ck, blockMax, (int)genericBlocks(P));
    if ((e = cudaGetLastError()) != cudaSuccess) return FV_ERR_SYSTEM;
    DevClock host;
    if ((e = cudaMemcpyAsync(&host, ck, sizeof(DevClock), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        fprintf(stderr, "fv_step_noalloc: %s\n", cudaGetErrorString(e));
        return FV_ERR_SYSTEM;
    }
    if (dt_next) *dt_next = host.dt_free;
    return host.err;
}
