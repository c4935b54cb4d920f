// fv_adjoint.cu -- recorded trajectories and the adjoint sweep behind fv_record / fv_replay /
// fv_adjoint (no reference counterpart: the reference has no adjoint).
//
// fv_record runs the device time loop of fv_run step by step on the handle's stream: before each
// step a one-thread kernel stores the step's dt and gravity vector (the clock's values, which the
// step kernel reads), after it the mixing-width objective of the new state is reduced per block
// and added, weighted by the step's dt, into a device accumulator in a fixed order.  Every
// `checkpoint_every` steps the state is copied into a checkpoint.  fv_adjoint walks the segments
// between checkpoints from the last one back: it recomputes the segment's states with the
// recorded dt and gravity on clocks of its own, one per step (the same step kernels, so the
// states are the recorded ones), then applies the adjoint step kernel from the segment's last
// step to its first.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "fv_adjoint_launch.cuh"
#include "fv_handle.h"

using fv::adj::StepRecord;

namespace {

constexpr int kObjThreads = 256;
constexpr int kObjBlocks = 148 * 8;

// rec = the clock's dt and gravity of the step about to run; ran = 0 when it will be a no-op.
__global__ void k_record_step(const DevClock* __restrict__ ck, StepRecord* rec) {
    StepRecord r;
    r.dt = ck->dt;
    for (int d = 0; d < 3; ++d) r.g[d] = ck->g[d];
    r.ran = ck->done ? 0 : 1;
    r.pad = 0;
    *rec = r;
}

// Clocks of the steps rec[0 .. count-1] of a recomputed segment, one per step (the recorded dt
// and gravity, no end time), so that the segment's step kernels run back to back with no clock
// or CFL kernel between them; first sets whether the segment's first step reads its primitives
// from the restart set.
__global__ void k_schedule_segment(DevClock* clocks, const StepRecord* __restrict__ rec, int count, int first) {
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
        DevClock c = {};
        c.dt = rec[j].dt;
        for (int d = 0; d < 3; ++d) c.g[d] = rec[j].g[d];
        c.t_end = INFINITY;
        c.first = j == 0 ? first : 0;
        clocks[j] = c;
    }
}

// Raises on ck the error a step of the segment raised (the first in step order).
__global__ void k_segment_errors(const DevClock* __restrict__ clocks, int count, DevClock* ck) {
    if (threadIdx.x != 0) return;
    for (int j = 0; j < count; ++j)
        if (clocks[j].err) {
            atomicCAS(&ck->err, 0, clocks[j].err);
            return;
        }
}

// Clock of a replayed or recomputed step: the recorded dt and gravity, no end time; first >= 0
// sets whether the step reads its primitives from the restart set.
__global__ void k_schedule_step(DevClock* ck, const StepRecord* __restrict__ rec, int first) {
    ck->dt = rec->dt;
    for (int d = 0; d < 3; ++d) ck->g[d] = rec->g[d];
    ck->done = 0;
    ck->t_end = INFINITY;
    if (first >= 0) ck->first = first;
}

__device__ __forceinline__ double blockSum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    v = 0;
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = l < nw ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;  // valid in thread 0
}

// Cell measure of the width integral: area in 2D, volume in 3D.
__device__ __forceinline__ double cellMeasure(const StepParams& P, long long i) {
    const int nx = P.n[0], ny = P.n[1];
    const int ix = (int)(i % nx);
    const int iy = (int)((i / nx) % ny);
    const int iz = (int)(i / ((long long)nx * ny));
    double a = P.geo.h[0][ix] * P.geo.h[1][iy];
    if (P.dims == 3) a *= P.geo.h[2][iz];
    return a;
}

__device__ __forceinline__ void moleFraction(const StepParams& P, const double* __restrict__ U, long long i, int heavy,
                                             double* c, double& c0, double& Xh) {
    c0 = 0;
    for (int k = 0; k < P.mix.ns; ++k) {
        c[k] = U[k * P.stride + i] * P.mix.invM[k];
        c0 += c[k];
    }
    Xh = c[heavy] / c0;
}

// Per-block partial sums of X_h (1 - X_h) * measure.
__global__ void k_width_partial(const StepParams P, const double* __restrict__ U, int heavy, double* partial) {
    __shared__ double red[32];
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        double c[FV_MAX_SPECIES], c0, Xh;
        moleFraction(P, U, i, heavy, c, c0, Xh);
        s += Xh * (1.0 - Xh) * cellMeasure(P, i);
    }
    s = blockSum(s, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// J += dt * scale * sum(partial) when the step ran (fixed summation order).
__global__ void k_width_accumulate(const double* __restrict__ partial, int n, double scale,
                                   const StepRecord* __restrict__ rec, double* J) {
    __shared__ double red[32];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
    s = blockSum(s, red);
    if (threadIdx.x == 0 && rec->ran) *J += rec->dt * scale * s;
}

// lam += gain * dt_{N-1} * dW/dU^N (the terminal term of the objective).
__global__ void k_width_gradient(const StepParams P, const double* __restrict__ U, double* lam, int heavy,
                                 double scale, double gain, const StepRecord* __restrict__ rec) {
    const double w = gain * rec->dt * scale;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P.ncell;
         i += (long long)gridDim.x * blockDim.x) {
        double c[FV_MAX_SPECIES], c0, Xh;
        moleFraction(P, U, i, heavy, c, c0, Xh);
        const double dWdX = w * cellMeasure(P, i) * (1.0 - 2.0 * Xh);
        for (int k = 0; k < P.mix.ns; ++k)
            lam[k * P.stride + i] += dWdX * ((k == heavy ? 1.0 : 0.0) - Xh) / c0 * P.mix.invM[k];
    }
}

}  // namespace

struct Trajectory {
    fv_record_config cfg{};
    std::vector<double*> checkpoints;
    StepRecord* rec = nullptr;
    long long recCap = 0;
    long long steps = 0;
    double* J = nullptr;
    double* partial = nullptr;
    DevClock* clock = nullptr;  // clock of recomputed steps
    DevClock* segClocks = nullptr;  // one clock per step of a recomputed segment
    long long segClockCap = 0;
    double* prim0 = nullptr;    // restart set of the recorded start state
    int first0 = 0;             // the recorded first step read the restart set
    std::vector<double*> segment;
    double* lam[2] = {nullptr, nullptr};
    bool configured = false;
    std::vector<cudaEvent_t> events;
    double scale = 0;
};

void releaseTrajectory(fv_handle* h) {
    Trajectory* t = h->traj;
    if (!t) return;
    for (double* p : t->checkpoints) cudaFree(p);
    for (double* p : t->segment) cudaFree(p);
    if (t->rec) cudaFree(t->rec);
    if (t->J) cudaFree(t->J);
    if (t->partial) cudaFree(t->partial);
    if (t->clock) cudaFree(t->clock);
    if (t->segClocks) cudaFree(t->segClocks);
    if (t->prim0) cudaFree(t->prim0);
    for (double* p : t->lam)
        if (p) cudaFree(p);
    for (cudaEvent_t e : t->events) cudaEventDestroy(e);
    delete t;
    h->traj = nullptr;
}

namespace {

fv_status fail(fv_handle* h, int code, const std::string& msg) {
    h->err = msg;
    return code;
}

#define FV_ADJ_CUDA(h, call)                                                                       \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail((h), FV_ERR_SYSTEM, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

size_t stateBytes(const fv_handle* h) { return sizeof(double) * (size_t)h->nConserved * h->P.ncell; }

fv_status readClock(fv_handle* h) {
    FV_ADJ_CUDA(h, cudaMemcpyAsync(h->ckHost, h->ck, sizeof(DevClock), cudaMemcpyDeviceToHost, h->stream));
    FV_ADJ_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

fv_status clockStatus(fv_handle* h, const DevClock& c) {
    if (!c.err) return FV_OK;
    if (c.err == FV_ERR_RIEMANN) return fail(h, c.err, "Fatal error in Riemann solver.");
    return fail(h, c.err, "device error");
}

// One forward step U -> Un on clock ck (step kernel, and the CFL finalize unless the clock is a
// recomputed step's); prim0 is the restart set a first step reads.
cudaError_t enqueueForward(fv_handle* h, const double* U, double* Un, DevClock* ck, const double* prim0,
                           bool finalize = true) {
    StepBuffers B{};
    B.U = U;
    B.Un = Un;
    B.prim0 = prim0;
    B.ck = ck;
    B.blockMax = h->blockMax;
    B.blockMaxCap = h->blockMaxCap;
    B.L = h->L;
    cudaError_t e = h->cfg.precision == FV_PREC_F64 ? launchStepF64(h->P, B, PATH_MARCH, h->shape, h->stream)
                                                     : launchStepF32(h->P, B, PATH_MARCH, h->shape, h->stream);
    if (e != cudaSuccess || !finalize) return e;
    k_finalize<<<1, 1024, 0, h->stream>>>(h->P, ck, h->blockMax, (int)marchBlocks(h->P, h->shape));
    return cudaGetLastError();
}

cudaError_t enqueueObjective(fv_handle* h, Trajectory* t, const double* U, const StepRecord* rec) {
    k_width_partial<<<kObjBlocks, kObjThreads, 0, h->stream>>>(h->P, U, t->cfg.heavy_species, t->partial);
    k_width_accumulate<<<1, 1024, 0, h->stream>>>(t->partial, kObjBlocks, t->scale, rec, t->J);
    return cudaGetLastError();
}

fv_status checkSupported(fv_handle* h) {
    if (h->path != PATH_MARCH)
        return fail(h, FV_ERR_INIT, "the adjoint differentiates the zero-slope multi-dimensional step (2D/3D, a "
                                    "limiter with zero multi-dimensional slopes); this case uses the generic path");
    if (h->cfg.eos != FV_EOS_IDEAL) return fail(h, FV_ERR_INIT, "the adjoint supports ideal-gas mixtures only");
    if (h->cfg.chemistry != FV_CHEM_NONE) return fail(h, FV_ERR_INIT, "the adjoint does not differentiate chemistry");
    if (h->cfg.diffusion) return fail(h, FV_ERR_INIT, "the adjoint does not differentiate the diffusion stage");
    if (h->cfg.order != FV_ORDER_SECOND)
        return fail(h, FV_ERR_INIT, "the adjoint differentiates the SecondOrder (MUSCL-Hancock) step");
    return FV_OK;
}

fv_status ensureTrajectory(fv_handle* h, Trajectory*& t) {
    if (!h->traj) {
        h->traj = new (std::nothrow) Trajectory();
        if (!h->traj) return fail(h, FV_ERR_SYSTEM, "out of host memory");
    }
    t = h->traj;
    if (!t->J) FV_ADJ_CUDA(h, cudaMalloc(&t->J, sizeof(double)));
    if (!t->partial) FV_ADJ_CUDA(h, cudaMalloc(&t->partial, sizeof(double) * kObjBlocks));
    if (!t->clock) {
        FV_ADJ_CUDA(h, cudaMalloc(&t->clock, sizeof(DevClock)));
        FV_ADJ_CUDA(h, cudaMemset(t->clock, 0, sizeof(DevClock)));
    }
    if (!t->prim0)
        FV_ADJ_CUDA(h, cudaMalloc(&t->prim0, sizeof(double) * (h->cfg.n_species + 4) * h->P.ncell));
    if (!t->configured) {
        adj::AdjParams A{};
        FV_ADJ_CUDA(h, h->cfg.precision == FV_PREC_F64 ? launchAdjointF64(h->cfg.n_species, h->cfg.dims, h->P, A, nullptr)
                                                        : launchAdjointF32(h->cfg.n_species, h->cfg.dims, h->P, A, nullptr));
        t->configured = true;
    }
    double area = h->cfg.L[0];
    if (h->cfg.dims == 3) area *= h->cfg.L[2];
    t->scale = 4.0 / area;
    return FV_OK;
}

fv_status ensureRecords(fv_handle* h, Trajectory* t, long long need) {
    if (need <= t->recCap) return FV_OK;
    long long cap = std::max<long long>(need, 2 * t->recCap);
    StepRecord* r = nullptr;
    FV_ADJ_CUDA(h, cudaMalloc(&r, sizeof(StepRecord) * cap));
    if (t->rec) {
        FV_ADJ_CUDA(h, cudaMemcpyAsync(r, t->rec, sizeof(StepRecord) * t->recCap, cudaMemcpyDeviceToDevice, h->stream));
        FV_ADJ_CUDA(h, cudaStreamSynchronize(h->stream));
        cudaFree(t->rec);
    }
    t->rec = r;
    t->recCap = cap;
    return FV_OK;
}

fv_status ensureEvents(fv_handle* h, Trajectory* t, size_t n) {
    while (t->events.size() < n) {
        cudaEvent_t e;
        FV_ADJ_CUDA(h, cudaEventCreate(&e));
        t->events.push_back(e);
    }
    return FV_OK;
}

}  // namespace

extern "C" {

fv_status fv_record(fv_handle* h, const fv_record_config* rc, double t_end, long long max_steps,
                    fv_record_stats* stats) {
    if (!h || !rc) return FV_ERR_INIT;
    if (rc->checkpoint_every < 1) return fail(h, FV_ERR_INIT, "checkpoint_every must be >= 1");
    if (rc->objective != FV_OBJ_NONE && rc->objective != FV_OBJ_MIXING_WIDTH)
        return fail(h, FV_ERR_INIT, "unknown objective");
    if (rc->objective == FV_OBJ_MIXING_WIDTH && (rc->heavy_species < 0 || rc->heavy_species >= h->cfg.n_species))
        return fail(h, FV_ERR_INIT, "heavy_species out of range");
    fv_status st = checkSupported(h);
    if (st != FV_OK) return st;
    Trajectory* t = nullptr;
    if ((st = ensureTrajectory(h, t)) != FV_OK) return st;
    t->cfg = *rc;
    t->steps = 0;
    if ((st = readClock(h)) != FV_OK) return st;
    DevClock& c = *h->ckHost;
    // fv_run's loop start: the first step is min(free CFL step, t_end - time)
    c.t_end = t_end;
    c.done = !(c.time < t_end);
    c.dt = std::min(c.dt_free, t_end - c.time);
    FV_ADJ_CUDA(h, cudaMemcpyAsync(h->ck, h->ckHost, sizeof(DevClock), cudaMemcpyHostToDevice, h->stream));
    FV_ADJ_CUDA(h, cudaMemsetAsync(t->J, 0, sizeof(double), h->stream));
    // the restart set a first step reads, kept so that recomputation repeats that step exactly
    t->first0 = c.first;
    if (c.first)
        FV_ADJ_CUDA(h, cudaMemcpyAsync(t->prim0, h->prim0, sizeof(double) * (h->cfg.n_species + 4) * h->P.ncell,
                                       cudaMemcpyDeviceToDevice, h->stream));
    FV_ADJ_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    const int C = rc->checkpoint_every;
    long long n = 0, nck = 0;
    while (!c.done && n < max_steps) {
        const long long k = n / C;
        if ((long long)t->checkpoints.size() <= k) {
            double* p = nullptr;
            FV_ADJ_CUDA(h, cudaMalloc(&p, stateBytes(h)));
            t->checkpoints.push_back(p);
        }
        FV_ADJ_CUDA(h, cudaMemcpyAsync(t->checkpoints[k], h->U[h->cur], stateBytes(h), cudaMemcpyDeviceToDevice,
                                       h->stream));
        nck = k + 1;
        const long long len = std::min<long long>(C, max_steps - n);
        if ((st = ensureRecords(h, t, n + len)) != FV_OK) return st;
        int from = h->cur;
        for (long long j = 0; j < len; ++j) {
            StepRecord* r = t->rec + n + j;
            k_record_step<<<1, 1, 0, h->stream>>>(h->ck, r);
            FV_ADJ_CUDA(h, enqueueForward(h, h->U[from], h->U[from ^ 1], h->ck, h->prim0));
            if (rc->objective == FV_OBJ_MIXING_WIDTH) FV_ADJ_CUDA(h, enqueueObjective(h, t, h->U[from ^ 1], r));
            from ^= 1;
        }
        const long long before = c.steps;
        if ((st = readClock(h)) != FV_OK) return st;
        const long long executed = c.steps - before;
        if (executed & 1) h->cur ^= 1;
        n += executed;
        if (c.err || executed < len) break;
    }
    FV_ADJ_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    FV_ADJ_CUDA(h, cudaEventSynchronize(h->ev1));
    t->steps = n;
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    double J = 0;
    FV_ADJ_CUDA(h, cudaMemcpy(&J, t->J, sizeof(double), cudaMemcpyDeviceToHost));
    if (stats) {
        stats->objective = J;
        stats->time = c.time;
        stats->steps = n;
        stats->checkpoints = nck;
        stats->device_ms = ms;
    }
    return clockStatus(h, c);
}

fv_status fv_replay(fv_handle* h, fv_record_stats* stats) {
    if (!h) return FV_ERR_INIT;
    Trajectory* t = h->traj;
    if (!t || t->steps < 1) return fail(h, FV_ERR_INIT, "no recorded trajectory (call fv_record first)");
    FV_ADJ_CUDA(h, cudaStreamSynchronize(h->stream));
    FV_ADJ_CUDA(h, cudaMemsetAsync(t->J, 0, sizeof(double), h->stream));
    FV_ADJ_CUDA(h, cudaMemsetAsync(&h->ck->err, 0, sizeof(int), h->stream));
    FV_ADJ_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    for (long long n = 0; n < t->steps; ++n) {
        const StepRecord* r = t->rec + n;
        k_schedule_step<<<1, 1, 0, h->stream>>>(h->ck, r, -1);
        FV_ADJ_CUDA(h, enqueueForward(h, h->U[h->cur], h->U[h->cur ^ 1], h->ck, h->prim0));
        if (t->cfg.objective == FV_OBJ_MIXING_WIDTH) FV_ADJ_CUDA(h, enqueueObjective(h, t, h->U[h->cur ^ 1], r));
        h->cur ^= 1;
    }
    FV_ADJ_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    fv_status st = readClock(h);
    if (st != FV_OK) return st;
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    double J = 0;
    FV_ADJ_CUDA(h, cudaMemcpy(&J, t->J, sizeof(double), cudaMemcpyDeviceToHost));
    const DevClock& c = *h->ckHost;
    if (stats) {
        stats->objective = J;
        stats->time = c.time;
        stats->steps = t->steps;
        stats->checkpoints = 0;
        stats->device_ms = ms;
    }
    return clockStatus(h, c);
}

fv_status fv_adjoint(fv_handle* h, const double* dJ_dU_T, double dJ_dJ, double* dJ_dU_0, fv_adjoint_stats* stats) {
    if (!h || !dJ_dU_0) return FV_ERR_INIT;
    Trajectory* t = h->traj;
    if (!t || t->steps < 1) return fail(h, FV_ERR_INIT, "no recorded trajectory (call fv_record first)");
    const long long N = t->steps;
    const int C = t->cfg.checkpoint_every;
    const long long K = (N + C - 1) / C;
    const bool objective = t->cfg.objective == FV_OBJ_MIXING_WIDTH && dJ_dJ != 0.0;
    const size_t bytes = stateBytes(h);
    const long long segStates = std::min<long long>(C, N) + 1;
    while ((long long)t->segment.size() < segStates) {
        double* p = nullptr;
        FV_ADJ_CUDA(h, cudaMalloc(&p, bytes));
        t->segment.push_back(p);
    }
    for (double*& p : t->lam)
        if (!p) FV_ADJ_CUDA(h, cudaMalloc(&p, bytes));
    if (t->segClockCap < segStates) {
        if (t->segClocks) FV_ADJ_CUDA(h, cudaFree(t->segClocks));
        t->segClocks = nullptr;
        t->segClockCap = 0;
        FV_ADJ_CUDA(h, cudaMalloc(&t->segClocks, sizeof(DevClock) * segStates));
        t->segClockCap = segStates;
    }
    fv_status st = ensureEvents(h, t, 2 * (size_t)K + 2);
    if (st != FV_OK) return st;
    FV_ADJ_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaEvent_t* ev = t->events.data();
    FV_ADJ_CUDA(h, cudaEventRecord(ev[0], h->stream));
    int cur = 0;
    // both buffers start as the terminal adjoint: a momentum component the case does not carry is
    // left alone by the adjoint steps (its adjoint passes through unchanged)
    for (double* l : t->lam) {
        if (dJ_dU_T) FV_ADJ_CUDA(h, cudaMemcpyAsync(l, dJ_dU_T, bytes, cudaMemcpyDeviceToDevice, h->stream));
        else FV_ADJ_CUDA(h, cudaMemsetAsync(l, 0, bytes, h->stream));
    }
    FV_ADJ_CUDA(h, cudaMemsetAsync(&t->clock->err, 0, sizeof(int), h->stream));
    long long recomputed = 0;
    for (long long k = K - 1; k >= 0; --k) {
        const long long s0 = k * C;
        const long long len = std::min<long long>(C, N - s0);
        // recompute U^{s0 + 1} .. U^{s0 + len - 1} (and U^N for the terminal objective term)
        const long long upto = (k == K - 1 && objective) ? len : len - 1;
        FV_ADJ_CUDA(h, cudaEventRecord(ev[1 + 2 * (K - 1 - k)], h->stream));
        FV_ADJ_CUDA(h, cudaMemcpyAsync(t->segment[0], t->checkpoints[k], bytes, cudaMemcpyDeviceToDevice, h->stream));
        if (upto > 0) {
            k_schedule_segment<<<1, 64, 0, h->stream>>>(t->segClocks, t->rec + s0, (int)upto,
                                                         s0 == 0 ? t->first0 : 0);
            for (long long j = 0; j < upto; ++j)
                FV_ADJ_CUDA(h, enqueueForward(h, t->segment[j], t->segment[j + 1], t->segClocks + j, t->prim0,
                                              false));
            k_segment_errors<<<1, 32, 0, h->stream>>>(t->segClocks, (int)upto, t->clock);
        }
        recomputed += upto;
        FV_ADJ_CUDA(h, cudaEventRecord(ev[2 + 2 * (K - 1 - k)], h->stream));
        if (k == K - 1 && objective) {
            k_width_gradient<<<kObjBlocks, kObjThreads, 0, h->stream>>>(h->P, t->segment[len], t->lam[cur],
                                                                        t->cfg.heavy_species, t->scale, dJ_dJ,
                                                                        t->rec + N - 1);
            FV_ADJ_CUDA(h, cudaGetLastError());
        }
        for (long long j = len - 1; j >= 0; --j) {
            const long long n = s0 + j;
            adj::AdjParams A{};
            A.U = t->segment[j];
            A.lamIn = t->lam[cur];
            A.lamOut = t->lam[cur ^ 1];
            A.rec = t->rec;
            A.n = n;
            A.objGain = objective ? dJ_dJ : 0.0;
            A.objScale = t->scale;
            A.heavy = t->cfg.heavy_species;
            A.rows = 0;  // tile height chosen by the launcher (whole waves of resident CTAs)
            FV_ADJ_CUDA(h, h->cfg.precision == FV_PREC_F64
                               ? launchAdjointF64(h->cfg.n_species, h->cfg.dims, h->P, A, h->stream)
                               : launchAdjointF32(h->cfg.n_species, h->cfg.dims, h->P, A, h->stream));
            cur ^= 1;
        }
    }
    FV_ADJ_CUDA(h, cudaMemcpyAsync(dJ_dU_0, t->lam[cur], bytes, cudaMemcpyDeviceToDevice, h->stream));
    FV_ADJ_CUDA(h, cudaEventRecord(ev[2 * K + 1], h->stream));
    FV_ADJ_CUDA(h, cudaEventSynchronize(ev[2 * K + 1]));
    DevClock c;
    FV_ADJ_CUDA(h, cudaMemcpy(&c, t->clock, sizeof(DevClock), cudaMemcpyDeviceToHost));
    float total = 0, rec = 0;
    cudaEventElapsedTime(&total, ev[0], ev[2 * K + 1]);
    for (long long i = 0; i < K; ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[1 + 2 * i], ev[2 + 2 * i]);
        rec += ms;
    }
    if (stats) {
        stats->steps = N;
        stats->recomputed = recomputed;
        stats->device_ms = total;
        stats->recompute_ms = rec;
    }
    return clockStatus(h, c);
}

fv_status fv_state_copy(fv_handle* h, double* dst) {
    if (!h || !dst) return FV_ERR_INIT;
    FV_ADJ_CUDA(h, cudaMemcpyAsync(dst, h->U[h->cur], stateBytes(h), cudaMemcpyDeviceToDevice, h->stream));
    FV_ADJ_CUDA(h, cudaStreamSynchronize(h->stream));
    return FV_OK;
}

}  // extern "C"
