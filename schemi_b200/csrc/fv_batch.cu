// fv_batch.cu -- batched ensemble of independent cases (no reference counterpart: the reference
// runs one case per process).
//
// All cases share dims, species count, EOS, flux, limiter and precision, and use the fused march.
// One ensemble step = the ensemble kernel (k_warp2d_batch, one CTA per tile, or k_march_batch, a
// persistent grid striding over the tiles of every case) + k_finalize_batch (one CTA per case: its
// own CFL step, clock and end-time clamp).  Each case
// reads and writes the buffer pair selected by the parity of its own step count, so a case that
// reached its end time simply stops while the others go on.  Ensemble steps are captured in a
// CUDA graph of `chunk` steps; the host polls the number of active cases once per chunk.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "fv_handle.h"

namespace {

__global__ void k_count_active(const BatchCase* __restrict__ cases, int n, int* active) {
    int a = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a += cases[i].ck->done ? 0 : 1;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    __shared__ int red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) s += red[w];
        *active = s;
    }
}

}  // namespace

struct fv_batch {
    std::vector<fv_handle*> cases;
    std::vector<BatchCase> host;
    BatchCase* dev = nullptr;
    int* activeDev = nullptr;
    int* activeHost = nullptr;
    long long totalTiles = 0;
    MarchShape shape{128, 1, 16};
    int grid = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int chunk = 16;
    int ns = 0, eos = 0, dims = 0, precision = 0;
};

namespace {

// Tiles of every case for the ensemble kernel: the warp-strip march when every case runs it
// (FP32-flux 2D cases without a transverse velocity), else the CTA march.  Each case's P is the
// handle's with the kernel choice written into it, so tile counts and kernels agree.
void layoutTiles(fv_batch* b) {
    bool warp = true, ring = true;
    for (fv_handle* h : b->cases) {
        // the ensemble kernel has the warp-strip layout in FP32-flux arithmetic only
        warp = warp && warpStripMarch(h->P) && h->cfg.precision == FV_PREC_F32_FLUX;
        ring = ring && h->P.tma != 0;
    }
    b->shape.warp = warp ? (ring ? 2 : 1) : 0;
    long long base = 0;
    for (size_t i = 0; i < b->cases.size(); ++i) {
        BatchCase& bc = b->host[i];
        bc.P = b->cases[i]->P;
        bc.P.warp2d = warp ? 1 : 0;
        // the finalize stays a launch of its own: a ticket per tile (the fused finalize) costs
        // each of the ensemble's tens of thousands of CTAs an atomic round trip at its end
        bc.P.fuseFinalize = 0;
        const StepParams& P = bc.P;
        const int cols = marchTileColumns(P, b->shape.bx);
        bc.tiles[0] = (P.n[0] + cols - 1) / cols;
        if (P.dims == 2) {
            bc.tiles[1] = 1;
            bc.tiles[2] = (P.n[1] + b->shape.rows - 1) / b->shape.rows;
        } else {
            bc.tiles[1] = (P.n[1] + b->shape.by - 3) / (b->shape.by - 2);
            bc.tiles[2] = (P.n[2] + b->shape.rows - 1) / b->shape.rows;
        }
        bc.nTiles = bc.tiles[0] * bc.tiles[1] * bc.tiles[2];
        bc.nPartials = bc.nTiles * marchPartialsPerTile(P, b->shape.bx);
        bc.tileBase = base;
        base += bc.nTiles;
    }
    b->totalTiles = base;
}

cudaError_t configureGrid(fv_batch* b) {
    int grid = 0;
    const int n = (int)b->cases.size();
    cudaError_t e = b->precision == FV_PREC_F64
                        ? launchBatchF64(b->ns, b->eos, b->dims, nullptr, n, 0, b->shape, &grid, nullptr)
                        : launchBatchF32(b->ns, b->eos, b->dims, nullptr, n, 0, b->shape, &grid, nullptr);
    if (e == cudaSuccess) b->grid = grid;
    return e;
}

cudaError_t enqueueEnsembleStep(fv_batch* b) {
    int grid = b->grid;
    cudaError_t e = b->precision == FV_PREC_F64
                        ? launchBatchF64(b->ns, b->eos, b->dims, b->dev, (int)b->cases.size(), b->totalTiles,
                                         b->shape, &grid, b->stream)
                        : launchBatchF32(b->ns, b->eos, b->dims, b->dev, (int)b->cases.size(), b->totalTiles,
                                         b->shape, &grid, b->stream);
    if (e != cudaSuccess) return e;
    k_finalize_batch<<<(unsigned)b->cases.size(), 256, 0, b->stream>>>(b->dev, (int)b->cases.size());
    return cudaGetLastError();
}

}  // namespace

extern "C" {

fv_status fv_batch_create(fv_handle* const* handles, int n_cases, fv_batch** out) {
    if (!handles || n_cases < 1 || !out) return FV_ERR_INIT;
    *out = nullptr;
    const fv_config& c0 = handles[0]->cfg;
    for (int i = 0; i < n_cases; ++i) {
        const fv_config& c = handles[i]->cfg;
        if (c.dims != c0.dims || c.n_species != c0.n_species || c.eos != c0.eos || c.flux != c0.flux ||
            c.limiter != c0.limiter || c.precision != c0.precision) {
            fprintf(stderr, "fv_batch_create: case %d differs from case 0 in dims/species/EOS/flux/limiter/precision\n",
                    i);
            return FV_ERR_INIT;
        }
        if (c.chemistry != FV_CHEM_NONE) {
            fprintf(stderr, "fv_batch_create: case %d has chemistry (the ensemble kernel advances the flow only)\n", i);
            return FV_ERR_INIT;
        }
        if (c.diffusion) {
            fprintf(stderr, "fv_batch_create: case %d has diffusion (the ensemble kernel advances the flow only)\n", i);
            return FV_ERR_INIT;
        }
        if (c.order != FV_ORDER_SECOND) {
            fprintf(stderr, "fv_batch_create: case %d uses SecondOrderRK (the ensemble kernel runs SecondOrder)\n", i);
            return FV_ERR_INIT;
        }
        if (handles[i]->path != PATH_MARCH) {
            fprintf(stderr, "fv_batch_create: case %d does not use the fused march (1D, or a limiter with non-zero "
                            "multi-dimensional slopes)\n", i);
            return FV_ERR_INIT;
        }
    }
    fv_batch* b = new (std::nothrow) fv_batch();
    if (!b) return FV_ERR_SYSTEM;
    b->cases.assign(handles, handles + n_cases);
    b->ns = c0.n_species;
    b->eos = c0.eos;
    b->dims = c0.dims;
    b->precision = c0.precision;
    b->shape = handles[0]->shape;
    b->stream = handles[0]->stream;
    auto bail = [&](const char* what, cudaError_t e) {
        fprintf(stderr, "fv_batch_create: %s: %s\n", what, cudaGetErrorString(e));
        fv_batch_destroy(b);
        return FV_ERR_SYSTEM;
    };
    // every case uses the ensemble's tile shape
    for (fv_handle* h : b->cases) {
        if (h->shape.bx != b->shape.bx || h->shape.by != b->shape.by || h->shape.rows != b->shape.rows) {
            const fv_status st = fv_set_march_shape(h, b->shape.bx, b->shape.by, b->shape.rows);
            if (st != FV_OK) {
                fv_batch_destroy(b);
                return st;
            }
        }
    }
    for (fv_handle* h : b->cases) {
        BatchCase bc;
        memset(&bc, 0, sizeof(bc));
        bc.ck = h->ck;
        bc.prim0 = h->prim0;
        bc.blockMax = h->blockMax;
        b->host.push_back(bc);
    }
    layoutTiles(b);
    cudaError_t e;
    if ((e = cudaMalloc(&b->dev, sizeof(BatchCase) * n_cases)) != cudaSuccess) return bail("case table", e);
    if ((e = cudaMalloc(&b->activeDev, sizeof(int))) != cudaSuccess) return bail("counter", e);
    if ((e = cudaMallocHost(&b->activeHost, sizeof(int))) != cudaSuccess) return bail("counter mirror", e);
    if ((e = cudaEventCreate(&b->ev0)) != cudaSuccess) return bail("event", e);
    if ((e = cudaEventCreate(&b->ev1)) != cudaSuccess) return bail("event", e);
    if ((e = configureGrid(b)) != cudaSuccess) return bail("kernel configuration", e);
    *out = b;
    return FV_OK;
}

void fv_batch_destroy(fv_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->dev) cudaFree(b->dev);
    if (b->activeDev) cudaFree(b->activeDev);
    if (b->activeHost) cudaFreeHost(b->activeHost);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    delete b;
}

fv_status fv_batch_run(fv_batch* b, const double* t_end, long long max_steps, fv_batch_stats* stats) {
    if (!b || !t_end) return FV_ERR_INIT;
    const int n = (int)b->cases.size();
    // per-case clocks: end time, first step clamp (Schemi.cpp:664-670), buffer pair and step base
    for (int i = 0; i < n; ++i)
        if (cudaStreamSynchronize(b->cases[i]->stream) != cudaSuccess) return FV_ERR_SYSTEM;
    // an upload may have changed a case's carried momentum count, and with it the kernel choice
    const int warpBefore = b->shape.warp;
    const long long tilesBefore = b->totalTiles;
    layoutTiles(b);
    if (b->shape.warp != warpBefore || b->totalTiles != tilesBefore) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        if (configureGrid(b) != cudaSuccess) return FV_ERR_SYSTEM;
    }
    for (int i = 0; i < n; ++i) {
        fv_handle* h = b->cases[i];
        DevClock c;
        cudaError_t e = cudaMemcpy(&c, h->ck, sizeof(DevClock), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return FV_ERR_SYSTEM;
        c.t_end = t_end[i];
        c.done = !(c.time < t_end[i]) || c.err;
        c.dt = (c.time + c.dt_free) > t_end[i] ? t_end[i] - c.time : c.dt_free;
        if ((e = cudaMemcpy(h->ck, &c, sizeof(DevClock), cudaMemcpyHostToDevice)) != cudaSuccess) return FV_ERR_SYSTEM;
        BatchCase& bc = b->host[i];
        bc.U0 = h->U[h->cur];
        bc.U1 = h->U[h->cur ^ 1];
        bc.stepsBase = c.steps;
    }
    if (cudaMemcpyAsync(b->dev, b->host.data(), sizeof(BatchCase) * n, cudaMemcpyHostToDevice, b->stream) !=
        cudaSuccess)
        return FV_ERR_SYSTEM;
    if (!b->graph) {
        cudaGraph_t g;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FV_ERR_SYSTEM;
        for (int s = 0; s < b->chunk; ++s) {
            if (enqueueEnsembleStep(b) != cudaSuccess) {
                cudaStreamEndCapture(b->stream, &g);
                return FV_ERR_SYSTEM;
            }
        }
        if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess) return FV_ERR_SYSTEM;
        if (cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) return FV_ERR_SYSTEM;
        cudaGraphDestroy(g);
    }
    cudaEventRecord(b->ev0, b->stream);
    long long steps = 0, launches = 0;
    int active = n;
    while (active > 0 && steps < max_steps) {
        const long long left = max_steps - steps;
        if (left >= b->chunk) {
            if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return FV_ERR_SYSTEM;
            steps += b->chunk;
            launches += 2LL * b->chunk;
        } else {
            for (long long s = 0; s < left; ++s)
                if (enqueueEnsembleStep(b) != cudaSuccess) return FV_ERR_SYSTEM;
            steps += left;
            launches += 2 * left;
        }
        k_count_active<<<1, 512, 0, b->stream>>>(b->dev, n, b->activeDev);
        cudaMemcpyAsync(b->activeHost, b->activeDev, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) return FV_ERR_SYSTEM;
        active = *b->activeHost;
    }
    cudaEventRecord(b->ev1, b->stream);
    cudaEventSynchronize(b->ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    // hand the buffers back to the handles
    long long cellUpdates = 0, stepsMax = 0;
    int err = 0;
    for (int i = 0; i < n; ++i) {
        fv_handle* h = b->cases[i];
        DevClock c;
        if (cudaMemcpy(&c, h->ck, sizeof(DevClock), cudaMemcpyDeviceToHost) != cudaSuccess) return FV_ERR_SYSTEM;
        const long long executed = c.steps - b->host[i].stepsBase;
        if (executed & 1) h->cur ^= 1;
        cellUpdates += executed * h->P.ncell;
        stepsMax = std::max(stepsMax, executed);
        if (c.err && !err) err = c.err;
        *h->ckHost = c;
    }
    if (stats) {
        stats->cell_updates = cellUpdates;
        stats->steps_max = stepsMax;
        stats->launches = launches;
        stats->device_ms = ms;
    }
    return err;
}

}  // extern "C"
