// fv_abi_oracle.cpp -- TEST INFRASTRUCTURE, not part of the product.
//
// The subset of the C-ABI of include/fvstep.h that the task-deck driver (schemi_b200/host/
// fvrun.cpp) and the reference-side step solver (schemi_b200/host/schemi_adapter) call --
// fv_create, fv_destroy, fv_last_error, fv_upload, fv_run, fv_step, fv_download, fv_get_time,
// fv_set_time, fv_get_source_timestep -- implemented over the FP64 CPU oracle (fv_oracle.cpp).  Linking the driver
// against this library instead of libschemi_fv.so gives lib/fvrun_oracle, with which the CPU
// tests check the driver's deck reader, time loop, restart and file writer against the
// reference's own result files without a GPU; linking the reference's main with the step
// solver against it checks the step solver the same way.  Neither shipped binary loads it.
#include <cstdio>
#include <string>

#include "fv_oracle.h"

struct fv_handle {
    fvo_case* c = nullptr;
    std::string err;
};

extern "C" {

fv_status fv_create(const fv_config* cfg, fv_handle** out) {
    if (!cfg || !out) return FV_ERR_INIT;
    char err[1024] = {0};
    fvo_case* c = fvo_create(cfg, err, sizeof err);
    if (!c) {
        std::fprintf(stderr, "%s\n", err);
        return FV_ERR_INIT;
    }
    *out = new fv_handle{c, {}};
    return FV_OK;
}

void fv_destroy(fv_handle* h) {
    if (!h) return;
    fvo_destroy(h->c);
    delete h;
}

const char* fv_last_error(const fv_handle* h) { return h ? h->err.c_str() : "no handle"; }

fv_status fv_upload(fv_handle* h, const double* const* prim) {
    if (!h || !prim) return FV_ERR_INIT;
    return (fv_status)fvo_upload(h->c, prim);
}

fv_status fv_run(fv_handle* h, double t_end, long long max_steps, fv_run_stats* stats) {
    if (!h) return FV_ERR_INIT;
    double t = 0, dt = 0;
    long long n = 0;
    const int st = fvo_run(h->c, t_end, max_steps, &t, &n);
    fvo_get_time(h->c, &t, &dt);
    if (st != FV_OK) h->err = "oracle step failed with status " + std::to_string(st);
    if (stats) {
        stats->time = t;
        stats->dt_next = dt;
        stats->steps = n;
        stats->device_ms = 0;
    }
    return (fv_status)st;
}

fv_status fv_step(fv_handle* h, double* dt_used, double* dt_next) {
    if (!h) return FV_ERR_INIT;
    double used = 0, next = 0;
    const int st = fvo_step(h->c, &used, &next);
    if (st != FV_OK) h->err = "oracle step failed with status " + std::to_string(st);
    if (dt_used) *dt_used = used;
    if (dt_next) *dt_next = next;
    return (fv_status)st;
}

fv_status fv_download(fv_handle* h, double* const* out) {
    if (!h || !out) return FV_ERR_INIT;
    return (fv_status)fvo_download(h->c, out);
}

fv_status fv_get_time(const fv_handle* h, double* time, double* dt) {
    if (!h) return FV_ERR_INIT;
    double t = 0, d = 0;
    fvo_get_time(h->c, &t, &d);
    if (time) *time = t;
    if (dt) *dt = d;
    return FV_OK;
}

fv_status fv_get_source_timestep(const fv_handle* h, double* dt_source) {
    if (!h) return FV_ERR_INIT;
    return (fv_status)fvo_get_source_timestep(h->c, dt_source);
}

fv_status fv_set_time(fv_handle* h, double time, double dt) {
    if (!h) return FV_ERR_INIT;
    return (fv_status)fvo_set_time(h->c, time, dt);
}

}  // extern "C"
