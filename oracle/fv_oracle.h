/*
 * fv_oracle.h -- TEST INFRASTRUCTURE, not part of the product.
 *
 * C interface of the FP64 CPU restatement of Schemi's explicit finite-volume step
 * (fv_oracle.cpp).  Only the parity tests, the smoke check and the bench's CPU-baseline
 * leg load it; the product path never does.
 */
#ifndef SCHEMI_B200_FV_ORACLE_H_
#define SCHEMI_B200_FV_ORACLE_H_

#include "../include/fvstep.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fvo_case fvo_case;

fvo_case* fvo_create(const fv_config* cfg, char* err, int err_len);
void fvo_destroy(fvo_case* c);

/* Restart set c_1..c_N, v_x, v_y, v_z, p; sets time = 0, dt = min_timestep. */
int fvo_upload(fvo_case* c, const double* const* prim);

/* One step with the current dt, then the CFL block (no end-time clamp). */
int fvo_step(fvo_case* c, double* dt_used, double* dt_next);

/* Main's time loop until time >= t_end or max_steps steps. */
int fvo_run(fvo_case* c, double t_end, long long max_steps, double* time, long long* steps);

/* Output set in fv_field order; out[f] may be NULL. */
int fvo_download(fvo_case* c, double* const* out);

int fvo_get_time(const fvo_case* c, double* time, double* dt);
int fvo_set_time(fvo_case* c, double time, double dt);
int fvo_get_source_timestep(const fvo_case* c, double* dt_source);

/* Conserved state rho_1..rho_N, rho, m_x, m_y, m_z, E (n_cells each): get / set. */
int fvo_get_conserved(const fvo_case* c, double* const* out);
int fvo_set_conserved(fvo_case* c, const double* const* in);

long long fvo_n_cells(const fvo_case* c);

/* Chemistry sub-cycling after a failed cell: carry = 1 (default) keeps the finer sub-step for the
 * cells that follow in cell order, as the reference's serial loop does; carry = 0 sub-cycles each
 * cell on its own, as the CUDA path does. */
int fvo_set_chem_carry(fvo_case* c, int carry);

#ifdef __cplusplus
}
#endif

#endif
