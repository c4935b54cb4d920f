// fv_validate.h -- the configuration checks of fv_create, shared by every entry point that takes
// an fv_config (fv_create, fv_step_noalloc).  Host code only.
#pragma once

#include <string>

#include "../../include/fvstep.h"

// True when `c` describes a case the step can run; otherwise false with the reason in `e`.
inline bool fvValidateConfig(const fv_config& c, std::string& e) {
    if (c.dims < 1 || c.dims > 3) { e = "dims must be 1, 2 or 3"; return false; }
    for (int d = 0; d < c.dims; ++d)
        if (c.n[d] < 1) { e = "cell counts must be positive"; return false; }
    for (int d = 0; d < 3; ++d)
        if (!(c.L[d] > 0)) { e = "parallelepiped extents must be positive"; return false; }
    if (c.n_species < 1 || c.n_species > FV_MAX_SPECIES) { e = "n_species must be 1..4"; return false; }
    if (c.eos != FV_EOS_IDEAL && c.eos != FV_EOS_VAN_DER_WAALS) { e = "unknown equation of state"; return false; }
    if (c.flux != FV_FLUX_HLLC && c.flux != FV_FLUX_HLL) { e = "unknown flux solver"; return false; }
    if (c.limiter < 0 || c.limiter > FV_LIM_SCHMIDTMANN) { e = "unknown limiter"; return false; }
    if (c.precision != FV_PREC_F64 && c.precision != FV_PREC_F32_FLUX) { e = "unknown precision"; return false; }
    for (int k = 0; k < c.n_species; ++k)
        if (!(c.M[k] > 0) || !(c.Cv[k] > 0)) { e = "molar mass and Cv must be positive"; return false; }
    static const int lo[3] = {FV_PATCH_TAIL, FV_PATCH_RIGHT, FV_PATCH_BOTTOM};
    static const int hi[3] = {FV_PATCH_POINT, FV_PATCH_LEFT, FV_PATCH_TOP};
    for (int a = 0; a < c.dims; ++a) {
        for (int side = 0; side < 2; ++side) {
            const int p = side ? hi[a] : lo[a];
            auto okType = [](int t) {
                return t == FV_BC_FREE || t == FV_BC_SLIP || t == FV_BC_FIXED_CELL || t == FV_BC_FIXED_SURFACE ||
                       t == FV_BC_PERIODIC;
            };
            if (!okType(c.bc_vel[p]) || !okType(c.bc_p[p])) { e = "unknown boundary condition type"; return false; }
            for (int k = 0; k < c.n_species; ++k)
                if (!okType(c.bc_conc[p][k])) { e = "unknown boundary condition type"; return false; }
        }
        const bool per = c.bc_vel[lo[a]] == FV_BC_PERIODIC;
        auto allPer = [&](int p) {
            if ((c.bc_vel[p] == FV_BC_PERIODIC) != per || (c.bc_p[p] == FV_BC_PERIODIC) != per) return false;
            for (int k = 0; k < c.n_species; ++k)
                if ((c.bc_conc[p][k] == FV_BC_PERIODIC) != per) return false;
            return true;
        };
        if (!allPer(lo[a]) || !allPer(hi[a])) {
            e = "a periodic axis needs periodic conditions for every field on both patches";
            return false;
        }
        if (per && c.n[a] < 2) { e = "a periodic axis needs at least 2 cells"; return false; }
    }
    if (c.chemistry < FV_CHEM_NONE || c.chemistry > FV_CHEM_CL2) { e = "unknown chemistry"; return false; }
    if (c.chemistry == FV_CHEM_A_B_2C && c.n_species != 3) { e = "A+B->2C needs 3 species (A, B, C)"; return false; }
    if (c.chemistry == FV_CHEM_CL2 && c.n_species != 2) { e = "Cl2 dissociation needs 2 species (Cl2, Cl)"; return false; }
    if (c.order < FV_ORDER_SECOND || c.order > FV_ORDER_THIRD_CADA) {
        e = "unknown step solver (order)";
        return false;
    }
    if (c.chemistry != FV_CHEM_NONE) {
        if (c.chem_solver < FV_CHEM_GAUSS_SEIDEL || c.chem_solver > FV_CHEM_JACOBI_CONJUGATE_GRADIENT) {
            e = "unknown chemical iterative solver";
            return false;
        }
        if (c.chem_max_iter < 1 || c.chem_max_iter > 1000000) {
            e = "chem_max_iter must be 1..1000000";
            return false;
        }
    }
    return true;
}
