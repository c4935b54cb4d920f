// fv_validate.h -- the configuration checks and the mixture parameters of fv_create, shared by
// every entry point that takes an fv_config (fv_create, fv_step_noalloc).  Host code only.
#pragma once

#include <cmath>
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
    if (c.eos < FV_EOS_IDEAL || c.eos > FV_EOS_KATAOKA) { e = "unknown equation of state"; return false; }
    if (c.eos == FV_EOS_STIFFENED)
        for (int k = 0; k < c.n_species; ++k)
            if (!(c.stiff_gamma[k] > 1) || !(c.stiff_p0[k] >= 0)) {
                e = "stiffened gas needs gamma > 1 and p0 >= 0 for every species";
                return false;
            }
    if (c.eos == FV_EOS_KATAOKA) {
        for (int k = 0; k < c.n_species; ++k)
            if (!(c.lj_sigma[k] > 0) || !(c.lj_eps[k] >= 0)) {
                e = "Kataoka needs a positive Lennard-Jones sigma and a non-negative eps for every species";
                return false;
            }
        if (!(c.kataoka_b_coeff > 0)) { e = "Kataoka needs a positive b coefficient"; return false; }
    }
    if (c.diffusion) {
        // the diffusion stage (Diffusion.cpp) this build runs: after the SecondOrder advection, HLLC
        // star states, FP64, ideal or van der Waals, the constant, hard-sphere or Lennard-Jones
        // coefficients, the explicit or Gauss-Seidel solver, no or explicit enthalpy flow; a
        // chemical mechanism follows the stage
        if (c.order != FV_ORDER_SECOND) { e = "the diffusion stage runs with the SecondOrder step"; return false; }
        if (c.flux != FV_FLUX_HLLC) { e = "the diffusion stage runs with the HLLC flux"; return false; }
        if (c.precision != FV_PREC_F64) { e = "the diffusion stage runs in FP64"; return false; }
        if (c.eos != FV_EOS_IDEAL && c.eos != FV_EOS_VAN_DER_WAALS) {
            e = "the diffusion stage runs with ideal and van der Waals mixtures";
            return false;
        }
        if (c.sle_solver < FV_SLE_EXPLICIT || c.sle_solver > FV_SLE_BICG) {
            e = "unknown matrix solver";
            return false;
        }
        if (c.sle_solver != FV_SLE_EXPLICIT) {
            // the implicit solvers index a cell's neighbours without wrap-around
            for (int p = 0; p < 6; ++p)
                if (c.bc_vel[p] == FV_BC_PERIODIC) {
                    e = "the implicit diffusion solvers run without periodic axes";
                    return false;
                }
            if (c.sle_max_iter < 1) { e = "the iterative solvers need at least one iteration"; return false; }
        }
        if (c.sle_solver == FV_SLE_THOMAS && (c.dims != 1 || c.n[0] < 2)) {
            e = "the Thomas solver runs on 1D meshes of at least 2 cells";
            return false;
        }
        if (c.transport < FV_TRANSPORT_CONSTANT || c.transport > FV_TRANSPORT_LENNARD_JONES) {
            e = "unknown transport model";
            return false;
        }
        for (int k = 0; k < c.n_species; ++k) {
            if (c.transport == FV_TRANSPORT_HARD_SPHERES && !(c.transport_diameter[k] > 0)) {
                e = "hard-sphere diameters must be positive";
                return false;
            }
            if (c.transport == FV_TRANSPORT_LENNARD_JONES && !(c.transport_lj_eps[k] > 0 && c.transport_lj_sigma[k] > 0)) {
                e = "Lennard-Jones parameters must be positive";
                return false;
            }
        }
        if (c.enthalpy_flow < FV_ENTHALPY_NO || c.enthalpy_flow > FV_ENTHALPY_IMPLICIT) {
            e = "unknown enthalpy flow flag";
            return false;
        }
    }
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
    if (c.chemistry != FV_CHEM_NONE && c.eos != FV_EOS_IDEAL && c.eos != FV_EOS_VAN_DER_WAALS) {
        e = "the chemistry pass runs with ideal and van der Waals mixtures";
        return false;
    }
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

// Mixture parameters of the device EOS (the reference's constructors, each in its own order):
// van der Waals mixtureVanDerWaals.cpp:33-52, Redlich-Kwong mixtureRedlichKwong.cpp:34-60,
// stiffened mixtureStiffened.cpp:19-42, Kataoka mixtureKataokaVanDerWaals.cpp:20-75.
template <class MixParamsT>
inline void fvMixParams(const fv_config& c, MixParamsT& mp) {
    const int N = c.n_species;
    mp.ns = N;
    mp.eos_kind = c.eos;
    mp.R = c.R;
    for (int k = 0; k < N; ++k) {
        mp.M[k] = c.M[k];
        mp.invM[k] = 1.0 / c.M[k];
        mp.Cv[k] = c.Cv[k];
    }
    auto pairs = [&](double (*m)[FV_MAX_SPECIES], bool cubeMean) {
        for (int k = 0; k < N; ++k)
            for (int l = 0; l < N; ++l)
                if (k != l)
                    m[k][l] = cubeMean ? std::pow(0.5 * (std::cbrt(m[k][k]) + std::cbrt(m[l][l])), 3)
                                       : std::sqrt(m[k][k] * m[l][l]);
    };
    if (c.eos == FV_EOS_VAN_DER_WAALS) {
        for (int k = 0; k < N; ++k) {
            mp.b[k][k] = c.Tc[k] * mp.R / (8 * c.Pc[k]);
            mp.a[k][k] = c.Pc[k] * mp.b[k][k] * mp.b[k][k] * 27;
        }
        pairs(mp.b, true);
        pairs(mp.a, false);
    } else if (c.eos == FV_EOS_REDLICH_KWONG) {
        // cbrt(2) correctly rounded, the value g++ folds std::cbrt(2) to in the reference's
        // constant expression (mixtureRedlichKwong.cpp:34-37)
        constexpr double chi{0x1.428a2f98d728bp+0 - 1.};
        constexpr double Sigma_a{1. / (9. * chi)}, Sigma_b{chi / 3.};
        for (int k = 0; k < N; ++k) {
            mp.b[k][k] = Sigma_b * mp.R * c.Tc[k] / c.Pc[k];
            mp.a[k][k] = Sigma_a * mp.R * mp.R * c.Tc[k] * c.Tc[k] * std::sqrt(c.Tc[k]) / c.Pc[k];
        }
        pairs(mp.b, true);
        pairs(mp.a, false);
    } else if (c.eos == FV_EOS_STIFFENED) {
        for (int k = 0; k < N; ++k) {
            mp.p0[k][k] = c.stiff_p0[k];
            mp.g[k][k] = c.stiff_gamma[k];
        }
        pairs(mp.p0, false);
        pairs(mp.g, false);
    } else if (c.eos == FV_EOS_KATAOKA) {
        constexpr double NA = 6.02214076E23;  // globalConstants.hpp NAvogardro
        for (int k = 0; k < N; ++k) {
            const double sg = c.lj_sigma[k];
            mp.b[k][k] = c.kataoka_b_critical ? c.kataoka_b_coeff * mp.R * c.Tc[k] / (8 * c.Pc[k])
                                              : c.kataoka_b_coeff * (sg * sg * sg) * NA;
            mp.V0[k][k] = (sg * sg * sg) / std::sqrt(2) * NA;
            mp.ep[k][k] = c.lj_eps[k];
        }
        pairs(mp.b, true);
        pairs(mp.V0, true);
        pairs(mp.ep, false);
    }
}

// The EOS template value of the device kernels for a configuration's EOS.
inline int fvEosTemplate(int eos) { return eos == FV_EOS_IDEAL ? 0 : eos == FV_EOS_VAN_DER_WAALS ? 1 : 9; }
