// fv_diffusion_launch.h -- launcher of the diffusion stage (fv_diffusion.cu).
#pragma once

#include <cuda_runtime.h>

#include "fv_kernels.cuh"

namespace fv {

struct GenericLayout;
namespace diff {

// Coefficients and buffers of the stage (allocated by the handle when cfg.diffusion is on).
struct DiffParams {
    double mu, D, kappa;       // the transport model's constants (fv_config mu/D/kappa_const)
    int transport;             // fv_transport
    int pad0;
    double diam[FV_MAX_SPECIES];   // HARD_SPHERES: kinetic diameters (angstrom)
    double ljEps[FV_MAX_SPECIES];  // LENNARD_JONES: eps / k_B (K)
    double ljSig[FV_MAX_SPECIES];  // LENNARD_JONES: sigma (angstrom)
    int enthalpy;              // 1: an enthalpy flow (explicit or implicit)
    int enthImplicit;          // 1: the implicit one (the upwind term in the temperature matrix)
    int molmass;               // 1: molar-mass diffusion correction
    int interpV;               // 1: cell velocity gradient from interpolated cell velocities
                               //    ("linear" reconstruction, or gravity), else the star velocities
    int dtDiff;                // 1: "Courant-Source-Diffusion" (the diffusion limit)
    int gs;                    // 1: an implicit solver (the stage's matrices; fv_sle_solver in sle)
    int sle;                   // fv_sle_solver of the implicit branch (gs)
    int maxIter;               // its iteration limit (#Number_of_iterations_of_SLE_matrix_solver)
    double coeffSource, coeffDiff;
    double* starV;             // [3][faces] Riemann star velocity of the advection (replaced by
                               //    the interpolated cell velocity when interpV)
    double* starP;             // [faces] its star pressure (the face coefficients' pressure)
    double* cellPrim;          // [2N + 5][stride]: c_1..c_N, v_x, v_y, v_z, p, T, w_1..w_N
    double* face;              // [faceSlotCount(N)][faces] face quantities (see faceSlots)
    double* stagePrim;         // [N + 6][stride]: c_1..c_N, v, p, Uv, T after the stage
    double* partMin;           // [2][blocks] per-CTA minima of the enthalpy and diffusion limits
    // the implicit solver's matrices and solutions (null with the explicit solver); face slots s
    // in the cell's face order [x-, x+, y+, y-, z-, z+]
    double* wDiag;             // [N][stride] mass fractions: diagonal, free term
    double* wFree;
    double* wOff;              // [N][6][stride] their off-diagonal coefficient per face slot
    double* vDiag;             // [stride] velocity: diagonal (shared by the components)
    double* vFree;             // [3][stride]
    double* vOff;              // [6][stride]
    double* tDiag;             // [stride] temperature
    double* tFree;
    double* tOff;              // [6][stride]
    double* sol;               // [N + 4][stride] solutions: w_1..w_N, v_x, v_y, v_z, T
    double* work;              // [7][stride] solver scratch: the Gauss-Seidel and Jacobi iterates
                               //    (when they exceed shared memory) and 1 / diag; the
                               //    conjugate-gradient vectors
    double* cNew;              // [N + 3][stride] concentrations c_0..c_N, CCVNew, old energy
};

// face quantity slots per face (fv_diffusion.cuh: faceSlots<N>() is the same count)
__host__ __device__ constexpr int faceSlotCount(int ns) { return 3 * ns + 13; }

}  // namespace diff

// CTAs of the stage's cell kernel (= blockMax entries it writes, and the partial minima per limit).
int diffusionBlocks(const StepParams& P);

// Opt the Gauss-Seidel solve in to the shared memory its iterates need (outside any capture).
cudaError_t configureDiffusion(int dims, const StepParams& P);

// Enqueue the diffusion stage of the advected state U (in place) with the clock's dt: the new
// state, its primitives (P.stagePrim), the CFL block maxima and the clock's source time step.
cudaError_t launchDiffusion(int ns, int eos, int dims, const StepParams& P, const GenericLayout& L,
                            const diff::DiffParams& X, double* U, DevClock* ck, double* blockMax, cudaStream_t st);

}  // namespace fv
