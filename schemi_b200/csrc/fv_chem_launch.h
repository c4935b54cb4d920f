// fv_chem_launch.h -- launcher of the chemistry pass (fv_chem.cu).
#pragma once

#include <cuda_runtime.h>

#include "fv_kernels.cuh"

namespace fv {
namespace chem {

// Mechanism, per-cell solver and Arrhenius parameters of the chemistry pass.
struct ChemParams {
    int mech;         // fv_chemistry
    int solver;       // fv_chem_solver
    int maxIter;
    double Af, nf, Ef, Ab, nb, Eb;
    double q;
    double* conc;     // concentrations c_0..c_N kept as state (stride apart) after a multi-stage
                      // average: read as the pass's input and replaced by their 0.5 average with
                      // the integrated ones; null: c_k = rho_k / M_k
    const double* stage;  // primitives a diffusion stage left (c_1..c_N, v, p, Uv, T; stride
                          // apart): the pass's input concentrations, velocity, internal energy and
                          // temperature (the phase after Diffusion, secondOrderStepSolver.cpp:69-91);
                          // null: from the state
};

}  // namespace chem

// CTAs of the chemistry pass (= blockMax entries it writes).
int chemistryBlocks(const StepParams& P);

// Enqueue the chemistry of the state U (in place) with the clock's dt, writing the CFL block maxima.
cudaError_t launchChemistry(int ns, int eos, int dims, const StepParams& P, const chem::ChemParams& C, double* U,
                            DevClock* ck, double* blockMax, cudaStream_t st);

}  // namespace fv
