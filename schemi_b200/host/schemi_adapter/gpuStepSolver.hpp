// gpuStepSolver.hpp -- the step solver a Schemi maintainer adds to run this library's step inside
// the reference's own main (the drop-in boundary of include/fvstep.h in use).
//
// It derives from schemi::abstractStepSolver (Schemi/headers/abstractStepSolver.hpp:27-112) and is
// registered in abstractStepSolver::createStepSolver (src/interfaces/abstractStepSolver.cpp:56-146)
// under the reference's approximation-order names with a "Gpu" prefix: a deck with
// "#Approximation_order GpuSecondOrder" (or GpuSecondOrderRK, GpuThirdOrder, GpuThirdOrderCada)
// runs the reference's main unchanged -- its task-file reader, its CFL block, its outputs -- with
// calculateStep() on the library.  The library is whichever implementation of fvstep.h the
// program links: libschemi_fv.so (the B200 kernels) or the CPU restatement that implements the
// same C-ABI.
//
// makeGpuStepSolver() refuses a "Gpu..." name whose rest is not an order name with the factory's
// own message, reads the deck (set/*.txt, with the reader of the task-deck driver; a deck outside
// the library's step is refused there, before the first step, with that reader's message), creates
// the handle and uploads the phase's initial set (c_1..c_N, v, p), so that the first step starts
// from the primitives main initialised, as the reference's step does.
//
// calculateStep():
//   * every call sets the step to main's time step (mesh::timestep()), runs one step (fv_step:
//     the whole step of the named step solver, e.g. secondOrderStepSolver::calculateStep,
//     src/solverStages/secondOrderStepSolver.cpp, over Advection.cpp:20-513), and writes the new
//     state back into the phase: concentrations, densities, velocity, pressure, momentum, total
//     and internal energy, temperature, and the Helmholtz energy and entropy from the phase's own
//     thermodynamics (as Advection.cpp:455-486 does), and the source time step a diffusion stage
//     set on the mesh (fv_get_source_timestep), so main's CFL block and outputs read what they
//     read after the reference's step;
//   * a failed step throws schemi::exception with the library's message and the reference's errors
//     value (fv_status numbers them alike), which main turns into its emergency output.
// The device state is kept between steps; main changes the phase only through this solver.
#ifndef GPUSTEPSOLVER_HPP_
#define GPUSTEPSOLVER_HPP_

#include <memory>
#include <string>

#include "abstractStepSolver.hpp"
#include "fvstep.h"

namespace schemi
{
class gpuStepSolver: public abstractStepSolver
{
	fv_handle* h = nullptr;

	void writeBack();

public:
	using abstractStepSolver::abstractStepSolver;

	~gpuStepSolver() noexcept override;

	// reads the deck, creates the handle and uploads the phase (throws schemi::exception)
	void open();

	void calculateStep() override;
};

// The factory's branch for the "Gpu..." names (the name, then the arguments of createStepSolver).
std::unique_ptr<abstractStepSolver> makeGpuStepSolver(const std::string & name,
		homogeneousPhase<cubicCell> & gasPhase_in,
		const abstractLimiter & limiter_in,
		const abstractFlowSolver & fsolver_in, const bool & gravitationFlag_in,
		const vector & g_in,
		const boundaryConditionValue & boundaryConditionValueCalc_in,
		scalar & timeForTVD_in, scalar & timeForHancock_in,
		scalar & timeForFlowCalculation_in, scalar & timeForTimeIntegration_in,
		const MPIHandler & parallelism_in, const bool & diffusionFlag_in,
		const abstractMatrixSolver & msolver_in,
		const abstractMatrixSolver & msolverEnthFl_in,
		const std::pair<scalar, scalar> & timestepCoeffs_in,
		scalar & timeForDiffusion_in,
		const std::vector<boundaryConditionType> & commonConditions_in,
		const enthalpyFlow & enthalpyFlowFlag_in, const bool & linearFlag_in,
		const volumeField<scalar> & minimalLengthScale_in,
		const timestep & sourceTimeFlag_in,
		const bool & molMassDiffusionFlag_in,
		chemicalKinetics::abstractChemicalKinetics & chemKin_in,
		const bool & nonLinearityIteratonsFlag_in);
}  // namespace schemi

#endif /* GPUSTEPSOLVER_HPP_ */
