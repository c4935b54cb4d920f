// gpuStepSolver.cpp -- see gpuStepSolver.hpp.
#include "gpuStepSolver.hpp"

#include <vector>

#include "../deck.hpp"
#include "exception.hpp"
#include "mesh.hpp"

schemi::gpuStepSolver::~gpuStepSolver() noexcept
{
	if (h)
		fv_destroy(h);
}

void schemi::gpuStepSolver::open()
{
	fv_config cfg;
	try
	{
		// the deck main has read, with the task-deck driver's reader (no result files touched);
		// the step solver is the one the "Gpu..." name names
		cfg = fvdeck::readDeck(".", false).cfg;
	} catch (const std::exception & e)
	{
		throw exception(e.what(), errors::initialisationError);
	}
	const fv_status st = fv_create(&cfg, &h);
	if (st != FV_OK)
	{
		h = nullptr;
		throw exception("fv_create failed", static_cast<errors>(st));
	}
	// the restart set as the phase holds it: c_1..c_N, v_x, v_y, v_z, p
	const std::size_t N = gasPhase.concentration.v.size() - 1;
	const std::size_t nc = gasPhase.pressure.cval().size();
	std::vector<std::vector<double>> prim(N + 4, std::vector<double>(nc));
	for (std::size_t k = 0; k < N; ++k)
		for (std::size_t i = 0; i < nc; ++i)
			prim[k][i] = gasPhase.concentration.v[k + 1].cval()[i];
	for (std::size_t i = 0; i < nc; ++i)
	{
		const auto & v = gasPhase.velocity.cval()[i]();
		prim[N][i] = v[0];
		prim[N + 1][i] = v[1];
		prim[N + 2][i] = v[2];
		prim[N + 3][i] = gasPhase.pressure.cval()[i];
	}
	std::vector<const double*> ptr(N + 4);
	for (std::size_t q = 0; q < N + 4; ++q)
		ptr[q] = prim[q].data();
	if (fv_upload(h, ptr.data()) != FV_OK)
		throw exception(fv_last_error(h), errors::systemError);
}

void schemi::gpuStepSolver::writeBack()
{
	const std::size_t N = gasPhase.concentration.v.size() - 1;
	const std::size_t nc = gasPhase.pressure.cval().size();
	std::vector<std::vector<double>> f(FV_F_COUNT, std::vector<double>(nc));
	std::vector<double*> ptr(FV_F_COUNT);
	for (int q = 0; q < FV_F_COUNT; ++q)
		ptr[q] = f[q].data();
	const fv_status st = fv_download(h, ptr.data());
	if (st != FV_OK)
		throw exception(fv_last_error(h), static_cast<errors>(st));
	for (std::size_t i = 0; i < nc; ++i)
	{
		gasPhase.concentration.v[0].val()[i] = f[FV_F_CONC0][i];
		gasPhase.density[0].val()[i] = f[FV_F_RHO][i];
		for (std::size_t k = 0; k < N; ++k)
		{
			gasPhase.concentration.v[k + 1].val()[i] = f[FV_F_CONC + k][i];
			gasPhase.density[k + 1].val()[i] = f[FV_F_RHO_K + k][i];
		}
		gasPhase.velocity.val()[i] = vector(f[FV_F_VX][i], f[FV_F_VY][i],
				f[FV_F_VZ][i]);
		gasPhase.momentum.val()[i] = vector(f[FV_F_MX][i], f[FV_F_MY][i],
				f[FV_F_MZ][i]);
		gasPhase.pressure.val()[i] = f[FV_F_P][i];
		gasPhase.totalEnergy.val()[i] = f[FV_F_E][i];
		gasPhase.internalEnergy.val()[i] = f[FV_F_UV][i];
		gasPhase.temperature.val()[i] = f[FV_F_T][i];
	}
	// Advection.cpp:481-486: the cell's Helmholtz energy and entropy from its thermodynamics
	gasPhase.HelmholtzEnergy.val() = gasPhase.phaseThermodynamics->Fv(
			gasPhase.concentration.p, gasPhase.temperature.cval());
	gasPhase.entropy.val() = gasPhase.phaseThermodynamics->Sv(
			gasPhase.concentration.p, gasPhase.temperature.cval());
}

void schemi::gpuStepSolver::calculateStep()
{
	if (!h)
		throw exception("the library's step solver was not opened", errors::initialisationError);
	double time = 0, dt = 0;
	fv_get_time(h, &time, &dt);
	// the step main chose (its CFL block, minimal step and end-time clamp)
	if (fv_set_time(h, time, gasPhase.pressure.meshRef().timestep()) != FV_OK)
		throw exception(fv_last_error(h), errors::systemError);
	double dtUsed = 0, dtNext = 0;
	const fv_status st = fv_step(h, &dtUsed, &dtNext);
	if (st != FV_OK)
		throw exception(fv_last_error(h), static_cast<errors>(st));
	// the source time step the step's diffusion stage set (Diffusion.cpp:688-706,1036-1049 set it
	// on the mesh), which main's CFL block takes into the next step
	double dtSource = 0;
	if (fv_get_source_timestep(h, &dtSource) != FV_OK)
		throw exception(fv_last_error(h), errors::systemError);
	const_cast<mesh&>(gasPhase.pressure.meshRef()).timestepSourceRef() = dtSource;
	writeBack();
}

std::unique_ptr<schemi::abstractStepSolver> schemi::makeGpuStepSolver(
		const std::string & name, homogeneousPhase<cubicCell> & gasPhase_in,
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
		const bool & nonLinearityIteratonsFlag_in)
{
	// the factory's own refusal (abstractStepSolver.cpp:87-94) for a name that is not an order
	if (name != "GpuSecondOrder" && name != "GpuSecondOrderRK" && name != "GpuThirdOrder"
			&& name != "GpuThirdOrderCada")
		throw exception("Unknown gas dynamics approximation order.",
				errors::initialisationError);
	auto solver = std::make_unique<gpuStepSolver>(gasPhase_in, limiter_in,
			fsolver_in, gravitationFlag_in, g_in, boundaryConditionValueCalc_in,
			timeForTVD_in, timeForHancock_in, timeForFlowCalculation_in,
			timeForTimeIntegration_in, parallelism_in, diffusionFlag_in,
			msolver_in, msolverEnthFl_in, timestepCoeffs_in, timeForDiffusion_in,
			commonConditions_in, enthalpyFlowFlag_in, linearFlag_in,
			minimalLengthScale_in, sourceTimeFlag_in, molMassDiffusionFlag_in,
			chemKin_in, nonLinearityIteratonsFlag_in);
	solver->open();
	return solver;
}
