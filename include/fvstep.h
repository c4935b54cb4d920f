/*
 * fvstep.h -- C-ABI of the B200 explicit finite-volume step (Schemi drop-in).
 *
 * One opaque handle owns one case: a structured parallelepiped mesh held on one GPU,
 * its conserved state in structure-of-arrays FP64 storage, and one CUDA stream.
 * Every entry point returns an int status whose values are the reference's `errors`
 * enumeration (Schemi/enumerations/errorsEnum.hpp:15-30): 0 = noErrors.
 *
 * Reference interfaces replaced by this boundary (paths inside the Schemi project):
 *   fv_create    <- main's factory/mesh/phase set-up: Schemi/main/Schemi.cpp:269-278,597-639,
 *                   abstractFlowSolver::createFlowSolver (src/interfaces/abstractFlowSolver.cpp:25-71),
 *                   abstractLimiter::createLimiter (src/interfaces/abstractLimiter.cpp:35-113),
 *                   abstractMixtureThermodynamics::createThermodynamics
 *                   (src/interfaces/abstractMixtureThermodynamics.cpp:32-159)
 *   fv_upload    <- phaseInitialization derived fields (src/thermodynamics/phaseInitialization.cpp:1827-1885)
 *                   fed with the restart set c_k, v, p (fieldsOutput/output_N/<field>.dat)
 *   fv_step      <- abstractStepSolver::calculateStep (headers/abstractStepSolver.hpp:108) as
 *                   implemented by secondOrderStepSolver (src/solverStages/secondOrderStepSolver.cpp:48-93)
 *                   with Advection() (src/Advections/Advection.cpp:20-513), followed by main's
 *                   CFL block (Schemi/main/Schemi.cpp:802-835)
 *   fv_run       <- main's time loop (Schemi/main/Schemi.cpp:664-670,767-940) incl. the last-step clamp
 *   fv_download  <- structForOutput::collectParallelData + output::dataOutput field set
 *                   (src/service/output.cpp:14-308), in internal cell order (x fastest)
 *   fv_batch_*   <- no reference counterpart (the reference runs one case per process)
 *   fv_adjoint_* <- no reference counterpart (the reference has no adjoint)
 */
#ifndef SCHEMI_B200_FVSTEP_H_
#define SCHEMI_B200_FVSTEP_H_

#ifdef __cplusplus
extern "C" {
#endif

#define FV_ABI_VERSION 7
#define FV_MAX_SPECIES 4

typedef int fv_status;

/* errors enum of the reference (errorsEnum.hpp:15-30). */
enum fv_error_code {
    FV_OK = 0,
    FV_ERR_RIEMANN = 1,           /* RiemannSolverError: NaN wave speeds (HLLCSolver.cpp:385-388) */
    FV_ERR_NEGATIVE_T = 2,        /* negativeTemperatureError */
    FV_ERR_TOO_BIG_OUTPUT = 3,
    FV_ERR_SYSTEM = 4,            /* systemError: CUDA failures, bad handle */
    FV_ERR_BOUNDARY = 5,          /* boundaryConditionError */
    FV_ERR_CUBIC = 6,
    FV_ERR_POSITIVENESS = 7,
    FV_ERR_MPI = 8,
    FV_ERR_FIELD_INIT = 9,
    FV_ERR_MESH = 10,             /* meshGenerationError */
    FV_ERR_INIT = 11,             /* initialisationError: invalid configuration */
    FV_ERR_NAN = 12               /* NaNError: non-finite state detected after a step */
};

/* Equation of state: the five names of abstractMixtureThermodynamics.cpp:39-43 ("ideal",
 * "vanDerWaals", "RedlichKwong", "stiffened", "Kataoka").  Ideal and van der Waals mixtures run
 * on every path; the other three on the generic path (fv_step / fv_run), without chemistry.
 *   REDLICH_KWONG  mixtureRedlichKwong.cpp: a, b from Tc and Pc, T from Uv by the cubic in sqrt(T)
 *                  of RedlichKwongFluid.cpp:46-127 (the reference solves it in long double; the
 *                  device in FP64)
 *   STIFFENED      mixtureStiffened.cpp: stiff_p0 and stiff_gamma per species
 *                  (set/stiffenedFluidData.txt)
 *   KATAOKA        mixtureKataokaVanDerWaals.cpp: T from Uv or p by the Newton iteration of
 *                  NewtonMethod.cpp:13-40 on KataokaVanDerWaalsFluid.cpp's series; lj_eps,
 *                  lj_sigma and the b rule (set/KataokaVanDerWaalsFluidData.txt) */
enum fv_eos {
    FV_EOS_IDEAL = 0, FV_EOS_VAN_DER_WAALS = 1, FV_EOS_REDLICH_KWONG = 2, FV_EOS_STIFFENED = 3,
    FV_EOS_KATAOKA = 4
};

/* Flux solver: names of abstractFlowSolver.cpp:29-35 that this build implements. */
enum fv_flux { FV_FLUX_HLLC = 0, FV_FLUX_HLL = 1 };

/* Limiter: values of typeOfTVDLimiterEnum.hpp (factory names abstractLimiter.cpp:39-53). */
enum fv_limiter {
    FV_LIM_ZERO = 0, FV_LIM_MINMOD = 1, FV_LIM_VANLEER = 2, FV_LIM_LINEAR = 3,
    FV_LIM_VANALBADA = 4, FV_LIM_HQUICK = 5, FV_LIM_VANLEER2 = 6, FV_LIM_SUPERBEE = 7,
    FV_LIM_VANALBADA2 = 8, FV_LIM_MINMOD2 = 9, FV_LIM_SWEBY = 10, FV_LIM_KOREN = 11,
    FV_LIM_KOREN2 = 12, FV_LIM_UTCDFS = 13, FV_LIM_SCHMIDTMANN = 14
};

/* Boundary-condition types: values of boundaryConditionTypesEnum.hpp:15-34.
 * FV_BC_PERIODIC has no counterpart in the reference (it offers no periodic patch); it must be
 * set on both patches of an axis for every field. */
enum fv_bc {
    FV_BC_FREE = 1, FV_BC_SLIP = 2, FV_BC_FIXED_CELL = 3, FV_BC_FIXED_SURFACE = 4,
    FV_BC_PERIODIC = 100
};

/* Patch order of the task files (#Tail, #Point, #Bottom, #Right, #Left, #Top):
 * tail = x-min, point = x-max, bottom = z-min, right = y-min, left = y-max, top = z-max
 * (mesh.cpp:350-420, 781-860, 1572-1760). */
enum fv_patch {
    FV_PATCH_TAIL = 0, FV_PATCH_POINT = 1, FV_PATCH_BOTTOM = 2,
    FV_PATCH_RIGHT = 3, FV_PATCH_LEFT = 4, FV_PATCH_TOP = 5
};

/* Arithmetic of the step.  F64: everything in FP64.  F32_FLUX: reconstruction, EOS
 * closures and face fluxes in FP32; conserved variables stored and accumulated in FP64. */
enum fv_precision { FV_PREC_F64 = 0, FV_PREC_F32_FLUX = 1 };

/* Chemistry source (per cell, after the advection step; abstractChemicalKinetics::
 * solveChemicalKinetics, headers/abstractChemicalKinetics.hpp:618, called from
 * secondOrderStepSolver.cpp:86-91).
 *   CL2     Cl2 + M <-> 2Cl + M, species 0 = Cl2, 1 = Cl, third body M = total concentration
 *           (chemicalKineticsChlorumDissociation.cpp; set/chemicalKinetics.txt "Cl2").
 *   A_B_2C  A + B -> 2C, species 0 = A, 1 = B, 2 = C (no counterpart in the reference; the same
 *           integrator, heat release q per mol of reaction as in chemicalKineticsH2Cl2Combustion.cpp). */
enum fv_chemistry { FV_CHEM_NONE = 0, FV_CHEM_A_B_2C = 1, FV_CHEM_CL2 = 2 };

/* Step solver of #Approximation_order (abstractStepSolver::createStepSolver,
 * src/interfaces/abstractStepSolver.cpp:56-146).
 *   SECOND_ORDER     "SecondOrder": MUSCL-Hancock, one stage (secondOrderStepSolver.cpp).
 *   SECOND_ORDER_RK  "SecondOrderRK": two stages of the TVD reconstruction without the Hancock
 *                    predictor (Advection2dOrder.cpp), then the 0.5 average with the step's start
 *                    state (secondOrderStepSolverRK.cpp:48-71, bunchOfFields::average); the
 *                    averaged concentrations are part of the state.
 *   THIRD            "ThirdOrder": SSP-RK3 of three advections reconstructed with per-face limited
 *                    surface gradients (Advection3dOrder.cpp, templates/thirdOrderLimiter.hpp),
 *                    averages 0.25 and 2/3 with the start state (thirdOrderStepSolver.cpp:48-82).
 *   THIRD_CADA       "ThirdOrderCada": the ThirdOrder stages with the smoothness-switched limiter
 *                    of templates/thirdOrderLimiterCada.hpp (per face and field: unlimited where
 *                    the indicator eta of the face's and the farthest face's surface gradients is
 *                    below 1 - 1e-6, limited above 1 + 1e-6, blended in between;
 *                    thirdOrderStepSolverCada.cpp, Advection3dOrderCada.cpp).
 * The multi-stage solvers run on the generic path (SecondOrderRK also on the fused march); with a
 * chemical mechanism the chemistry pass follows the last average (secondOrderStepSolverRK.cpp:
 * 114-118, thirdOrderStepSolver.cpp:125-129).  They are not combined with the batched ensemble,
 * the adjoint or fv_step_noalloc. */
enum fv_step_solver { FV_ORDER_SECOND = 0, FV_ORDER_SECOND_RK = 1, FV_ORDER_THIRD = 2, FV_ORDER_THIRD_CADA = 3 };

/* Per-cell linear solver of the backward-Euler step (set/chemicalKinetics.txt #Iterative_solver:
 * "Gauss-Seidel", "Jacobi", "GaussElimination", "conjugateGradient", "JacobiConjugateGradient"). */
enum fv_chem_solver {
    FV_CHEM_GAUSS_SEIDEL = 0, FV_CHEM_JACOBI = 1, FV_CHEM_GAUSS_ELIMINATION = 2,
    FV_CHEM_CONJUGATE_GRADIENT = 3, FV_CHEM_JACOBI_CONJUGATE_GRADIENT = 4
};

/* Linear solver of the diffusion stage (#Type_of_SLE_solver_flag, abstractMatrixSolver.cpp:51-70):
 * "explicit" (the stage's fields advance explicitly, Diffusion.cpp:437-441,787-797,818-825),
 * "GaussSeidel" (GaussSeidelSolver.cpp), "Jacobi" (JacobiSolver.cpp), on 1D meshes "Thomas"
 * (ThomasSolver.cpp, the tridiagonal sweep), each solving the matrices of
 * SLEMatrix::generateDTimeLaplacian, or "noSolver" (noMatrixSolver.cpp: the stage takes the
 * implicit branch and every solve returns its start field), or the conjugate-gradient solvers
 * "conjugateGradient", "JacobiConjugateGradient" and "biConjugateGradient"
 * (conjugateGradientSolver.cpp, JacobiConjugateGradientSolver.cpp, biConjugateGradientSolver.cpp;
 * on the device their dot products are block sums, not the reference's serial order, and agree
 * with it to rounding). */
enum fv_sle_solver {
    FV_SLE_EXPLICIT = 0, FV_SLE_GAUSS_SEIDEL = 1, FV_SLE_JACOBI = 2, FV_SLE_THOMAS = 3, FV_SLE_NO_SOLVER = 4,
    FV_SLE_CG = 5, FV_SLE_JACOBI_CG = 6, FV_SLE_BICG = 7
};

/* Transport-coefficient model (transportCoefficients.txt #Transport_coefficient_model,
 * phaseInitialization.cpp:211-222, abstractTransportModel.cpp:37-80):
 *   CONSTANT        "constant": mu, D and kappa as given (abstractTransportModel.cpp:82-187);
 *   HARD_SPHERES    "hardSpheres": the constants plus the hard-sphere kinetic-theory values of
 *                   each species (transport_diameter, sub_k.txt #Kinetic_diameter_(A)), mixed by
 *                   Wilke's rule (hardSpheresTransportModel.cpp);
 *   LENNARD_JONES   "LennardJones": the same with the collision integrals of the Lennard-Jones
 *                   potential (transport_lj_eps, transport_lj_sigma: sub_k.txt
 *                   #Lennard_Jones_eps/kB_(K), #Lennard_Jones_sigma_(A);
 *                   LennardJonesTransportModel.cpp).
 * The coefficients of a face follow from its interpolated temperature and concentrations and the
 * Riemann star pressure; the cell viscosity of the viscous heating from the cell's
 * (Diffusion.cpp:130-132,238-240,506). */
enum fv_transport { FV_TRANSPORT_CONSTANT = 0, FV_TRANSPORT_HARD_SPHERES = 1, FV_TRANSPORT_LENNARD_JONES = 2 };

/* transportCoefficients.txt #Flag_for_enthalpy_flow_solution (phaseInitialization.cpp:224-235):
 * the species' enthalpy flow explicit in the temperature's free term and diagonal (with its
 * source time-step limit), or implicit as the upwind term of SLEMatrix::addNabla in the
 * temperature matrix (Diffusion.cpp:820-826; with the explicit solver the temperature stays). */
enum fv_enthalpy_flow { FV_ENTHALPY_NO = 0, FV_ENTHALPY_EXPLICIT = 1, FV_ENTHALPY_IMPLICIT = 2 };

/* Arrhenius rate constant k = A * T^n * exp(-E / (R T)), E in J/mol (R units of the case). */
typedef struct fv_arrhenius {
    double A, n, E;
} fv_arrhenius;

typedef struct fv_config {
    int dims;                 /* 1, 2 or 3 (#Dimensions_of_the_task) */
    int n[3];                 /* cells per direction (#Number_of_cells_in_direction) */
    double L[3];              /* parallelepiped radius-vector (#Radius-vector...); origin at 0 */
    int n_species;            /* 1..FV_MAX_SPECIES (#Number_of_components) */
    double R;                 /* universal gas constant value (SI / "1" / CGS / CGmS) */
    double M[FV_MAX_SPECIES];   /* molar masses (sub_k.txt #Molar_mass) */
    double Cv[FV_MAX_SPECIES];  /* molar isochoric heat capacities */
    double Tc[FV_MAX_SPECIES];  /* critical temperatures (van der Waals) */
    double Pc[FV_MAX_SPECIES];  /* critical pressures (van der Waals) */
    int eos;                  /* fv_eos */
    int flux;                 /* fv_flux */
    int limiter;              /* fv_limiter */
    int precision;            /* fv_precision */
    double courant;           /* #Courant_number */
    double min_timestep;      /* #Minimal_timestep (also the first time step) */
    int courant_only;         /* 1 when #Source_timestep_correction is "Courant" */
    int gravity;              /* g.txt #Free_fall_acceleration_flag */
    double g[3];              /* free-fall acceleration */
    double g_delta[3];        /* #Acceleration_growth (g += g_delta*dt after each step) */
    /* Boundary conditions per patch (fv_patch) and per field. */
    int bc_conc[6][FV_MAX_SPECIES];
    double bc_conc_value[6][FV_MAX_SPECIES];
    int bc_vel[6];
    double bc_vel_value[6][3];
    int bc_p[6];
    double bc_p_value[6];
    /* Chemistry (set/chemicalKinetics.txt). */
    int chemistry;            /* fv_chemistry */
    fv_arrhenius chem_forward;  /* A_B_2C: the reaction; CL2: dissociation (#A_forw #n_forw #E_forw) */
    fv_arrhenius chem_backward; /* CL2: recombination (#A_backw #n_backw #E_backw) */
    double chem_q;            /* A_B_2C: heat release per mol of reaction (J/mol, > 0 exothermic) */
    int chem_solver;          /* fv_chem_solver */
    int chem_max_iter;        /* #Number_of_chemical_solver_iterations */
    /* #Constant_timestep: > 0 fixes every step to this dt (main then skips its CFL block,
     * Schemi.cpp:178-181,664-668,807); <= 0 keeps the CFL step. */
    double const_timestep;
    /* #Approximation_order: the step solver (fv_step_solver). */
    int order;
    /* Equation-of-state data beyond M, Cv, Tc and Pc (ABI version 5). */
    double stiff_p0[FV_MAX_SPECIES];     /* STIFFENED: p0 of each species */
    double stiff_gamma[FV_MAX_SPECIES];  /* STIFFENED: gamma of each species */
    double lj_eps[FV_MAX_SPECIES];       /* KATAOKA: Lennard-Jones epsilon of each species */
    double lj_sigma[FV_MAX_SPECIES];     /* KATAOKA: Lennard-Jones sigma of each species */
    int kataoka_b_critical;              /* KATAOKA: 1 "critical": b = coeff R Tc / (8 Pc);
                                            0 "Kataoka": b = coeff sigma^3 N_A */
    double kataoka_b_coeff;
    /* Diffusion stage (ABI version 6): #Diffusion_flag on runs Diffusion.cpp:20-1061 after each
     * advection (secondOrderStepSolver.cpp:69-80), with the gas's molecular transport and no
     * turbulence. */
    int diffusion;            /* 1: #Diffusion_flag on */
    int sle_solver;           /* fv_sle_solver */
    int sle_max_iter;         /* #Number_of_iterations_of_SLE_matrix_solver */
    int transport;            /* fv_transport */
    double mu_const;          /* #Viscosity_coefficient (the constant model's mu) */
    double D_const;           /* #Diffusion_coefficient */
    double kappa_const;       /* #Heat_conduction_coefficient */
    int enthalpy_flow;        /* fv_enthalpy_flow */
    int molmass_diffusion;    /* #Flag_for_molar_mass_diffusion_correction on */
    int linear_reconstruction;  /* #Reconstruction "linear" (1) or "star" (0): the stage's velocity
                                   gradient from the cells or from the Riemann star states */
    int diffusion_timestep;   /* 1: #Source_timestep_correction "Courant-Source-Diffusion" (the
                                 stage limits the next step, Diffusion.cpp:1036-1049) */
    double dt_coeff_source;   /* the flag's first coefficient (explicit enthalpy flow limit) */
    double dt_coeff_diffusion;  /* its second (diffusion limit) */
    /* Species data of the transport models (ABI version 7). */
    double transport_diameter[FV_MAX_SPECIES];  /* HARD_SPHERES: kinetic diameter (angstrom) */
    double transport_lj_eps[FV_MAX_SPECIES];    /* LENNARD_JONES: eps / k_B (K) */
    double transport_lj_sigma[FV_MAX_SPECIES];  /* LENNARD_JONES: sigma (angstrom) */
} fv_config;

/* Field indices of fv_download / fv_upload arrays (n_cells doubles each, x fastest).
 * Upload takes the restart set: c_1..c_N, v_x, v_y, v_z, p  (N+4 arrays). */
enum fv_field {
    FV_F_CONC = 0,            /* c_1..c_N occupy FV_F_CONC + k */
    FV_F_VX = FV_MAX_SPECIES, FV_F_VY, FV_F_VZ, FV_F_P,
    FV_F_RHO_K,               /* rho_1..rho_N occupy FV_F_RHO_K + k */
    FV_F_RHO = FV_F_RHO_K + FV_MAX_SPECIES,
    FV_F_MX, FV_F_MY, FV_F_MZ, FV_F_E, FV_F_UV, FV_F_T, FV_F_SONIC,
    FV_F_CONC0,               /* total concentration c_0 as the state holds it: after a SecondOrderRK,
                                 ThirdOrder or ThirdOrderCada step the averaged field
                                 (bunchOfFields::average), which can differ from the sum of c_1..c_N in
                                 the last bit; otherwise that sum (ABI version 4) */
    FV_F_COUNT
};

typedef struct fv_handle fv_handle;

typedef struct fv_run_stats {
    double time;              /* simulated time reached */
    double dt_next;           /* time step that would be used next */
    long long steps;          /* steps taken in this call */
    float device_ms;          /* device time of the call (CUDA events on the handle's stream) */
} fv_run_stats;

int fv_abi_version(void);

/* Validates cfg, builds geometry tables and allocates device memory on the current device. */
fv_status fv_create(const fv_config* cfg, fv_handle** out);
void fv_destroy(fv_handle* h);
const char* fv_last_error(const fv_handle* h);

/* Host arrays (n_cells each): c_1..c_N, v_x, v_y, v_z, p.  Derives rho_k, rho, m, E as
 * phaseInitialization.cpp:1827-1885 does, and sets time = 0, dt = min_timestep. */
fv_status fv_upload(fv_handle* h, const double* const* prim);

/* Same, from device pointers (no host copy). */
fv_status fv_upload_device(fv_handle* h, const double* const* prim_dev);

/* One step with the handle's current dt (first call: min_timestep), then the CFL block:
 * dt_next = max(min(Courant / max_i((|v_i| + c_i) / minEdge_i), dtSource), minTimestep).
 * Writes the dt used and the new dt.  No clamp to an end time. */
fv_status fv_step(fv_handle* h, double* dt_used, double* dt_next);

/* Runs main's time loop on the device until time >= t_end (or max_steps), with the
 * last-step clamp dt = t_end - time.  Steps are launched in CUDA-graph chunks; the host
 * synchronises once per chunk. */
fv_status fv_run(fv_handle* h, double t_end, long long max_steps, fv_run_stats* stats);

/* Output set (fv_field order).  out[f] may be NULL to skip field f. */
fv_status fv_download(fv_handle* h, double* const* out);

/* Time and time step held by the handle. */
fv_status fv_get_time(const fv_handle* h, double* time, double* dt);
fv_status fv_set_time(fv_handle* h, double time, double dt);

/* The source time step the last step's diffusion stage set (mesh::timestepSource after
 * Diffusion.cpp:688-706,1036-1049; 1e-3 * DBL_MAX, the reference's veryBig, when no stage
 * limited it): the limit main's CFL block applies to the next step unless #Source_timestep_correction
 * is "Courant".  A host that runs its own CFL block (the step-solver adapter) hands it on. */
fv_status fv_get_source_timestep(const fv_handle* h, double* dt_source);

/* Conserved state (rho_1..rho_N, rho, m_x, m_y, m_z, E) as device pointers, SoA, n_cells each.
 * A 1D/2D case whose restart set has no transverse velocity leaves the transverse momentum
 * fields untouched (they stay zero).  The arrays are for reading: the step keeps data derived
 * from the current state between steps, so a new state goes in through fv_upload or
 * fv_upload_device. */
fv_status fv_state_device(fv_handle* h, double** fields, int* n_fields, long long* n_cells);

/* Synchronises the handle's stream. */
fv_status fv_sync(fv_handle* h);

/* Asynchronous stepping for callers that keep the host off the step's critical path:
 * fv_begin_steps puts the clock in single-step mode (no end-time clamp); fv_step_async enqueues
 * one step + CFL on the handle's stream without synchronising or reading anything back;
 * fv_check synchronises and reports a device-side error raised by any enqueued step. */
fv_status fv_begin_steps(fv_handle* h);
fv_status fv_step_async(fv_handle* h);
fv_status fv_check(fv_handle* h);

/* The handle's CUDA stream (cudaStream_t), for event timing and interop. */
void* fv_stream(fv_handle* h);

/* Kernel launches one step issues (the fused march: 1, the generic path: 4, each finalizing the
 * CFL block in its last CTA; more with chemistry, a diffusion stage or a multi-stage step). */
long long fv_kernels_per_step(const fv_handle* h);

/* ---- One step that allocates no device memory (no counterpart in the reference) ----
 * For hosts that cannot call cudaMalloc on the step's path: an application whose device memory
 * belongs to a pooling allocator that forbids driver allocations, or a time loop that cannot
 * afford the device-wide synchronisation cudaMalloc / cudaFree may cause.  The caller owns the
 * state buffers; all intermediates live in one file-scope device array of
 * FV_NOALLOC_SCRATCH_BYTES (2.5 MiB) that every GPU which loads the library keeps until exit.
 *   state_in / state_out  device arrays, (n_species + 5) fields x n_cells, the layout of
 *                          fv_state_device (rho_1..rho_N, rho, m_x, m_y, m_z, E; x fastest)
 *   dt                     step to take; dt_next receives main's CFL step of the new state
 *                          (unclamped); cfg->g is the gravity vector of this step
 *   stream                 cudaStream_t or NULL
 * Runs the full MUSCL-Hancock path of the SecondOrder step solver (any limiter, 1D/2D/3D, both
 * precisions) on meshes of at most FV_NOALLOC_MAX_CELLS cells.  Rejected with FV_ERR_INIT: every
 * configuration fv_create rejects, larger meshes, cases with chemistry, the SecondOrderRK,
 * ThirdOrder and ThirdOrderCada step solvers, the diffusion stage, and state_in / state_out arrays
 * that overlap.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress).  Every call rewrites each part of the array it reads, so no state
 * carries over between calls; calls that overlap on the GPU share the array and race.  The call
 * synchronises `stream` before returning (it reads the new time step back), so it cannot be
 * captured in a CUDA graph. */
#define FV_NOALLOC_MAX_CELLS 1024
#define FV_NOALLOC_SCRATCH_BYTES 2621440
fv_status fv_step_noalloc(const fv_config* cfg, const double* state_in, double* state_out, double dt,
                          double* dt_next, void* stream);

/* ---- Batched ensemble: many independent cases advanced by one persistent kernel ---- */
typedef struct fv_batch fv_batch;

typedef struct fv_batch_stats {
    long long cell_updates;   /* sum over cases of cells x steps */
    long long steps_max;      /* largest step count of any case */
    long long launches;       /* kernel launches issued */
    float device_ms;          /* device time of the run */
} fv_batch_stats;

/* All handles must share dims, n_species, eos, flux, limiter and precision. */
fv_status fv_batch_create(fv_handle* const* cases, int n_cases, fv_batch** out);
fv_status fv_batch_run(fv_batch* b, const double* t_end, long long max_steps, fv_batch_stats* stats);
void fv_batch_destroy(fv_batch* b);

/* ---- Adjoint of the step (no counterpart in the reference: it has no adjoint) ----
 * Differentiates the zero-slope multi-dimensional step -- the fused march, i.e. 2D/3D with a
 * limiter whose multi-dimensional slopes are zero, ideal-gas mixtures -- with every step's dt
 * and gravity vector frozen at the recorded values.
 *
 * fv_record runs the time loop of fv_run from the handle's current state to t_end, stores the
 * state every `checkpoint_every` steps on the device, records each step's dt and gravity, and
 * accumulates the objective J = sum_{n=1..N} dt_{n-1} W(U^n) with the mixing width
 * W = 4 / (L_x [L_z in 3D]) * sum_cells X_h (1 - X_h) * (cell area in 2D, cell volume in 3D),
 * X_h the mole fraction of species `heavy_species`.
 * fv_replay runs the recorded number of steps again from the handle's current state with the
 * recorded dt and gravity of each step (e.g. after uploading a perturbed initial state).
 * fv_adjoint sweeps the recorded trajectory backwards, recomputing the states between
 * checkpoints, and returns dJtot/dU^0 for Jtot = dJ_dJ * J + <dJ_dU_T, U^N>.
 * All state arrays are device pointers in the fv_state_device layout
 * ((n_species + 5) fields x n_cells, rho_1..rho_N, rho, m_x, m_y, m_z, E; x fastest).
 * dJ_dU_T may be NULL (zero). */
enum fv_objective { FV_OBJ_NONE = 0, FV_OBJ_MIXING_WIDTH = 1 };

typedef struct fv_record_config {
    int checkpoint_every;     /* steps between stored states (>= 1) */
    int objective;            /* fv_objective */
    int heavy_species;        /* 0-based species index of X_h */
    int pad;
} fv_record_config;

typedef struct fv_record_stats {
    double objective;         /* J */
    double time;              /* time reached */
    long long steps;          /* N */
    long long checkpoints;    /* stored states */
    float device_ms;
} fv_record_stats;

typedef struct fv_adjoint_stats {
    long long steps;          /* adjoint steps (= N) */
    long long recomputed;     /* forward steps recomputed from checkpoints */
    float device_ms;          /* whole sweep incl. recomputation */
    float recompute_ms;       /* recomputation share */
} fv_adjoint_stats;

fv_status fv_record(fv_handle* h, const fv_record_config* rc, double t_end, long long max_steps,
                    fv_record_stats* stats);
fv_status fv_replay(fv_handle* h, fv_record_stats* stats);
fv_status fv_adjoint(fv_handle* h, const double* dJ_dU_T, double dJ_dJ, double* dJ_dU_0, fv_adjoint_stats* stats);

/* Copies the handle's conserved state (fv_state_device layout) to the device array dst. */
fv_status fv_state_copy(fv_handle* h, double* dst);

#ifdef __cplusplus
}
#endif

#endif /* SCHEMI_B200_FVSTEP_H_ */
