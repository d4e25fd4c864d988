/*
 * philip_b200 — C-ABI of the B200 explicit strong-form DG/FR residual and RK stage.
 *
 * Plain C types only (pointers, sizes, scalars); no exceptions cross this boundary.
 * Every entry point returns 0 on success or a PH_ERR_* code; ph_last_error() gives
 * the message of the calling thread's last failure.
 *
 * State layout (the reference's DoF order with do_renumber_dofs=false): cell-major in
 * deal.II active-cell order, then conservative component (rho, rho u, rho v, rho w, E),
 * then the (p+1)^3 GLL support points lexicographically with x fastest
 * (local dof = istate*n_shape + ishape, src/dg/strong_dg.cpp:142-147).
 *
 * Thread-safety: one context per host thread; a context is bound to one CUDA stream.
 */
#ifndef PHILIP_B200_H
#define PHILIP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ph_ctx ph_ctx;

enum {
    PH_OK = 0,
    PH_ERR_INVALID = 1,      /* bad argument */
    PH_ERR_UNSUPPORTED = 2,  /* configuration outside the GPU path (e.g. overintegration 3, p = 7) */
    PH_ERR_CUDA = 3,         /* CUDA runtime failure */
    PH_ERR_NOMEM = 4,        /* device allocation failed */
    PH_ERR_EXCHANGE = 5      /* the halo exchange callback of a slab context failed */
};

enum { PH_HOST = 0, PH_DEVICE = 1 };                 /* where a pointer lives */
enum { PH_FP64 = 0, PH_FP32_RESIDUAL = 1 };          /* arithmetic of the residual */

/* .prm keys of the hot path (src/parameters/all_parameters.cpp:39-400,
 * parameters_ode_solver.cpp, parameters_euler.cpp, parameters_navier_stokes.cpp).
 * Enumerations use the reference's spelling order:
 *   flux_nodes_type: 0 GL, 1 GLL            pde_type: 0 euler, 1 navier_stokes
 *   two_point_num_flux_type: 0 KG, 1 IR, 2 CH, 3 Ra
 *   conv_num_flux: 0 lax_friedrichs, 1 roe, 2 central_flux, 3 two_point_flux,
 *                  4 two_point_flux_with_lax_friedrichs_dissipation,
 *                  5 two_point_flux_with_roe_dissipation
 *   diss_num_flux: 0 symm_internal_penalty, 1 bassi_rebay_2, 2 central_visc_flux
 *   flux_reconstruction: 0 cDG, 1 cSD, 2 cHU, 3 cNegative, 4 cNegative2, 5 cPlus,
 *                        6 c10Thousand, 7 cHULumped, 8 user_specified_value
 *   flux_reconstruction_aux: 0 kDG, 1 kSD, 2 kHU, 3 kNegative, 4 kNegative2, 5 kPlus (p = 2..5),
 *                            6 k10Thousand
 *   runge_kutta_method: 0 rk4_ex, 1 ssprk3_ex, 2 heun2_ex, 3 euler_ex (4-6 implicit: not on this path),
 *                       7 RK4_3_5_3SStar, 8 RK3_2_5F_3SStarPlus, 9 RK4_3_9F_3SStarPlus,
 *                       10 RK5_4_10F_3SStarPlus (low-storage, with an embedded error estimate)
 *   non_physical_behavior: 0 return_big_number, 1 abort_run, 2 print_warning */
typedef struct ph_params {
    int poly_degree;
    int overintegration;
    int flux_nodes_type;
    int pde_type;
    int use_split_form;
    int two_point_num_flux_type;
    int conv_num_flux;
    int diss_num_flux;
    int flux_reconstruction;
    int flux_reconstruction_aux;
    int runge_kutta_method;
    int use_constant_viscosity;
    int non_physical_behavior;
    int precision;                        /* PH_FP64 or PH_FP32_RESIDUAL */
    double FR_user_specified_correction_parameter_value;
    double gamma_gas;
    double mach_infinity;
    double reynolds_number_inf;
    double prandtl_number;
    double temperature_inf;
    double nondimensionalized_constant_viscosity;
    double sipg_penalty_factor;
    double rk_atol;                       /* low-storage RK error estimate: absolute and relative */
    double rk_rtol;                       /* tolerances (ODE solver atol / rtol) */
    /* Precision form only (no counterpart in the reference's parameters): a constant reference
     * pressure subtracted from the pressure in every momentum flux. A constant pressure adds
     * the same amount to the volume and the face terms, which cancel, so the residual is
     * unchanged in exact arithmetic; in FP32 the mean pressure of a low-Mach flow
     * (1/(gamma M^2) in the Taylor-Green scaling, 1/gamma in the isentropic vortex's) would
     * otherwise swamp its O(1) variations. 0 = no shift. Ignored by the FP64 path. */
    double pressure_shift;
    /* Relaxation Runge-Kutta, root-finding form for the Euler / Navier-Stokes entropy
     * (ODE solver/rrk root solver: use_relaxation_runge_kutta, relaxation_runge_kutta_root_tolerance;
     * src/ode_solver/relaxation_runge_kutta/root_finding_rrk_ode_solver.cpp). The Butcher methods
     * in FP64, two-point fluxes other than KG; GLL or GL flux nodes, with or without
     * overintegration (off the solution nodes the entropy is integrated at the flux nodes and the
     * estimate takes the entropy variables projected on the solution basis). */
    int use_relaxation_runge_kutta;
    double relaxation_runge_kutta_root_tolerance;
    /* limiter/bound_preserving_limiter (src/parameters/parameters_limiter.cpp:17-30):
     * 0 none, 1 maximum_principle (scalar equations: not on this path),
     * 2 positivity_preservingZhang2010, 3 positivity_preservingWang2012; and limiter/min_density.
     * A positivity limiter is applied to every RK stage solution and to the new solution
     * (Butcher methods), and with it the non-physical replacement of negative densities and
     * pressures is off, as in the reference (Euler::check_positive_quantity). */
    int bound_preserving_limiter;
    double min_density;
    /* Boundary conditions of a non-periodic mesh (ph_mesh_desc.boundary_type):
     * euler/angle_of_attack and side_slip_angle in degrees (the free stream of the farfield,
     * Riemann and inflow conditions, velocities (cos a cos b, sin a cos b, sin b); the side slip
     * must be 0, Euler::Euler, src/physics/euler.cpp:14-70), navier_stokes/
     * thermal_boundary_condition_type (0 adiabatic, 1 isothermal) and
     * nondimensionalized_isothermal_wall_temperature of the no-slip wall
     * (src/parameters/parameters_navier_stokes.cpp:21-50; the .prm default is 1.0). */
    double angle_of_attack;
    double side_slip_angle;
    int thermal_boundary_condition_type;
    double isothermal_wall_temperature;
    /* use_projected_entropy_variables_for_nsfr_boundary_term (all_parameters.cpp:399; default 0):
     * the split form's boundary states and convective boundary flux take the face state of the
     * projected entropy variables instead of the interpolated solution (strong_dg.cpp:2255-2273).
     * On collocated GLL nodes the two agree to rounding. */
    int use_projected_entropy_variables_for_nsfr_boundary_term;
} ph_params;

/* Periodic cube [left,right]^3 with n^3 cells (PeriodicCubeFlow::generate_grid,
 * src/flow_solver/flow_solver_cases/periodic_cube_flow.cpp:25-65). cell_order:
 * 0 = as deal.II numbers it (recursive children when n is a power of two,
 * lexicographic otherwise), 1 = lexicographic, 2 = recursive children. */
typedef struct ph_mesh_desc {
    int n_cells_per_direction;
    int cell_order;
    double left;
    double right;
    /* Curvilinear cube when warp != 0: every coordinate of the straight-sided mesh is moved
     * by warp (L/2pi) sin(2pi(x-l)/L) sin(2pi(y-l)/L) sin(2pi(z-l)/L) (L = right - left,
     * l = left; zero on the cube's faces, so periodic faces still match), through a mapping
     * of degree grid_degree on GLL support points. The GPU path takes grid_degree =
     * poly_degree; split or conservative, any FR type (the weight-adjusted inverse mass);
     * GLL or GL flux nodes, overintegration 0..2; Navier-Stokes with bassi_rebay_2 or
     * central_visc_flux (and, on collocated GLL nodes, flux_reconstruction_aux = kDG).
     * Not a reference grid:
     * the construction follows the reference's curved periodic grids
     * (src/mesh/grids/curved_periodic_grid.cpp) with this warp. */
    double warp;
    int grid_degree;
    /* Optional: physical coordinates of every cell's mapping support points, [cell][3][(p+1)^3]
     * (GLL points, x fastest, cells in the state's order). When set, the mesh is curvilinear
     * with this mapping (any curved periodic grid, e.g. the reference's curved_periodic_grid
     * or nonsymmetric_curved_periodic_grid with grid_degree = poly_degree) and warp is
     * ignored. The caller keeps the array alive during ph_ctx_create / ph_batch_admit. */
    const double* mapping_support_points;
    /* Boundary condition of each side x-, x+, y-, y+, z-, z+: 0 = periodic (a pair of sides is
     * periodic on both sides or on neither), else the boundary_id its faces carry
     * (Euler::boundary_face_values, src/physics/euler.cpp:1508-1560): 1001 wall (Euler: slip;
     * Navier-Stokes: no-slip, adiabatic or isothermal), 1002 pressure outflow, 1003 inflow,
     * 1004 Riemann farfield, 1005 farfield, 1006 slip wall, 1007 extrapolation. Navier-Stokes
     * takes 1001 and 1006 (NavierStokes::boundary_face_values_viscous_flux defines no viscous
     * exterior state for the others). Contexts (ph_ctx_create), affine or curvilinear, GLL or GL
     * flux nodes, overintegration 0..2; as a flow case's grid sets boundary ids, e.g.
     * channel_flow.cpp:324-343. */
    int boundary_type[6];
} ph_mesh_desc;

/* Builds host index maps, 1-D operators and device buffers (replaces DGFactory::
 * create_discontinuous_galerkin + DGBase::allocate_system, src/dg/dg_factory.cpp:11,
 * src/dg/dg_base.hpp:184, and ODESolverFactory::create_ODESolver + allocate_ode_system,
 * src/ode_solver/ode_solver_factory.cpp:22, ode_solver_base.h:79).
 * cuda_stream may be NULL (the default stream). */
int ph_ctx_create(const ph_mesh_desc* mesh, const ph_params* prm, void* cuda_stream, ph_ctx** out);
int ph_ctx_destroy(ph_ctx* ctx);

int64_t ph_ndofs(const ph_ctx* ctx);
/* Physical coordinates of the solution nodes, [cell][node][3] in the state's cell and node
 * order (the points VectorTools::interpolate evaluates an initial condition at,
 * src/solution/set_initial_condition.cpp:51). */
int ph_node_xyz(const ph_ctx* ctx, double* xyz);
int ph_cell_ijk(const ph_ctx* ctx, int32_t* ijk /* 3 per cell */);

/* DGBase::solution assignment / read-back (src/dg/dg_base.hpp:396). */
int ph_set_state(ph_ctx* ctx, const double* U, int where);
int ph_get_state(ph_ctx* ctx, double* U, int where);

/* DGBase::assemble_residual (src/dg/dg_base.hpp:571, dg_base.cpp:2599-2915): R(U),
 * the right-hand side before the inverse mass matrix, in the reference DoF order. */
int ph_residual(ph_ctx* ctx, const double* U, double* R, int where);

/* DGBase::apply_inverse_global_mass_matrix (src/dg/dg_base.hpp:267, dg_base.cpp:4089-4260). */
int ph_apply_inverse_mass(ph_ctx* ctx, const double* R, double* out, int where);

/* ODESolverBase::step_in_time for the explicit Butcher RK solver
 * (src/ode_solver/ode_solver_base.h:70, runge_kutta_base.cpp:21-39), nsteps times
 * with the same dt, on the context's state. Asynchronous on the context stream. */
int ph_rk_step(ph_ctx* ctx, double dt, int nsteps);

/* Relaxation RK: the relaxation parameter gamma of the last step (RRKODESolverBase::
 * update_relaxation_parameter, rrk_ode_solver_base.cpp:13-33) and the time the state advanced
 * over the last ph_rk_step call, sum over its steps of gamma dt (RungeKuttaODESolver::
 * adjust_time_step, runge_kutta_ode_solver.cpp:102-110). gamma = 1 and elapsed = nsteps dt
 * without relaxation. */
int ph_rk_relaxation(ph_ctx* ctx, double* gamma, double* elapsed);

/* Weighted RMS error estimate of the last low-storage RK step,
 * sqrt(mean(((S1 - S_embedded) / (atol + rtol max(|S1|, |S_embedded|)))^2)) over all DOFs
 * (LowStorageRungeKuttaODESolver::get_automatic_error_adaptive_step_size,
 * src/ode_solver/low_storage_runge_kutta_ode_solver.cpp:80-110, before the step-size
 * controller). Synchronises the context stream. */
int ph_rk_error_norm(ph_ctx* ctx, double* w);

/* PeriodicTurbulence::compute_and_update_integrated_quantities subset
 * (src/flow_solver/flow_solver_cases/periodic_turbulence.cpp:439-672):
 * out[0] kinetic energy, out[1] enstrophy, out[2] vorticity-based dissipation rate
 * (2 enstrophy / Re; zero for the Euler equations),
 * out[3] maximum convective wave speed; all divided by the domain volume except out[3]. */
int ph_integrals(ph_ctx* ctx, double out[4]);

/* All nine integrated quantities of PeriodicTurbulence::compute_and_update_integrated_quantities
 * (periodic_turbulence.cpp:439-672), in the order of its IntegratedQuantitiesEnum
 * (periodic_turbulence.h:176-186), each divided by the domain volume. The integrands are the
 * NavierStokes physics' whatever the PDE (navier_stokes.cpp:399-740, euler.cpp:378-402); the
 * palinstrophy differentiates the vorticity after its L2 projection onto the solution basis;
 * the angular momentum (0.5 |x|^2 |omega|) is always computed, where the reference computes it
 * only under do_compute_angular_momentum. Derived rates, as the reference forms them:
 * pressure-dilatation-based dissipation = -out[2]; deviatoric / strain-rate based =
 * 2 out[3] / Re and 2 out[4] / Re (zero for the Euler equations). */
enum {
    PH_IQ_KINETIC_ENERGY = 0,
    PH_IQ_ENSTROPHY = 1,
    PH_IQ_PRESSURE_DILATATION = 2,
    PH_IQ_VISCOSITY_TIMES_DEVIATORIC_STRAIN_RATE_SQR = 3,
    PH_IQ_VISCOSITY_TIMES_STRAIN_RATE_SQR = 4,
    PH_IQ_INCOMPRESSIBLE_KINETIC_ENERGY = 5,
    PH_IQ_INCOMPRESSIBLE_ENSTROPHY = 6,
    PH_IQ_INCOMPRESSIBLE_PALINSTROPHY = 7,
    PH_IQ_ANGULAR_MOMENTUM = 8,
    PH_N_INTEGRATED_QUANTITIES = 9
};
int ph_integrated_quantities(ph_ctx* ctx, double out[PH_N_INTEGRATED_QUANTITIES]);

/* The time loop of FlowSolver::run (src/flow_solver/flow_solver.cpp:540-620) with the
 * periodic-turbulence unsteady data (PeriodicTurbulence::compute_unsteady_data_and_write_to_table,
 * periodic_turbulence.cpp:923-972) on the device: nsteps steps of dt as ph_rk_step takes
 * them; after every record_every-th step the four values of ph_integrals are reduced on the
 * device into a table, which is copied once, at the end, to rows (nsteps / record_every
 * rows of 4 doubles: kinetic energy, enstrophy, vorticity-based dissipation rate, max wave
 * speed). record_every = 0 records nothing. On a caller-given stream each record interval
 * replays one captured graph (steps, integrals, row). Synchronises the context stream. */
int ph_run(ph_ctx* ctx, double dt, int nsteps, int record_every, double* rows);

/* Status word: bit 0 = a negative density or pressure was met (Euler::check_positive_quantity,
 * src/physics/euler.cpp:155-172); bit 1 = a bulk copy into shared memory did not complete within
 * a kernel's wait limit (that launch's outputs were not written). Reading clears it. */
int ph_status(ph_ctx* ctx, uint32_t* flags);

/* Rate of change of the volume-averaged kinetic energy at the current solution,
 * dKE/dt = (1/|Omega|) integral of (v . dm/dt - |v|^2/2 drho/dt) with dU/dt = M^-1 R(U) evaluated
 * by the residual kernel of the context's precision and the QGauss(p+11) cubature of the kinetic
 * energy (periodic_turbulence.cpp:439-672). No counterpart in the reference, whose dissipation
 * rates come from the enstrophy and strain integrals; this one measures the precision form's
 * kinetic-energy dissipation directly. Whole affine meshes. Synchronises the context stream. */
int ph_kinetic_energy_rate(ph_ctx* ctx, double* out);

/* PositivityPreservingLimiter::limit (src/limiter/positivity_preserving_limiter.cpp:381-678) on the
 * context's solution for a stage of time step dt, as set_initial_condition.cpp:56 applies it to
 * an initial condition. Requires bound_preserving_limiter 2 or 3. */
int ph_limit(ph_ctx* ctx, double dt);

/* Measurement hooks (no counterpart in the reference, which times with dealii::Timer,
 * src/flow_solver/flow_solver.cpp:690-711). enable = 1: every kernel launch is bracketed
 * by CUDA events on the context stream and the stream is synchronised after it (steps
 * launch directly). enable = 2: the captured RK step that ph_rk_step replays carries an
 * event-record node before its first kernel and after each kernel, on a side branch of the
 * graph that the kernels do not wait for, and every replay records a fresh set of events, so
 * the kernels are timed inside the replayed steps themselves (each duration includes the
 * launch gap before the kernel); changing to or
 * from mode 2 drops the captured step, which the next multi-step ph_rk_step captures
 * again (its first step runs directly and is not timed). Every call resets the sums.
 * out[0..5] = {stage-kernel ms, stage launches, auxiliary-kernel ms, auxiliary
 * launches, other ms, other launches}, out[6] = kernel launches counted since the last
 * ph_set_timing call (counted with timing enabled or not). */
int ph_set_timing(ph_ctx* ctx, int enable);
int ph_get_timing(ph_ctx* ctx, double out[7]);

/* ---- One mesh over several GPUs: slabs of cell layers and a halo exchange ----
 * The reference distributes the triangulation over MPI ranks and refreshes the ghost values
 * of the solution before every residual (DGBase::assemble_residual, src/dg/dg_base.cpp:2742)
 * and of the auxiliary solution before the viscous face terms (src/dg/strong_dg.cpp:648).
 * Here a rank owns the cell layers z_first .. z_first + z_count - 1 (periodically) of the
 * affine periodic cube and keeps one ghost layer below and one above. Before each residual
 * evaluation the library packs, for each partition face, only what the neighbour's kernels
 * read: the state at the face nodes (5 (p+1)^2 doubles per cell) and, for Navier-Stokes, after
 * the auxiliary kernel, the face-normal viscous flux (4 (p+1)^2 values per cell in the
 * arithmetic type). The transfer itself is the caller's (NCCL, CUDA-aware MPI, peer copies),
 * through the callback below; the cells that read no ghost data are computed while the
 * transfer is in flight.
 *
 * Owned cells are numbered lexicographically (x fastest, then y, then z from z_first; see
 * ph_cell_ijk), whatever mesh->cell_order says; the state, ph_ndofs and the integrals cover
 * the owned cells only (ph_integrals / ph_integrated_quantities give this rank's share of
 * each volume average: sum them over ranks, and take the max of the wave speed). Slab
 * contexts launch directly (no step graph, ph_run refused); with relaxation RK they need
 * ph_set_rank_sum; on a curvilinear mesh mapping_support_points, when given,
 * covers the slab's own cells in the slab's state order. z_count = n is the whole mesh on one rank: its ghost layers are its own last
 * and first layers (a halo that copies send_hi to recv_lo and send_lo to recv_hi). */
enum { PH_HALO_STATE = 0, PH_HALO_VISCOUS = 1 };   /* what is exchanged */
enum { PH_HALO_BEGIN = 0, PH_HALO_END = 1 };        /* phase of the exchange */

/* Called twice per exchange, on the host thread that called the library:
 *   phase PH_HALO_BEGIN: send_lo (the first owned layer's data, for the rank that owns the layer
 *     below) and send_hi (the last layer's, for the rank above) are packed in stream order on
 *     cuda_stream; the callback starts the transfer of send_lo to the rank below and of send_hi to
 *     the rank above, and the receipt into recv_lo (from the rank below, its send_hi) and recv_hi
 *     (from the rank above, its send_lo). Ordered after the packing (e.g. NCCL send/recv enqueued
 *     on, or made to wait on, cuda_stream). With two ranks the rank below and above are the same:
 *     deliver the downward pair (send_lo -> recv_hi) before the upward pair.
 *   phase PH_HALO_END: the receive buffers must be complete in cuda_stream order when it returns
 *     (a stream wait on the transfer, or a synchronous copy), and the send buffers free for reuse.
 * bytes: the size of each of the four buffers (device memory, the library's). A nonzero return
 * fails the calling entry point with PH_ERR_EXCHANGE. */
typedef int (*ph_halo_fn)(void* user, int what, int phase, const void* send_lo, const void* send_hi,
                          void* recv_lo, void* recv_hi, size_t bytes, void* cuda_stream);

/* A context for the slab z_first .. z_first + z_count - 1 of mesh (1 <= z_count <= n). */
int ph_ctx_create_slab(const ph_mesh_desc* mesh, const ph_params* prm, int z_first, int z_count,
                       void* cuda_stream, ph_ctx** out);
/* Registers the exchange; every slab context needs one before it evaluates a residual. */
int ph_set_halo_exchange(ph_ctx* ctx, ph_halo_fn fn, void* user);
/* Sum over the ranks of one mesh, for relaxation RK on slab contexts (the root of the
 * relaxation parameter needs the mesh's entropy integrals, RootFindingRRKODESolver,
 * root_finding_rrk_ode_solver.cpp:15-180, where the reference's MPI vector reductions give
 * them): on the host thread that called the library, replace values[0..count-1] by their sum
 * over every rank's values, the same result on every rank (an all-reduce). Every rank makes
 * the same calls in the same order. A nonzero return fails the calling entry point with
 * PH_ERR_EXCHANGE. */
typedef int (*ph_rank_sum_fn)(void* user, double* values, int count);
/* Registers the sum; a slab context with relaxation RK needs one before its first step. */
int ph_set_rank_sum(ph_ctx* ctx, ph_rank_sum_fn fn, void* user);
/* Host only (no device work): the owned cells' (i, j, k) [z_count n^2][3] and neighbour table
 * [z_count n^2][6] (faces x-, x+, y-, y+, z-, z+) of a slab. A neighbour index below z_count n^2
 * is an owned cell; z_count n^2 + j n + i is the lower ghost (the cell (i, j) of layer
 * z_first - 1, filled from the rank below), z_count n^2 + n^2 + j n + i the upper ghost. */
int ph_slab_connectivity(int n, int z_first, int z_count, int32_t* ijk, int32_t* nbr);

/* R(U) as ph_residual computes it, on caller-owned DEVICE buffers U and R, without a
 * context and without allocating device memory. No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc (loops that must not synchronise the
 * device, or a framework that owns all device memory). U and R need no initialisation
 * beyond U's values. Its scratch lives in fixed file-scope device arrays: at most 32768 cells, and
 * for Navier-Stokes at most cells x (4 (p+1)^3 + 24 (p+1)^2) <= 4 Mi doubles of viscous-term scratch
 * (32 MiB); larger meshes are rejected with PH_ERR_INVALID. The mesh and parameters pass the
 * checks of ph_ctx_create before anything is launched. The first call on a device
 * resolves the arrays' device addresses and should come before any stream capture.
 * Every call shares the same arrays: calls that overlap on the GPU (other streams or
 * threads) race, so serialise them. Asynchronous on cuda_stream (NULL = default). */
int ph_residual_noalloc(const ph_mesh_desc* mesh, const ph_params* prm, const double* U, double* R,
                        void* cuda_stream);
/* The status word of the last ph_residual_noalloc on this device (bit 0: a non-positive density
 * or pressure was met; the residual then holds the non-physical branch's values, as ph_status
 * reports for a context). Each ph_residual_noalloc clears it first. Waits for cuda_stream. */
int ph_residual_noalloc_status(void* cuda_stream, uint32_t* flags);

/* Self-test of the quotient used inside the flux kernels against IEEE division on n
 * pseudo-random operand pairs; out[0] = max relative error in FP64, out[1] in FP32.
 * No counterpart in the reference. */
int ph_quotient_selftest(uint64_t seed, int n, double out[2]);

/* ---- Batch of independent solves (the parameter-swept snapshot solves of
 * AdaptiveSamplingBase::solveSnapshotFOM, src/reduced_order/adaptive_sampling_base.cpp:255-265,
 * served together). No single counterpart in the reference, which runs one FlowSolver per
 * snapshot. Every admitted solve keeps its state resident in a device arena reserved once
 * (the HBM budget); each RK stage of all admitted solves of one order runs as one persistent
 * kernel over a tile list, the stages of all orders form one CUDA graph per step, and solves
 * join and leave between steps (continuous batching). Split-form Euler, GLL, rk4_ex or
 * ssprk3_ex; affine or curvilinear meshes, periodic or with the Euler boundary conditions of
 * ph_mesh_desc.boundary_type (the solves with boundary faces form groups of their own, run by
 * the boundary-face instance of the batched kernel); one precision per batch. A solve's result is
 * bitwise the one ph_rk_step gives for it alone. Calls on one batch are not thread-safe. */
typedef struct ph_batch ph_batch;
int ph_batch_create(size_t hbm_budget_bytes, int precision, void* cuda_stream, ph_batch** out);
int ph_batch_destroy(ph_batch* b);
/* device bytes one solve takes from the budget */
int ph_batch_bytes(const ph_mesh_desc* mesh, const ph_params* prm, size_t* bytes);
/* Admit one solve with initial state U0 (host, the reference DoF order), time step dt and
 * nsteps steps. *slot receives its id. PH_ERR_NOMEM when the budget has no room now. */
int ph_batch_admit(ph_batch* b, const ph_mesh_desc* mesh, const ph_params* prm, const double* U0, double dt,
                   int nsteps, int* slot);
/* Advance every unfinished solve by up to nsteps steps (each stops at its own count).
 * Asynchronous on the batch stream. */
int ph_batch_step(ph_batch* b, int nsteps);
/* steps done and steps asked of a solve; *active = number of unfinished solves */
int ph_batch_progress(ph_batch* b, int slot, int* steps_done, int* nsteps);
int ph_batch_active(ph_batch* b, int* active);
/* state of a solve (host; a finished solve waits for its own last step only), status word
 * (read clears) */
int ph_batch_get_state(ph_batch* b, int slot, double* U);
int ph_batch_status(ph_batch* b, int slot, uint32_t* flags);
/* return a solve's memory to the budget (a finished or an abandoned solve) */
int ph_batch_release(ph_batch* b, int slot);
/* *complete = 1 once the GPU has finished the solve's last step (non-blocking) */
int ph_batch_poll(ph_batch* b, int slot, int* complete);
/* fence after the work queued so far; wait for a fence (bounds the work in flight) */
int ph_batch_fence(ph_batch* b, long long* ticket);
int ph_batch_fence_wait(ph_batch* b, long long ticket);
/* physical coordinates of the solution nodes of a mesh, [cell][node][3] (no context) */
int ph_mesh_node_xyz(const ph_mesh_desc* mesh, int poly_degree, double* xyz);
/* Tile-shape autotuner: times every cells-per-CTA variant of the batched stage kernel for
 * (poly_degree, curvilinear) on a synthetic periodic-cube solve and keeps the fastest for
 * this process; ms[] (up to 4) receives each variant's time per stage, *best the choice.
 * A batch tunes each new (order, mesh kind) on first use unless a choice is already set. */
int ph_batch_autotune(int poly_degree, int precision, int curvilinear, int* best, double ms[4], int* nvariants);
int ph_batch_set_variant(int poly_degree, int precision, int curvilinear, int variant);
/* launches of this library's kernels issued by ph_batch_step so far (graph nodes counted) */
int ph_batch_launches(ph_batch* b, long long* launches);

/* ---- Served solves: continuous batching behind a submission queue. Callers on any host
 * thread submit solves and collect results; one worker thread owns a ph_batch (HBM budget,
 * precision) and, pass after pass, admits queued solves in FIFO order while the budget holds
 * them (a solve that does not fit waits and holds the ones behind it) for at most admit_slice_s of
 * host time while solves are resident, enqueues chunk_steps RK
 * steps of every resident solve with at most two chunks in flight, and retires each solve
 * whose last step the GPU has finished (final state and status word copied to host memory,
 * arena range released). The solves are the batch's (split-form Euler, ...), with the batch's
 * results. No counterpart in the reference, which runs one FlowSolver per snapshot
 * (AdaptiveSamplingBase::solveSnapshotFOM, src/reduced_order/adaptive_sampling_base.cpp:255-265). */
typedef struct ph_server ph_server;
enum { PH_SOLVE_QUEUED = 0, PH_SOLVE_RUNNING = 1, PH_SOLVE_DONE = 2, PH_SOLVE_FAILED = 3 };
/* admit_slice_s: host time per pass the worker may spend admitting while solves are resident
 * (an admission builds the solve's geometry on the host; e.g. 0.004) */
int ph_server_create(size_t hbm_budget_bytes, int precision, int chunk_steps, double admit_slice_s, ph_server** out);
/* Checks the solve, builds its host-side set-up (operators, connectivity, geometry) on the
 * calling thread, copies U0 (host, n^3 5 (p+1)^3 doubles) and returns a ticket without waiting
 * for the GPU. Thread-safe. */
int ph_server_submit(ph_server* s, const ph_mesh_desc* mesh, const ph_params* prm, const double* U0, double dt,
                     int nsteps, long long* ticket);
int ph_server_poll(ph_server* s, long long ticket, int* state);
/* blocks until the solve is done or failed, or timeout_s passes; *state as ph_server_poll */
int ph_server_wait(ph_server* s, long long ticket, double timeout_s, int* state);
/* A finished solve: final state into U (may be NULL), status word, seconds from submission to
 * admission and to completion; the ticket is then forgotten. A failed solve returns its error. */
int ph_server_result(ph_server* s, long long ticket, double* U, uint32_t* flags, double seconds[2]);
/* out = {solves queued now, admissions deferred for lack of room so far, most solves resident,
 * kernel launches issued so far (graph nodes counted)} */
int ph_server_stats(ph_server* s, long long out[4]);
/* Cancels the solves not yet admitted (they fail), lets the resident ones finish, then frees
 * everything. */
int ph_server_destroy(ph_server* s);

/* ---- Snapshot matrix on the device and its POD basis (OnlinePOD::addSnapshot / computeBasis,
 * src/reduced_order/pod_basis_online.cpp:28-89; fed by FlowSolver::run every
 * output_snapshot_every_x_timesteps, src/flow_solver/flow_solver.cpp:110-120, :675-679, and by
 * the snapshot solves of adaptive sampling, adaptive_sampling_base.cpp:249). The snapshots are
 * the columns of an ndofs x capacity matrix resident on the device; a context's or a batch
 * solve's state is appended by a device copy ordered after that solver's queued work. */
typedef struct ph_snapshots ph_snapshots;
int ph_snapshots_create(int64_t ndofs, int capacity, ph_snapshots** out);
int ph_snapshots_destroy(ph_snapshots* s);
/* appending to a full matrix doubles its capacity (PH_ERR_NOMEM when that allocation fails) */
int ph_snapshots_add(ph_snapshots* s, const double* U, int where);
int ph_snapshots_add_state(ph_snapshots* s, ph_ctx* ctx);            /* the context's current solution */
int ph_snapshots_add_batch(ph_snapshots* s, ph_batch* b, int slot);  /* a batch solve's state */
int ph_snapshots_count(const ph_snapshots* s, int* m);
/* the matrix, column-major: S[j * ndofs + i] = DOF i of snapshot j */
int ph_snapshots_get(ph_snapshots* s, double* S, int where);
/* OnlinePOD::computeBasis: reference_state = the row mean (ndofs), the snapshots centred on it,
 * and the thin SVD of the centred matrix: singular_values (m, descending) and basis (the left
 * singular vectors, column-major ndofs x rank). By the method of snapshots: G = Sc^T Sc on the
 * device (cuBLAS DSYRK), its eigenvectors on the host (Jacobi rotations), U = Sc V / sigma
 * (cuBLAS DGEMM); a singular value below rel_tol x the largest is reported as 0 and its vector
 * is not formed (*rank counts those kept). Each vector's entry of largest magnitude is positive.
 * Output pointers may be NULL; where = PH_HOST or PH_DEVICE for reference_state and basis.
 * Accuracy: sigma_k carries a relative error of about 1e-16 (sigma_1 / sigma_k)^2. */
int ph_snapshots_pod(ph_snapshots* s, double rel_tol, double* reference_state, double* singular_values, double* basis,
                     int where, int* rank);

int ph_sync(ph_ctx* ctx);
const char* ph_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PHILIP_B200_H */
