// CPU oracle for the explicit strong-form DG/FR residual and Runge-Kutta stage.
//
// TEST INFRASTRUCTURE ONLY. This is a from-source restatement, in plain C++, of
// PHiLiP's DGStrong residual (src/dg/strong_dg.cpp), its sum-factorised operators
// (src/operators/operators.cpp), Euler/Navier-Stokes physics (src/physics/euler.cpp,
// src/physics/navier_stokes.cpp), numerical fluxes (src/numerical_flux/*.cpp), the
// inverse mass matrix (src/dg/dg_base.cpp:4089-4260) and the Butcher RK stage loop
// (src/ode_solver/runge_kutta_ode_solver.cpp). It is the checker against which the
// CUDA path is compared, and the timed CPU baseline. Nothing in the shipped library
// links or calls it.
//
// Parity pin: the Taylor-Green kinetic-energy / dissipation-rate golden values from
// tests/integration_tests_control_files/taylor_green_vortex_integration/*.prm
// (see tests/test_oracle_golden.py).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace oracle {

constexpr int NSTATE = 5;
constexpr int DIM = 3;

enum FluxNodes { GL = 0, GLL = 1 };
enum Pde { EULER = 0, NAVIER_STOKES = 1 };
enum TwoPoint { KG = 0, IR = 1, CH = 2, RA = 3 };
enum ConvFlux { LAX_FRIEDRICHS = 0, ROE = 1, CENTRAL = 2, TWO_POINT = 3, TWO_POINT_LXF = 4, TWO_POINT_ROE = 5 };
enum DissFlux { SIPG = 0, BR2 = 1, CENTRAL_VISC = 2 };
enum RkMethod { RK_EULER = 0, SSPRK3 = 1, RK4 = 2, HEUN2 = 3,
                LS_RK4_3_5 = 4, LS_RK3_2_5F = 5, LS_RK4_3_9F = 6, LS_RK5_4_10F = 7 };
enum FrType { C_DG = 0, C_SD = 1, C_HU = 2, C_NEGATIVE = 3, C_NEGATIVE2 = 4, C_PLUS = 5, C_10THOUSAND = 6, C_HU_LUMPED = 7, C_USER = 8 };
enum FrAuxType { K_DG = 0, K_SD = 1, K_HU = 2, K_NEGATIVE = 3, K_NEGATIVE2 = 4, K_PLUS = 5, K_10THOUSAND = 6 };
enum CellOrder { ORDER_AUTO = 0, ORDER_LEXICOGRAPHIC = 1, ORDER_MORTON = 2 };
enum NonPhysical { RETURN_BIG_NUMBER = 0, ABORT_RUN = 1, PRINT_WARNING = 2 };
// limiter/bound_preserving_limiter (parameters_limiter.cpp:17-30); the positivity-preserving ones
enum Limiter { LIMITER_NONE = 0, LIMITER_MAXIMUM_PRINCIPLE = 1, PPL_ZHANG2010 = 2, PPL_WANG2012 = 3 };
enum ThermalBc { THERMAL_ADIABATIC = 0, THERMAL_ISOTHERMAL = 1 };
// boundary_id values of the boundary conditions (euler.cpp:1508-1560, navier_stokes.cpp:1354-1390);
// 0 marks a periodic pair of cube sides here
enum BoundaryType { BC_WALL = 1001, BC_PRESSURE_OUTFLOW = 1002, BC_INFLOW = 1003, BC_RIEMANN = 1004,
                    BC_FARFIELD = 1005, BC_SLIP_WALL = 1006, BC_EXTRAPOLATION = 1007 };

// Plain parameter block (mirrors the .prm keys of the hot path).
struct Params {
    int poly_degree = 2;
    int overintegration = 0;
    int flux_nodes = GL;
    int pde = NAVIER_STOKES;
    int use_split_form = 0;
    int two_point = KG;
    int conv_flux = ROE;
    int diss_flux = SIPG;
    int fr_type = C_DG;
    int fr_aux_type = K_DG;
    double fr_user_value = 0.0;
    int rk_method = RK4;
    double gamma = 1.4;
    double mach_inf = 0.1;
    double reynolds_inf = 1.0e7;
    double prandtl = 0.72;
    double temperature_inf = 273.15;
    int use_constant_viscosity = 0;
    double constant_viscosity = 1.0;
    double sipg_penalty_factor = 1.0;
    int non_physical = RETURN_BIG_NUMBER;
    double atol = 1e-3, rtol = 1e-3;   // low-storage error estimate
    int use_rrk = 0;                   // relaxation Runge-Kutta (root-finding, entropy)
    double rrk_tol = 5e-10;            // relaxation_runge_kutta_root_tolerance
    int limiter = LIMITER_NONE;        // limiter/bound_preserving_limiter
    double min_density = 1e-13;        // limiter/min_density
    // boundary conditions: the free stream's angles in radians (euler/angle_of_attack and
    // side_slip_angle, given in degrees, parameters_euler.cpp:39-43) and the wall's thermal
    // condition (navier_stokes/thermal_boundary_condition_type, 0 adiabatic / 1 isothermal, and
    // nondimensionalized_isothermal_wall_temperature, parameters_navier_stokes.cpp:21-50)
    double angle_of_attack = 0.0, side_slip_angle = 0.0;
    int thermal_bc = THERMAL_ADIABATIC;
    double wall_temperature = 1.0;
    // use_projected_entropy_variables_for_nsfr_boundary_term (all_parameters.cpp:399, default false)
    int bc_projected = 0;
};

// One-dimensional operators on the reference interval [0,1]
// (operators.cpp:1217-2005, dg_base.cpp:131-261).
struct Ops1D {
    int nd = 0;                 // solution shape functions per direction (p+1)
    int nq = 0;                 // flux/volume cubature nodes per direction
    std::vector<double> xs;     // solution support points (GLL points of FE_DGQ)
    std::vector<double> xq, wq; // flux nodes and weights
    std::vector<double> chi, dchi;      // nq x nd, solution basis / derivative at flux nodes
    std::array<std::vector<double>, 2> chi_s;   // 1 x nd, solution basis at xi=0 and xi=1
    std::vector<double> phi, dphi;      // nq x nq, flux (Lagrange on flux nodes) basis / derivative
    std::array<std::vector<double>, 2> phi_s;   // 1 x nq
    std::vector<double> skew;           // nq x nq, S - S^T of the flux basis
    std::vector<double> proj;           // nd x nq, M^{-1} chi^T W
    std::vector<double> minv;           // nd x nd, (M + K)^{-1}
    std::vector<double> minv_aux;       // nd x nd, (M + K_aux)^{-1}
};

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);   // on [0,1]
void gauss_lobatto(int n, std::vector<double>& x, std::vector<double>& w);    // on [0,1]
void lagrange_eval(const std::vector<double>& nodes, double x, double* val, double* der);
Ops1D build_ops(const Params& prm);
double fr_correction_parameter(int fr_type, int p, double user_value);

// Structured periodic hexahedral mesh with per-node metric terms.
struct Mesh {
    int n = 0;                  // cells per direction
    int nc = 0;                 // number of cells
    int order = ORDER_LEXICOGRAPHIC;
    double left = 0.0, right = 1.0;
    std::vector<std::array<int, 3>> ijk;        // cell -> (ix,iy,iz)
    std::vector<int> cell_of;                   // lexicographic index -> cell id
    std::vector<std::array<int, 6>> nbr;        // cell, face -> neighbour cell (-1: boundary face)
    std::vector<std::array<int, 6>> bnd;        // cell, face -> boundary_id of a boundary face (0 inside)
    // metric terms at volume flux nodes: C[cell][node][3][3], detJ[cell][node]
    bool affine = true;
    double h = 1.0;
    std::vector<double> cof;     // nc * nq^3 * 9
    std::vector<double> detj;    // nc * nq^3
    std::vector<double> cof_face; // nc * 6 * nq^2 * 9 (facet metric, interior side)
    std::vector<double> xnode;   // nc * nd^3 * 3 physical positions of solution support points
    double warp = 0.0;           // amplitude of x_i += warp*sin(x)sin(y)sin(z) (curvilinear)
    int grid_degree = 1;
};

Mesh build_periodic_cube(int n, double left, double right, int order, const Ops1D& ops,
                         double warp = 0.0, int grid_degree = 1);

// DG discretisation state.
constexpr int NUM_INTEGRATED = 9;   // PeriodicTurbulence::IntegratedQuantitiesEnum

struct Solver {
    Params prm;
    Ops1D ops;
    Mesh mesh;
    int nd3 = 0, nq3 = 0, ndofs_cell = 0;
    std::vector<double> aux;     // 3 * ndofs (auxiliary gradient, dof-major per dimension)
    int status = 0;              // bit 0: non-physical state met
    double last_error = 0.0;     // weighted RMS error estimate of the last low-storage step
    double current_time = 0.0;
    int nthreads = 0;

    void init(const Params& p, int n, double left, double right, int order,
              double warp = 0.0, int grid_degree = 1);
    std::size_t ndofs() const { return (std::size_t)mesh.nc * ndofs_cell; }
    // non-periodic sides of the cube: types[f] for the sides x-, x+, y-, y+, z-, z+ (0 keeps
    // a periodic pair; a pair is periodic on both sides or on neither), as the boundary_id a flow
    // case's grid gives its boundary faces (e.g. channel_flow.cpp:324-343)
    void set_boundaries(const int types[6]);
    // the exterior states of boundary `type` at one face node (outward unit normal n): the
    // convective one (boundary_face_values) and the viscous one with its gradient
    // (boundary_face_values_viscous_flux)
    void boundary_values(int type, const double* n, const double* u, const double* g, double* ub_conv,
                         double* ub_visc, double* gb_visc);
    // right-hand side R(U) (before the inverse mass matrix), dg_base.cpp:2599-2915
    void assemble_residual(const double* U, double* R);
    // out = M^{-1} in (dg_base.cpp:4089-4260)
    void apply_inverse_mass(const double* in, double* out, bool aux_eq = false);
    // one explicit Butcher RK step (runge_kutta_base.cpp:21-39)
    void rk_step(double* U, double dt);
    // one low-storage 3S* / 3S*+ step, leaving its error estimate in last_error
    void lsrk_step(double* U, double dt);
    // relaxation Runge-Kutta: the last step's relaxation parameter (also the next step's
    // initial guess, rrk_ode_solver_base.h:28) and the integrated numerical entropy
    double rrk_gamma = 1.0;
    double numerical_entropy(const double* U) const;
    double entropy_vars_dot_mass(const double* st, const double* R);
    double relaxation_parameter(const double* un, const std::vector<std::vector<double>>& k, const double* b,
                                int ns, double dt, double est);
    // PositivityPreservingLimiter::limit (positivity_preserving_limiter.cpp:381-678) on a state,
    // for the stage solution of time step dt; no-op unless prm.limiter is a positivity limiter
    void limit(double* U, double dt);
    // nodal interpolation of an initial condition (set_initial_condition.cpp:51)
    void interpolate_ic(double* U, int ic, const double* ic_params);
    // TGV integrated quantities (periodic_turbulence.cpp:439-672):
    // out[0]=KE, out[1]=enstrophy, out[2]=vorticity dissipation rate, out[3]=max wave speed
    void integrals(const double* U, double* out);
    // out[0..8]: the nine integrated quantities in the order of PeriodicTurbulence's
    // IntegratedQuantitiesEnum (periodic_turbulence.h:176-186), each over the domain volume
    // (angular momentum always computed); out[9] = max wave speed
    void integrated_quantities(const double* U, double* out);
};

enum InitialCondition { IC_TGV = 0, IC_ISENTROPIC_VORTEX = 1, IC_VORTEX_PARAM = 2 };

} // namespace oracle
