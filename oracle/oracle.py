"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain C++ restatement of PHiLiP's strong-form DG/FR residual and
explicit RK stage (see dg_oracle.hpp for the reference citations). Only the test
suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` load it;
the product library never does.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libphilip_oracle.so")

# enum values shared with dg_oracle.hpp
FLUX_NODES = {"GL": 0, "GLL": 1}
PDE = {"euler": 0, "navier_stokes": 1}
TWO_POINT = {"KG": 0, "IR": 1, "CH": 2, "Ra": 3}
CONV_FLUX = {"lax_friedrichs": 0, "roe": 1, "central_flux": 2, "two_point_flux": 3,
             "two_point_flux_with_lax_friedrichs_dissipation": 4,
             "two_point_flux_with_roe_dissipation": 5}
DISS_FLUX = {"symm_internal_penalty": 0, "bassi_rebay_2": 1, "central_visc_flux": 2}
RK = {"euler_ex": 0, "ssprk3_ex": 1, "rk4_ex": 2, "heun2_ex": 3, "RK4_3_5_3SStar": 4, "RK3_2_5F_3SStarPlus": 5,
      "RK4_3_9F_3SStarPlus": 6, "RK5_4_10F_3SStarPlus": 7}
FR = {"cDG": 0, "cSD": 1, "cHU": 2, "cNegative": 3, "cNegative2": 4, "cPlus": 5,
      "c10Thousand": 6, "cHULumped": 7, "user_specified_value": 8}
FR_AUX = {"kDG": 0, "kSD": 1, "kHU": 2, "kNegative": 3, "kNegative2": 4, "kPlus": 5, "k10Thousand": 6}
ORDER = {"auto": 0, "lexicographic": 1, "morton": 2}
IC = {"tgv": 0, "isentropic_vortex": 1, "vortex_param": 2}
LIMITER = {"none": 0, "maximum_principle": 1, "positivity_preservingZhang2010": 2, "positivity_preservingWang2012": 3}
THERMAL_BC = {"adiabatic": 0, "isothermal": 1}
# boundary_id of each boundary condition (euler.cpp:1508-1560); 0 keeps a periodic pair of sides
BOUNDARY = {"periodic": 0, "wall": 1001, "pressure_outflow": 1002, "inflow": 1003, "riemann_farfield": 1004,
            "farfield": 1005, "slip_wall": 1006, "extrapolation": 1007}


class OrcParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "poly_degree", "overintegration", "flux_nodes", "pde", "use_split_form", "two_point",
        "conv_flux", "diss_flux", "fr_type", "fr_aux_type", "rk_method", "use_constant_viscosity",
        "non_physical", "use_rrk")] + [(n, ctypes.c_double) for n in (
        "fr_user_value", "gamma", "mach_inf", "reynolds_inf", "prandtl", "temperature_inf",
        "constant_viscosity", "sipg_penalty_factor", "atol", "rtol", "rrk_tol")] + [
        ("limiter", ctypes.c_int), ("min_density", ctypes.c_double),
        ("angle_of_attack", ctypes.c_double), ("side_slip_angle", ctypes.c_double),
        ("thermal_bc", ctypes.c_int), ("wall_temperature", ctypes.c_double), ("bc_projected", ctypes.c_int)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.POINTER(vp)]
        L.orc_create_curved.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_ndofs.argtypes = [vp]; L.orc_ndofs.restype = ctypes.c_longlong
        L.orc_nd.argtypes = [vp]; L.orc_nq.argtypes = [vp]; L.orc_status.argtypes = [vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_cell_ijk.argtypes = [vp, ip]
        L.orc_node_xyz.argtypes = [vp, dp]
        L.orc_ops.argtypes = [vp, dp, dp, dp]
        L.orc_minv.argtypes = [vp, dp, dp]
        L.orc_initial_condition.argtypes = [vp, dp, ctypes.c_int, dp]
        L.orc_residual.argtypes = [vp, dp, dp]
        L.orc_aux.argtypes = [vp, dp]
        L.orc_inverse_mass.argtypes = [vp, dp, dp]
        L.orc_rk_step.argtypes = [vp, dp, ctypes.c_double]; L.orc_rk_step.restype = ctypes.c_int
        L.orc_integrals.argtypes = [vp, dp, dp]
        L.orc_limit.argtypes = [vp, dp, ctypes.c_double]
        L.orc_integrated_quantities.argtypes = [vp, dp, dp]
        L.orc_rk_error.argtypes = [vp]; L.orc_rk_error.restype = ctypes.c_double
        L.orc_rrk_gamma.argtypes = [vp]; L.orc_rrk_gamma.restype = ctypes.c_double
        L.orc_numerical_entropy.argtypes = [vp, dp]; L.orc_numerical_entropy.restype = ctypes.c_double
        L.orc_set_boundaries.argtypes = [vp, ip]; L.orc_set_boundaries.restype = ctypes.c_int
        L.orc_boundary_values.argtypes = [vp, ctypes.c_int, dp, dp, dp, dp, dp, dp]
        L.orc_boundary_values.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(cfg: dict) -> OrcParams:
    p = OrcParams()
    p.poly_degree = cfg["poly_degree"]
    p.overintegration = cfg.get("overintegration", 0)
    p.flux_nodes = FLUX_NODES[cfg.get("flux_nodes_type", "GL")]
    p.pde = PDE[cfg.get("pde_type", "navier_stokes")]
    p.use_split_form = int(cfg.get("use_split_form", False))
    p.two_point = TWO_POINT[cfg.get("two_point_num_flux_type", "KG")]
    p.conv_flux = CONV_FLUX[cfg.get("conv_num_flux", "roe")]
    p.diss_flux = DISS_FLUX[cfg.get("diss_num_flux", "symm_internal_penalty")]
    p.fr_type = FR[cfg.get("flux_reconstruction", "cDG")]
    p.fr_aux_type = FR_AUX[cfg.get("flux_reconstruction_aux", "kDG")]
    p.fr_user_value = cfg.get("FR_user_specified_correction_parameter_value", 0.0)
    p.rk_method = RK[cfg.get("runge_kutta_method", "rk4_ex")]
    p.gamma = cfg.get("gamma_gas", 1.4)
    p.mach_inf = cfg.get("mach_infinity", 0.5)
    p.reynolds_inf = cfg.get("reynolds_number_inf", 1.0e7)
    p.prandtl = cfg.get("prandtl_number", 0.72)
    p.temperature_inf = cfg.get("temperature_inf", 273.15)
    p.use_constant_viscosity = int(cfg.get("use_constant_viscosity", False))
    p.constant_viscosity = cfg.get("nondimensionalized_constant_viscosity", 1.0)
    sipg = cfg.get("sipg_penalty_factor", 1.0)
    if cfg.get("diss_num_flux") == "bassi_rebay_2":
        sipg = 0.0   # all_parameters.cpp:611-614
    p.sipg_penalty_factor = sipg
    p.non_physical = {"return_big_number": 0, "abort_run": 1, "print_warning": 2}[cfg.get("non_physical_behavior", "return_big_number")]
    p.atol = cfg.get("atol", 1e-3)
    p.rtol = cfg.get("rtol", 1e-3)
    p.use_rrk = int(cfg.get("use_relaxation_runge_kutta", False))
    p.rrk_tol = cfg.get("relaxation_runge_kutta_root_tolerance", 5e-10)
    p.limiter = LIMITER[cfg.get("bound_preserving_limiter", "none")]
    p.min_density = cfg.get("min_density", 1e-13)
    pi = math.atan(1.0) * 4.0   # degrees to radians as parameters_euler.cpp:41-43
    p.angle_of_attack = cfg.get("angle_of_attack", 0.0) * pi / 180.0
    p.side_slip_angle = cfg.get("side_slip_angle", 0.0) * pi / 180.0
    p.thermal_bc = THERMAL_BC[cfg.get("thermal_boundary_condition_type", "adiabatic")]
    p.wall_temperature = cfg.get("nondimensionalized_isothermal_wall_temperature", 1.0)
    p.bc_projected = int(cfg.get("use_projected_entropy_variables_for_nsfr_boundary_term", False))
    return p


class Oracle:
    """One DG discretisation on a periodic cube, evaluated on the CPU."""

    def __init__(self, cfg: dict, n_cells: int, left: float, right: float, order: str = "auto",
                 warp: float = 0.0, grid_degree: int | None = None, boundaries=None):
        """warp != 0: the sine-warped periodic cube (every coordinate moved by
        warp (L/2pi) sin(2pi(x-l)/L) sin(2pi(y-l)/L) sin(2pi(z-l)/L)) with a mapping of degree
        grid_degree (default: the polynomial degree). boundaries: six boundary types (names of
        BOUNDARY or boundary_id values) for the sides x-, x+, y-, y+, z-, z+; a pair is periodic
        on both sides or on neither."""
        self.cfg = dict(cfg)
        self._p = make_params(cfg)
        h = ctypes.c_void_p()
        if warp != 0.0:
            g = cfg["poly_degree"] if grid_degree is None else grid_degree
            rc = lib().orc_create_curved(ctypes.byref(self._p), n_cells, left, right, ORDER[order], warp, g,
                                         ctypes.byref(h))
        else:
            rc = lib().orc_create(ctypes.byref(self._p), n_cells, left, right, ORDER[order], ctypes.byref(h))
        if rc != 0:
            raise RuntimeError("oracle creation failed")
        self.h = h
        self.n = n_cells
        self.ndofs = int(lib().orc_ndofs(h))
        self.nd = int(lib().orc_nd(h))
        self.nq = int(lib().orc_nq(h))
        self.nc = n_cells ** 3
        if boundaries is not None:
            t = (ctypes.c_int * 6)(*boundary_ids(boundaries))
            if lib().orc_set_boundaries(h, t) != 0:
                raise RuntimeError("oracle: boundaries refused")

    def boundary_values(self, btype, normal, u, grad=None):
        """The boundary states at one face node: (convective exterior state, viscous exterior
        state, viscous exterior gradient [5][3])."""
        n = np.ascontiguousarray(normal, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        g = np.zeros((5, 3)) if grad is None else np.ascontiguousarray(grad, dtype=np.float64)
        uc, uv, gv = np.zeros(5), np.zeros(5), np.zeros((5, 3))
        if lib().orc_boundary_values(self.h, boundary_ids([btype])[0], _dp(n), _dp(u), _dp(g), _dp(uc), _dp(uv),
                                     _dp(gv)) != 0:
            raise RuntimeError("oracle: boundary type refused")
        return uc, uv, gv

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    @staticmethod
    def set_threads(n: int):
        lib().orc_set_threads(n)

    def cell_ijk(self):
        out = np.zeros((self.nc, 3), dtype=np.int32)
        lib().orc_cell_ijk(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return out

    def node_xyz(self):
        out = np.zeros((self.nc, self.nd ** 3, 3))
        lib().orc_node_xyz(self.h, _dp(out))
        return out

    def ops(self):
        xs, xq, wq = np.zeros(self.nd), np.zeros(self.nq), np.zeros(self.nq)
        lib().orc_ops(self.h, _dp(xs), _dp(xq), _dp(wq))
        return xs, xq, wq

    def initial_condition(self, ic="tgv", params=None):
        U = np.zeros(self.ndofs)
        icp = np.zeros(16) if params is None else np.ascontiguousarray(params, dtype=np.float64)
        lib().orc_initial_condition(self.h, _dp(U), IC[ic], _dp(icp))
        return U

    def residual(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros(self.ndofs)
        lib().orc_residual(self.h, _dp(U), _dp(R))
        return R

    def aux(self):
        out = np.zeros(3 * self.ndofs)
        lib().orc_aux(self.h, _dp(out))
        return out.reshape(3, self.ndofs)

    def inverse_mass(self, R):
        R = np.ascontiguousarray(R, dtype=np.float64)
        out = np.zeros(self.ndofs)
        lib().orc_inverse_mass(self.h, _dp(R), _dp(out))
        return out

    def rk_step(self, U, dt):
        if lib().orc_rk_step(self.h, _dp(U), dt) != 0:
            raise RuntimeError("oracle RK step failed (relaxation root finding)")

    def rrk_gamma(self) -> float:
        """Relaxation parameter of the last relaxation-RK step (1 before the first)."""
        return float(lib().orc_rrk_gamma(self.h))

    def numerical_entropy(self, U) -> float:
        """Integrated numerical entropy sum W det J (-rho log(p rho^-gamma)) over the nodes."""
        return float(lib().orc_numerical_entropy(self.h, _dp(np.ascontiguousarray(U))))

    def rk_error(self) -> float:
        """Weighted RMS error estimate of the last low-storage step."""
        return float(lib().orc_rk_error(self.h))

    def limit(self, U, dt):
        """PositivityPreservingLimiter::limit on U in place (for a stage of time step dt)."""
        lib().orc_limit(self.h, _dp(U), dt)

    def integrals(self, U):
        out = np.zeros(4)
        lib().orc_integrals(self.h, _dp(np.ascontiguousarray(U)), _dp(out))
        return out

    def integrated_quantities(self, U):
        """The nine PeriodicTurbulence integrated quantities (IntegratedQuantitiesEnum order, each
        over the domain volume) and the max wave speed as a tenth entry."""
        out = np.zeros(10)
        lib().orc_integrated_quantities(self.h, _dp(np.ascontiguousarray(U)), _dp(out))
        return out

    def status(self):
        return int(lib().orc_status(self.h))


def boundary_ids(types):
    """boundary_id values of boundary types given by name or by id."""
    return [BOUNDARY[t] if isinstance(t, str) else int(t) for t in types]


def tgv_constant_dt(cfl, left, right, n_cells, poly_degree):
    """PeriodicTurbulence::get_constant_time_step (periodic_turbulence.cpp:115-127)."""
    ndof_per_state = (n_cells * (poly_degree + 1)) ** 3
    return cfl * (right - left) / ndof_per_state ** (1.0 / 3.0)


def run_to_final_time(stepper, U, dt, final_time, t0=0.0):
    """FlowSolver::run time loop with end_exactly_at_final_time (flow_solver.cpp:554-574)."""
    t = t0
    nsteps = 0
    while t < final_time:
        step = dt
        if t + step > final_time:
            step = final_time - t
        stepper(U, step)
        t += step
        nsteps += 1
    return t, nsteps
