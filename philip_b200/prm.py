"""Reader of PHiLiP ``.prm`` files (dealii::ParameterHandler syntax) for the keys of
the explicit strong-form DG/FR path.

Syntax: ``set key = value``, ``subsection name`` ... ``end``, ``#`` comments. Keys
outside the hot path are kept in the tree but ignored. Defaults follow the
reference's declarations (src/parameters/all_parameters.cpp:39-400,
parameters_euler.cpp, parameters_navier_stokes.cpp, parameters_ode_solver.cpp,
parameters_flow_solver.cpp).
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import _lib

FLUX_NODES = {"GL": 0, "GLL": 1}
PDE = {"euler": 0, "navier_stokes": 1}
TWO_POINT = {"KG": 0, "IR": 1, "CH": 2, "Ra": 3}
CONV_FLUX = {"lax_friedrichs": 0, "roe": 1, "central_flux": 2, "two_point_flux": 3,
             "two_point_flux_with_lax_friedrichs_dissipation": 4, "two_point_flux_with_roe_dissipation": 5}
DISS_FLUX = {"symm_internal_penalty": 0, "bassi_rebay_2": 1, "central_visc_flux": 2}
FR = {"cDG": 0, "cSD": 1, "cHU": 2, "cNegative": 3, "cNegative2": 4, "cPlus": 5, "c10Thousand": 6,
      "cHULumped": 7, "user_specified_value": 8}
FR_AUX = {"kDG": 0, "kSD": 1, "kHU": 2, "kNegative": 3, "kNegative2": 4, "kPlus": 5,   # all_parameters.h:299
          "k10Thousand": 6}
RK = {"rk4_ex": 0, "ssprk3_ex": 1, "heun2_ex": 2, "euler_ex": 3,   # parameters_ode_solver.h:66-78 order
      "RK4_3_5_3SStar": 7, "RK3_2_5F_3SStarPlus": 8, "RK4_3_9F_3SStarPlus": 9, "RK5_4_10F_3SStarPlus": 10}
RK_ORDER = {"rk4_ex": 4, "ssprk3_ex": 3, "heun2_ex": 2, "euler_ex": 1, "RK4_3_5_3SStar": 4,
            "RK3_2_5F_3SStarPlus": 3, "RK4_3_9F_3SStarPlus": 4, "RK5_4_10F_3SStarPlus": 5}
NON_PHYSICAL = {"return_big_number": 0, "abort_run": 1, "print_warning": 2}
LIMITER = {"none": 0, "maximum_principle": 1, "positivity_preservingZhang2010": 2, "positivity_preservingWang2012": 3}
THERMAL_BC = {"adiabatic": 0, "isothermal": 1}

DEFAULTS = {
    "dimension": "-1", "pde_type": "advection", "use_weak_form": "true", "flux_nodes_type": "GL",
    "overintegration": "0", "use_split_form": "false", "two_point_num_flux_type": "KG",
    "use_curvilinear_split_form": "false", "conv_num_flux": "lax_friedrichs",
    "diss_num_flux": "symm_internal_penalty", "flux_reconstruction": "cDG", "flux_reconstruction_aux": "kDG",
    "FR_user_specified_correction_parameter_value": "0.0", "sipg_penalty_factor": "1.0",
    "use_inverse_mass_on_the_fly": "false", "non_physical_behavior": "return_big_number",
    "all_boundaries_are_periodic": "false", "do_renumber_dofs": "true", "test_type": "run_control",
    "ODE solver/ode_solver_type": "implicit", "ODE solver/runge_kutta_method": "ssprk3_ex",
    "euler/mach_infinity": "0.5", "euler/gamma_gas": "1.4",
    "navier_stokes/prandtl_number": "0.72", "navier_stokes/reynolds_number_inf": "10000000.0",
    "navier_stokes/temperature_inf": "273.15", "navier_stokes/use_constant_viscosity": "false",
    "navier_stokes/nondimensionalized_constant_viscosity": "1.0",
    "flow_solver/flow_case_type": "taylor_green_vortex", "flow_solver/poly_degree": "1",
    "flow_solver/final_time": "1", "flow_solver/constant_time_step": "0",
    "flow_solver/courant_friedrichs_lewy_number": "1", "flow_solver/adaptive_time_step": "false",
    "flow_solver/end_exactly_at_final_time": "true",
    "flow_solver/grid/grid_left_bound": "0.0", "flow_solver/grid/grid_right_bound": "1.0",
    "flow_solver/grid/number_of_grid_elements_per_dimension": "4",
    "ODE solver/low-storage rk solver/atol": "0.001", "ODE solver/low-storage rk solver/rtol": "0.001", "ODE solver/low-storage rk solver/beta1": "0.70",
    "ODE solver/low-storage rk solver/beta2": "-0.23", "ODE solver/low-storage rk solver/beta3": "0.0", "flow_solver/error_adaptive_time_step": "false",
    "ODE solver/rrk root solver/use_relaxation_runge_kutta": "false",
    "ODE solver/rrk root solver/relaxation_runge_kutta_root_tolerance": "5e-10",
    "ODE solver/rrk root solver/rrk_root_solver_output": "quiet",
    "ODE solver/initial_time": "0.0", "ODE solver/initial_iteration": "0", "ODE solver/initial_time_step": "100.0",
    "ODE solver/initial_desired_time_for_output_solution_every_dt_time_intervals": "0.0",
    "flow_solver/unsteady_data_table_filename": "unsteady_data_table",
    "flow_solver/dipole_wall_collision/do_compute_angular_momentum": "false",
    "reduced order/output_snapshot_every_x_timesteps": "0",
    "flow_solver/output_restart_files": "false", "flow_solver/restart_computation_from_file": "false",
    "flow_solver/restart_files_directory_name": ".", "flow_solver/restart_file_index": "1",
    "flow_solver/output_restart_files_every_x_steps": "1",
    "flow_solver/output_restart_files_every_dt_time_intervals": "0.0",
    "limiter/bound_preserving_limiter": "none", "limiter/min_density": "1e-13",
    "euler/angle_of_attack": "0.0", "euler/side_slip_angle": "0.0",
    "navier_stokes/thermal_boundary_condition_type": "adiabatic",
    "navier_stokes/nondimensionalized_isothermal_wall_temperature": "1.0",
    "use_projected_entropy_variables_for_nsfr_boundary_term": "false",
    "flow_solver/taylor_green_vortex/expected_kinetic_energy_at_final_time": "0",
    "flow_solver/taylor_green_vortex/expected_theoretical_dissipation_rate_at_final_time": "0",
}


def parse_text(text: str) -> dict:
    """Return a flat dict 'sub/sub/key' -> value string for every ``set`` line."""
    out: dict = {}
    stack: list = []
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("subsection"):
            stack.append(line[len("subsection"):].strip())
        elif line == "end":
            if not stack:
                raise ValueError("unbalanced 'end' in parameter file")
            stack.pop()
        elif line.startswith("set "):
            body = line[4:]
            if "=" not in body:
                raise ValueError(f"malformed line: {raw!r}")
            key, val = body.split("=", 1)
            out["/".join(stack + [key.strip()])] = val.strip()
        else:
            raise ValueError(f"unrecognised line: {raw!r}")
    if stack:
        raise ValueError(f"unterminated subsection(s): {stack}")
    return out


def format_text(values: dict) -> str:
    """The inverse of parse_text: a .prm text with one ``set`` line per key, subsections
    nested in the order their keys first appear."""
    tree: dict = {}
    for key, val in values.items():
        node = tree
        *subs, leaf = key.split("/")
        for sub in subs:
            node = node.setdefault(("sub", sub), {})
        node[("set", leaf)] = val
    lines: list = []

    def emit(node, depth):
        pad = "  " * depth
        for (kind, name), v in node.items():
            if kind == "set":
                lines.append(f"{pad}set {name} = {v}")
        for (kind, name), v in node.items():
            if kind == "sub":
                lines.append(f"{pad}subsection {name}")
                emit(v, depth + 1)
                lines.append(f"{pad}end")
    emit(tree, 0)
    return "\n".join(lines) + "\n"


def parse_file(path: str) -> dict:
    with open(path) as f:
        return parse_text(f.read())


def _b(v: str) -> bool:
    v = v.strip().lower()
    if v in ("true", "1", "yes"):
        return True
    if v in ("false", "0", "no"):
        return False
    raise ValueError(f"not a bool: {v}")


@dataclass
class Parameters:
    """The hot-path subset of AllParameters, with the reference's defaults."""
    raw: dict = field(default_factory=dict)

    def get(self, key: str) -> str:
        if key in self.raw:
            return self.raw[key]
        return DEFAULTS[key]

    @classmethod
    def from_text(cls, text: str) -> "Parameters":
        return cls(parse_text(text))

    @classmethod
    def from_file(cls, path: str) -> "Parameters":
        return cls(parse_file(path))

    def with_values(self, updates: dict) -> "Parameters":
        """A copy with the given keys set (values as the .prm spells them)."""
        raw = dict(self.raw)
        for k, v in updates.items():
            raw[k] = str(v).lower() if isinstance(v, bool) else str(v)
        return Parameters(raw)

    def to_text(self) -> str:
        return format_text(self.raw)

    @classmethod
    def from_dict(cls, d: dict) -> "Parameters":
        return cls({k: str(v).lower() if isinstance(v, bool) else str(v) for k, v in d.items()})

    # -- typed accessors
    @property
    def poly_degree(self) -> int:
        return int(self.get("flow_solver/poly_degree"))

    @property
    def n_cells(self) -> int:
        return int(self.get("flow_solver/grid/number_of_grid_elements_per_dimension"))

    @property
    def use_relaxation_runge_kutta(self) -> bool:
        """ODE solver/rrk root solver/use_relaxation_runge_kutta, or the deprecated
        ode_solver_type = rrk_explicit (parameters_ode_solver.cpp:299-315)."""
        return (_b(self.get("ODE solver/rrk root solver/use_relaxation_runge_kutta"))
                or self.get("ODE solver/ode_solver_type") == "rrk_explicit")

    @property
    def grid_bounds(self):
        return float(self.get("flow_solver/grid/grid_left_bound")), float(self.get("flow_solver/grid/grid_right_bound"))

    def to_ph_params(self, precision: int = _lib.PH_FP64) -> _lib.PhParams:
        p = _lib.PhParams()
        pde = self.get("pde_type")
        if pde not in PDE:
            raise ValueError(f"pde_type {pde!r} is outside the strong-form Euler/Navier-Stokes path")
        if _b(self.get("use_weak_form")):
            raise ValueError("use_weak_form = true: the B200 path implements the strong form (DGStrong)")
        p.poly_degree = self.poly_degree
        p.overintegration = int(self.get("overintegration"))
        p.flux_nodes_type = FLUX_NODES[self.get("flux_nodes_type")]
        p.pde_type = PDE[pde]
        p.use_split_form = int(_b(self.get("use_split_form")) or _b(self.get("use_curvilinear_split_form")))
        p.two_point_num_flux_type = TWO_POINT[self.get("two_point_num_flux_type")]
        p.conv_num_flux = CONV_FLUX[self.get("conv_num_flux")]
        p.diss_num_flux = DISS_FLUX[self.get("diss_num_flux")]
        p.flux_reconstruction = FR[self.get("flux_reconstruction")]
        aux = self.get("flux_reconstruction_aux")
        if aux not in FR_AUX:
            raise ValueError(f"flux_reconstruction_aux {aux!r} is not a reference value")
        p.flux_reconstruction_aux = FR_AUX[aux]
        p.FR_user_specified_correction_parameter_value = float(self.get("FR_user_specified_correction_parameter_value"))
        if self.get("ODE solver/ode_solver_type") not in ("runge_kutta", "rrk_explicit"):
            raise ValueError("ode_solver_type must be runge_kutta (explicit RK)")
        p.runge_kutta_method = RK[self.get("ODE solver/runge_kutta_method")]
        p.gamma_gas = float(self.get("euler/gamma_gas"))
        p.mach_infinity = float(self.get("euler/mach_infinity"))
        p.reynolds_number_inf = float(self.get("navier_stokes/reynolds_number_inf"))
        p.prandtl_number = float(self.get("navier_stokes/prandtl_number"))
        p.temperature_inf = float(self.get("navier_stokes/temperature_inf"))
        p.use_constant_viscosity = int(_b(self.get("navier_stokes/use_constant_viscosity")))
        p.nondimensionalized_constant_viscosity = float(self.get("navier_stokes/nondimensionalized_constant_viscosity"))
        sipg = float(self.get("sipg_penalty_factor"))
        if self.get("diss_num_flux") == "bassi_rebay_2":
            sipg = 0.0        # all_parameters.cpp:611-614
        p.sipg_penalty_factor = sipg
        p.non_physical_behavior = NON_PHYSICAL[self.get("non_physical_behavior")]
        p.precision = precision
        p.rk_atol = float(self.get("ODE solver/low-storage rk solver/atol"))
        p.rk_rtol = float(self.get("ODE solver/low-storage rk solver/rtol"))
        p.use_relaxation_runge_kutta = int(self.use_relaxation_runge_kutta)
        p.relaxation_runge_kutta_root_tolerance = float(
            self.get("ODE solver/rrk root solver/relaxation_runge_kutta_root_tolerance"))
        p.pressure_shift = self.reference_pressure()
        p.bound_preserving_limiter = LIMITER[self.get("limiter/bound_preserving_limiter")]
        p.min_density = float(self.get("limiter/min_density"))
        p.angle_of_attack = float(self.get("euler/angle_of_attack"))
        p.side_slip_angle = float(self.get("euler/side_slip_angle"))
        p.thermal_boundary_condition_type = THERMAL_BC[self.get("navier_stokes/thermal_boundary_condition_type")]
        p.isothermal_wall_temperature = float(self.get("navier_stokes/nondimensionalized_isothermal_wall_temperature"))
        p.use_projected_entropy_variables_for_nsfr_boundary_term = int(
            _b(self.get("use_projected_entropy_variables_for_nsfr_boundary_term")))
        return p

    def reference_pressure(self) -> float:
        """The flow case's free-stream pressure in its nondimensional scaling, which the
        precision form takes out of its momentum fluxes: 1/(gamma M^2) for the Taylor-Green
        vortex (initial_condition_function.cpp:261-310), 1/gamma for the isentropic vortex
        (:643-690); 0 (no shift) otherwise."""
        gamma = float(self.get("euler/gamma_gas"))
        case = self.get("flow_solver/flow_case_type")
        if case == "taylor_green_vortex":
            mach = float(self.get("euler/mach_infinity"))
            return 1.0 / (gamma * mach * mach)
        if case == "isentropic_vortex":
            return 1.0 / gamma
        return 0.0

    def oracle_cfg(self) -> dict:
        """The same settings in the key set the CPU oracle's wrapper takes (tests only)."""
        return {
            "poly_degree": self.poly_degree, "overintegration": int(self.get("overintegration")),
            "flux_nodes_type": self.get("flux_nodes_type"), "pde_type": self.get("pde_type"),
            "use_split_form": _b(self.get("use_split_form")),
            "two_point_num_flux_type": self.get("two_point_num_flux_type"),
            "conv_num_flux": self.get("conv_num_flux"), "diss_num_flux": self.get("diss_num_flux"),
            "flux_reconstruction": self.get("flux_reconstruction"),
            "flux_reconstruction_aux": self.get("flux_reconstruction_aux"),
            "runge_kutta_method": self.get("ODE solver/runge_kutta_method"),
            "gamma_gas": float(self.get("euler/gamma_gas")), "mach_infinity": float(self.get("euler/mach_infinity")),
            "reynolds_number_inf": float(self.get("navier_stokes/reynolds_number_inf")),
            "prandtl_number": float(self.get("navier_stokes/prandtl_number")),
            "temperature_inf": float(self.get("navier_stokes/temperature_inf")),
            "use_constant_viscosity": _b(self.get("navier_stokes/use_constant_viscosity")),
            "sipg_penalty_factor": float(self.get("sipg_penalty_factor")),
            "FR_user_specified_correction_parameter_value": float(self.get("FR_user_specified_correction_parameter_value")),
            "atol": float(self.get("ODE solver/low-storage rk solver/atol")), "rtol": float(self.get("ODE solver/low-storage rk solver/rtol")),
            "use_relaxation_runge_kutta": self.use_relaxation_runge_kutta,
            "relaxation_runge_kutta_root_tolerance": float(
                self.get("ODE solver/rrk root solver/relaxation_runge_kutta_root_tolerance")),
            "bound_preserving_limiter": self.get("limiter/bound_preserving_limiter"),
            "min_density": float(self.get("limiter/min_density")),
            "nondimensionalized_constant_viscosity": float(self.get("navier_stokes/nondimensionalized_constant_viscosity")),
            "angle_of_attack": float(self.get("euler/angle_of_attack")),
            "side_slip_angle": float(self.get("euler/side_slip_angle")),
            "thermal_boundary_condition_type": self.get("navier_stokes/thermal_boundary_condition_type"),
            "nondimensionalized_isothermal_wall_temperature": float(
                self.get("navier_stokes/nondimensionalized_isothermal_wall_temperature")),
            "use_projected_entropy_variables_for_nsfr_boundary_term": _b(
                self.get("use_projected_entropy_variables_for_nsfr_boundary_term")),
        }
