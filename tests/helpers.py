"""Shared set-up of matching oracle / device discretisations for the tests."""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 6.28318530717958623200


def prm_dict(poly_degree=3, n_cells=4, pde="euler", split=True, two_point="CH",
             conv="two_point_flux_with_roe_dissipation", diss="symm_internal_penalty", fr="cDG",
             fr_aux="kDG", rk="rk4_ex", mach=0.1, reynolds=1600.0, prandtl=0.71, left=0.0, right=TWO_PI,
             cfl=0.1, final_time=1.0, flow_case="taylor_green_vortex"):
    return {
        "dimension": 3, "pde_type": pde, "use_weak_form": False, "flux_nodes_type": "GLL",
        "use_split_form": split, "two_point_num_flux_type": two_point, "conv_num_flux": conv,
        "diss_num_flux": diss, "flux_reconstruction": fr, "flux_reconstruction_aux": fr_aux,
        "all_boundaries_are_periodic": True,
        "do_renumber_dofs": False,
        "ODE solver/ode_solver_type": "runge_kutta", "ODE solver/runge_kutta_method": rk,
        "euler/mach_infinity": mach, "navier_stokes/reynolds_number_inf": reynolds,
        "navier_stokes/prandtl_number": prandtl,
        "flow_solver/flow_case_type": flow_case, "flow_solver/poly_degree": poly_degree,
        "flow_solver/final_time": final_time, "flow_solver/courant_friedrichs_lewy_number": cfl,
        "flow_solver/grid/grid_left_bound": left, "flow_solver/grid/grid_right_bound": right,
        "flow_solver/grid/number_of_grid_elements_per_dimension": n_cells,
    }


def perturbed_tgv(orc, seed=0, amp=0.02):
    """TGV nodal state with a seeded smooth-ish random perturbation (keeps rho, p > 0)."""
    U = orc.initial_condition("tgv")
    rng = np.random.default_rng(seed)
    U = U * (1.0 + amp * rng.standard_normal(U.shape))
    return U


def rel_max_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
