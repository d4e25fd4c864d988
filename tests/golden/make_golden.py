"""Extracts the Taylor-Green energy-check golden values from the reference's own
integration-test parameter files into tests/golden/tgv_energy_check.json.

Run where a checkout of the reference is present, giving the path of its root:
    python tests/golden/make_golden.py <path-to-PHiLiP-checkout>
Only parameter values and expected numbers are copied, not the files.
"""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from philip_b200.prm import parse_file  # noqa: E402

REL = "tests/integration_tests_control_files/taylor_green_vortex_integration"
FILES = [
    "viscous_taylor_green_vortex_energy_check_strong_quick.prm",
    "viscous_taylor_green_vortex_energy_check_nsfr_gll_flux_nodes_quick.prm",
    "viscous_taylor_green_vortex_energy_check_nsfr_gl_flux_nodes_quick.prm",
]
KEYS = ["pde_type", "use_weak_form", "use_split_form", "flux_nodes_type", "flux_reconstruction",
        "two_point_num_flux_type", "conv_num_flux", "diss_num_flux", "use_inverse_mass_on_the_fly",
        "ODE solver/ode_solver_type", "ODE solver/runge_kutta_method", "euler/mach_infinity",
        "navier_stokes/prandtl_number", "navier_stokes/reynolds_number_inf", "flow_solver/flow_case_type",
        "flow_solver/poly_degree", "flow_solver/final_time", "flow_solver/courant_friedrichs_lewy_number",
        "flow_solver/grid/grid_left_bound", "flow_solver/grid/grid_right_bound",
        "flow_solver/grid/number_of_grid_elements_per_dimension",
        "flow_solver/taylor_green_vortex/expected_kinetic_energy_at_final_time",
        "flow_solver/taylor_green_vortex/expected_theoretical_dissipation_rate_at_final_time"]


def main(ref_root):
    out = {}
    for f in FILES:
        d = parse_file(os.path.join(ref_root, REL, f))
        out[f.replace(".prm", "")] = {"source": f"{REL}/{f}", "params": {k: d[k] for k in KEYS if k in d}}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tgv_energy_check.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path-to-PHiLiP-checkout>")
    main(sys.argv[1])
