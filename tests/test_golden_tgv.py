"""Golden Taylor-Green energy checks from the reference's own integration tests
(taylor_green_vortex_energy_check.cpp:19-47: KE and vorticity-based dissipation rate
at the final time within 1e-10 relative).

The CPU oracle must reproduce all three (GL and GLL flux nodes, strong and split
forms); the CUDA path reproduces the GLL one here and the two on GL flux nodes in
test_gpu_gl.py.
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, run_to_final_time, tgv_constant_dt
from philip_b200.prm import Parameters

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tgv_energy_check.json")))
TOL = 1e-10


def _expected(case):
    p = GOLDEN[case]["params"]
    return (float(p["flow_solver/taylor_green_vortex/expected_kinetic_energy_at_final_time"]),
            float(p["flow_solver/taylor_green_vortex/expected_theoretical_dissipation_rate_at_final_time"]))


def _params(case):
    return Parameters.from_dict(GOLDEN[case]["params"])


@pytest.mark.parametrize("case", sorted(GOLDEN))
def test_oracle_reproduces_reference_golden(case):
    prm = _params(case)
    cfg = prm.oracle_cfg()
    cfg["non_physical_behavior"] = "print_warning"
    left, right = prm.grid_bounds
    orc = Oracle(cfg, prm.n_cells, left, right)
    U = orc.initial_condition("tgv")
    cfl = float(prm.get("flow_solver/courant_friedrichs_lewy_number"))
    dt = tgv_constant_dt(cfl, left, right, prm.n_cells, prm.poly_degree)
    final = float(prm.get("flow_solver/final_time"))
    run_to_final_time(orc.rk_step, U, dt, final)
    ke, eps = orc.integrals(U)[[0, 2]]
    ke_ref, eps_ref = _expected(case)
    assert abs(ke - ke_ref) / ke_ref <= TOL
    assert abs(eps - eps_ref) / eps_ref <= TOL


@pytest.mark.gpu
def test_gpu_reproduces_reference_golden_gll():
    from philip_b200.dg import FlowSolver
    case = "viscous_taylor_green_vortex_energy_check_nsfr_gll_flux_nodes_quick"
    prm = _params(case)
    fs = FlowSolver(prm)
    fs.run()
    ke, _, eps, _ = fs.dg.integrals()
    ke_ref, eps_ref = _expected(case)
    print(f"GPU golden: KE rel err {abs(ke-ke_ref)/ke_ref:.3e}, eps rel err {abs(eps-eps_ref)/eps_ref:.3e}")
    assert abs(ke - ke_ref) / ke_ref <= TOL
    assert abs(eps - eps_ref) / eps_ref <= TOL
