"""Restart files (FlowSolver::output_restart_files / restart_computation_from_file,
flow_solver.cpp:58-100, :240-395): a run stopped after k steps and restarted from the
written restart-NNNNN.prm continues bitwise like the uninterrupted run."""
import os

import numpy as np
import pytest

from philip_b200.dg import FlowSolver, read_restart_state, restart_filename_without_extension
from philip_b200.prm import Parameters

from helpers import TWO_PI, prm_dict

pytestmark = pytest.mark.gpu


def test_restart_continues_bitwise(tmp_path):
    base = prm_dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2", cfl=0.05)
    base.update({"flow_solver/constant_time_step": 1e-3, "flow_solver/final_time": 6e-3,
                 "flow_solver/restart_files_directory_name": str(tmp_path)})
    straight = FlowSolver(Parameters.from_dict(base))
    straight.run()
    U_straight = straight.dg.solution

    first = dict(base, **{"flow_solver/final_time": 3e-3, "flow_solver/output_restart_files": True,
                          "flow_solver/output_restart_files_every_x_steps": 3})
    FlowSolver(Parameters.from_dict(first)).run()
    name = restart_filename_without_extension(1)
    prm_path = os.path.join(tmp_path, name + ".prm")
    assert os.path.exists(prm_path) and os.path.exists(os.path.join(tmp_path, name + ".sol"))
    U3, t3, it3, dt3 = read_restart_state(os.path.join(tmp_path, name + ".sol"))
    assert it3 == 3 and abs(t3 - 3e-3) < 1e-15 and dt3 == 1e-3

    restarted = Parameters.from_file(prm_path).with_values({"flow_solver/final_time": "6e-3",
                                                            "flow_solver/output_restart_files": "false"})
    assert restarted.get("flow_solver/restart_computation_from_file") == "true"
    second = FlowSolver(restarted)
    assert second.ode_solver.current_iteration == 3
    second.run()
    assert second.ode_solver.current_iteration == 6
    assert np.array_equal(second.dg.solution, U_straight)
    assert len(second.unsteady_data) == len(straight.unsteady_data)
