"""The flow solver's time loop on the device (ph_run): steps as ph_rk_step takes them, with the
four integrals reduced on the device every record_every steps (FlowSolver::run with
PeriodicTurbulence::compute_unsteady_data_and_write_to_table, periodic_turbulence.cpp:923-972).

The state after ph_run is bitwise the state after the same steps through ph_rk_step (on the
legacy stream, where every launch is direct, and on a caller-given stream, where each record
interval replays one captured graph); each row matches ph_integrals at that step within
1e-14 relative (the device sums the per-cell partials in a tree, the host in cell order)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200.dg import DGStrong, FlowSolver, RungeKuttaODESolver
from philip_b200.prm import Parameters

from helpers import TWO_PI, prm_dict

pytestmark = pytest.mark.gpu

CASES = [
    ("ns_rk4_p3", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 3, 4),
    ("euler_ssprk3_p2", dict(poly_degree=2, n_cells=4, rk="ssprk3_ex"), 2, 5),
    ("euler_forward_euler_p2", dict(poly_degree=2, n_cells=3, rk="euler_ex"), 3, 3),
    ("euler_lsrk_p3", dict(poly_degree=3, n_cells=3, rk="RK3_2_5F_3SStarPlus"), 2, 4),
]


def _setup(kw):
    prm = Parameters.from_dict(prm_dict(**kw))
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    return prm, orc.initial_condition("tgv")


def _close(a, b):
    return np.all(np.abs(a - b) <= 1e-14 * np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("name,kw,every,nrec", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("on_stream", [False, True], ids=["legacy_stream", "caller_stream"])
def test_run_matches_stepping_and_host_integrals(name, kw, every, nrec, on_stream):
    import torch
    prm, U0 = _setup(kw)
    dt = 0.1 * TWO_PI / 16 / 11.0
    nsteps = every * nrec + 1                    # one step after the last record
    s = torch.cuda.Stream() if on_stream else None
    dev = DGStrong(prm, stream=s.cuda_stream if s is not None else None)
    dev.solution = U0
    rows = RungeKuttaODESolver(dev).step_in_time_with_records(dt, nsteps, every)
    ref = DGStrong(prm)
    ref.solution = U0
    ode = RungeKuttaODESolver(ref)
    host_rows = []
    for _ in range(nrec):
        ode.step_in_time(dt, nsteps=every)
        host_rows.append((ode.current_time, *ref.integrals()))
    ode.step_in_time(dt)
    if s is not None:
        s.synchronize()
    assert np.array_equal(dev.solution, ref.solution)
    assert dev.status() == 0 and ref.status() == 0
    assert len(rows) == nrec
    for r, h in zip(rows, host_rows):
        assert r[0] == h[0]
        assert _close(np.array(r[1:]), np.array(h[1:])), (r, h)
    # a second run on the same context reuses the captured interval
    rows2 = RungeKuttaODESolver(dev).step_in_time_with_records(dt, every * 2, every)
    assert len(rows2) == 2 and all(np.isfinite(r[1]) for r in rows2)


def test_flow_solver_records_on_the_device():
    """FlowSolver.run with a constant time step records every record_every steps on the device;
    the rows and times equal a host loop's over the same steps (within 1e-14), the final state
    is bitwise the host loop's, and the clipped last step is taken on the host."""
    kw = dict(poly_degree=3, n_cells=4, pde="navier_stokes", final_time=0.05, cfl=0.01)
    prm = Parameters.from_dict(prm_dict(**kw))
    fs = FlowSolver(prm)
    dt = fs.time_step()
    fs.run(record_every=4)
    ref = FlowSolver(prm)
    ode = ref.ode_solver
    rows = [(ode.current_time, *ref.dg.integrals())]
    while ode.current_time < 0.05:
        step = min(dt, 0.05 - ode.current_time)
        ode.step_in_time(step)
        if ode.current_iteration % 4 == 0:
            rows.append((ode.current_time, *ref.dg.integrals()))
    assert abs(fs.ode_solver.current_time - 0.05) < 1e-15
    assert fs.dg.status() == 0 and np.all(np.isfinite(fs.dg.solution))
    assert fs.ode_solver.current_iteration == ode.current_iteration
    assert np.array_equal(fs.dg.solution, ref.dg.solution)
    assert len(fs.unsteady_data) == len(rows)
    for a, b in zip(fs.unsteady_data, rows):
        assert a[0] == b[0]
        assert _close(np.array(a[1:]), np.array(b[1:])), (a, b)
