"""Low-storage Runge-Kutta methods (LowStorageRungeKuttaODESolver,
low_storage_runge_kutta_ode_solver.cpp, tableaux low_storage_runge_kutta_methods.cpp).

The oracle's restated tableaux are pinned by the methods' convergence order on a smooth
inviscid TGV (a wrong coefficient drops the order); the CUDA path, whose stage update and
error reduction are fused into the residual kernel, is held to the oracle step by step and
in its error estimate."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200.prm import Parameters

from helpers import TWO_PI, perturbed_tgv, prm_dict, rel_max_err

METHODS = [("RK4_3_5_3SStar", 4), ("RK3_2_5F_3SStarPlus", 3), ("RK4_3_9F_3SStarPlus", 4),
           ("RK5_4_10F_3SStarPlus", 5)]


def _oracle(rk, **kw):
    prm = Parameters.from_dict(prm_dict(rk=rk, **kw))
    return prm, Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)


@pytest.mark.parametrize("rk,order", METHODS)
def test_oracle_tableau_convergence_order(rk, order):
    _, orc = _oracle(rk, poly_degree=2, n_cells=2, mach=0.3)
    U0 = orc.initial_condition("tgv")
    T = 0.4

    def run(n):
        U = U0.copy()
        for _ in range(n):
            orc.rk_step(U, T / n)
        return U
    ref = run(64)
    e1 = np.max(np.abs(run(8) - ref))
    e2 = np.max(np.abs(run(16) - ref))
    rate = np.log2(e1 / e2)
    print(f"{rk}: errors {e1:.3e} {e2:.3e}, observed order {rate:.2f}")
    assert rate > order - 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("rk,order", METHODS)
@pytest.mark.parametrize("visc", [False, True])
def test_lowstorage_steps_and_error_match_oracle(rk, order, visc):
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    kw = dict(poly_degree=3, n_cells=3, pde="navier_stokes" if visc else "euler", diss="bassi_rebay_2")
    prm, orc = _oracle(rk, **kw)
    dg = DGStrong(prm)
    ode = RungeKuttaODESolver(dg)
    U = perturbed_tgv(orc, seed=4, amp=0.005)
    dg.solution = U
    dt = 0.1 * TWO_PI / 12 / 11.0
    for step in range(3):
        orc.rk_step(U, dt)
        ode.step_in_time(dt)
        err = rel_max_err(dg.solution, U)
        w_gpu, w_orc = ode.error_norm(), orc.rk_error()
        print(f"{rk} visc={visc} step {step}: state rel err {err:.3e}, error norm {w_gpu:.6e} vs {w_orc:.6e}")
        assert err <= 1e-12
        assert abs(w_gpu - w_orc) <= 1e-8 * abs(w_orc) + 1e-300
        assert dg.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("rk,nodes,over,visc", [("RK3_2_5F_3SStarPlus", "GL", 0, True),
                                                ("RK4_3_5_3SStar", "GL", 0, False),
                                                ("RK5_4_10F_3SStarPlus", "GLL", 1, True)],
                         ids=["gl_ns_rk3_2_5f", "gl_euler_rk4_3_5", "gll_overint1_ns_rk5_4_10f"])
def test_lowstorage_on_uncollocated_flux_nodes(rk, nodes, over, visc):
    """The low-storage stage update and its error reduction in the uncollocated stage kernel's
    epilogue (one tile per cell): steps and error norm against the oracle."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    d = prm_dict(rk=rk, poly_degree=3, n_cells=2, pde="navier_stokes" if visc else "euler", diss="bassi_rebay_2")
    d["flux_nodes_type"] = nodes
    d["overintegration"] = over
    prm = Parameters.from_dict(d)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm)
    ode = RungeKuttaODESolver(dg)
    U = perturbed_tgv(orc, seed=6, amp=0.005)
    dg.solution = U
    dt = 0.1 * TWO_PI / 8 / 11.0
    for step in range(3):
        orc.rk_step(U, dt)
        ode.step_in_time(dt)
        err = rel_max_err(dg.solution, U)
        w_gpu, w_orc = ode.error_norm(), orc.rk_error()
        print(f"{rk} {nodes} overint {over} step {step}: state rel err {err:.3e}, error norm {w_gpu:.6e} "
              f"vs {w_orc:.6e}")
        assert err <= 1e-12
        assert abs(w_gpu - w_orc) <= 1e-8 * abs(w_orc) + 1e-300
        assert dg.status() == 0
