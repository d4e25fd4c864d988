"""Parity of the CUDA path (through the C-ABI) with the CPU oracle.

Tolerance: the FP64 path must match the oracle's residual within 1e-12 relative
max-norm (max |R_gpu - R_oracle| / max |R_oracle|), as the residual contract asks.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.dg import DGStrong, RungeKuttaODESolver
from philip_b200.prm import Parameters

from helpers import prm_dict, perturbed_tgv, rel_max_err

RTOL = 1e-12

CASES = [
    # name, kwargs
    ("euler_CH_roe_p3_morton", dict(poly_degree=3, n_cells=4)),
    ("euler_IR_ec_p2_lex", dict(poly_degree=2, n_cells=3, two_point="IR", conv="two_point_flux")),
    ("euler_KG_lxf_p4", dict(poly_degree=4, n_cells=2, two_point="KG", conv="two_point_flux_with_lax_friedrichs_dissipation")),
    ("euler_Ra_roe_p5", dict(poly_degree=5, n_cells=2, two_point="Ra")),
    ("euler_conservative_roe_p3", dict(poly_degree=3, n_cells=3, split=False, conv="roe")),
    ("euler_conservative_lxf_p1", dict(poly_degree=1, n_cells=4, split=False, conv="lax_friedrichs")),
    ("euler_conservative_central_p6", dict(poly_degree=6, n_cells=2, split=False, conv="central_flux")),
    ("ns_CH_roe_br2_p3", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2")),
    ("ns_IR_ec_sipg_p2", dict(poly_degree=2, n_cells=4, pde="navier_stokes", two_point="IR", conv="two_point_flux")),
    ("ns_conservative_roe_sipg_p3", dict(poly_degree=3, n_cells=3, pde="navier_stokes", split=False, conv="roe")),
    ("ns_CH_br2_p5", dict(poly_degree=5, n_cells=2, pde="navier_stokes", diss="bassi_rebay_2")),
    ("ns_KG_lxf_central_p4", dict(poly_degree=4, n_cells=2, pde="navier_stokes", two_point="KG",
                                  conv="two_point_flux_with_lax_friedrichs_dissipation", diss="central_visc_flux")),
]


def _pair(kw, precision=_lib.PH_FP64):
    prm = Parameters.from_dict(prm_dict(**kw))
    cfg = prm.oracle_cfg()
    left, right = prm.grid_bounds
    orc = Oracle(cfg, prm.n_cells, left, right)
    dg = DGStrong(prm, precision=precision)
    return prm, orc, dg


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_residual_parity(name, kw):
    prm, orc, dg = _pair(kw)
    assert np.array_equal(dg.cell_ijk(), orc.cell_ijk())
    assert np.allclose(dg.node_coordinates(), orc.node_xyz(), rtol=0, atol=1e-14)
    U = perturbed_tgv(orc, seed=len(name))
    R_orc = orc.residual(U)
    R_gpu = dg.residual_of(U)
    err = rel_max_err(R_gpu, R_orc)
    print(f"{name}: residual rel max err {err:.3e}")
    assert err <= RTOL
    # bitwise repeatable
    assert np.array_equal(dg.residual_of(U), R_gpu)


@pytest.mark.gpu
@pytest.mark.parametrize("fr", ["cDG", "cHU", "cPlus", "cSD"])
def test_inverse_mass_and_rk_step_parity(fr):
    kw = dict(poly_degree=3, n_cells=3, pde="navier_stokes", diss="bassi_rebay_2", fr=fr)
    prm, orc, dg = _pair(kw)
    U = perturbed_tgv(orc, seed=7)
    R = orc.residual(U)
    k_orc = orc.inverse_mass(R)
    k_gpu = np.empty_like(R)
    dg.apply_inverse_global_mass_matrix(R, k_gpu)
    assert rel_max_err(k_gpu, k_orc) <= RTOL
    for rk in ("rk4_ex", "ssprk3_ex", "heun2_ex", "euler_ex"):
        kw2 = dict(kw, rk=rk)
        prm, orc, dg = _pair(kw2)
        U0 = perturbed_tgv(orc, seed=3)
        dt = 1e-3
        Uo = U0.copy()
        orc.rk_step(Uo, dt)
        dg.solution = U0
        RungeKuttaODESolver(dg).step_in_time(dt)
        Ug = dg.solution
        du_orc = Uo - U0
        err = float(np.max(np.abs((Ug - U0) - du_orc)) / np.max(np.abs(du_orc)))
        print(f"fr={fr} rk={rk}: step increment rel err {err:.3e}")
        assert err <= 1e-11


@pytest.mark.gpu
def test_integrals_parity():
    prm, orc, dg = _pair(dict(poly_degree=3, n_cells=4, pde="navier_stokes"))
    U = perturbed_tgv(orc, seed=11, amp=0.01)
    dg.solution = U
    q_gpu = dg.integrals()
    q_orc = orc.integrals(U)
    for i in range(4):
        assert abs(q_gpu[i] - q_orc[i]) <= 1e-12 * abs(q_orc[i]) + 1e-300, (i, q_gpu[i], q_orc[i])


@pytest.mark.gpu
def test_nonphysical_status_flag():
    prm, orc, dg = _pair(dict(poly_degree=2, n_cells=2))
    U = orc.initial_condition("tgv")
    U[4 * 27 + 5] = -1.0      # negative total energy at one node -> negative pressure
    dg.solution = U
    dg.assemble_residual()
    assert dg.status() & 1
    assert dg.status() == 0   # reading clears it


@pytest.mark.gpu
@pytest.mark.parametrize("rk", ["rk4_ex", "ssprk3_ex", "heun2_ex"])
@pytest.mark.parametrize("visc", [False, True])
def test_multistep_parity_and_clean_status(rk, visc):
    """Several steps at the TGV time step: the state follows the oracle and no
    non-physical state is flagged."""
    kw = dict(poly_degree=3, n_cells=4, rk=rk, pde="navier_stokes" if visc else "euler",
              diss="bassi_rebay_2")
    prm, orc, dg = _pair(kw)
    U = orc.initial_condition("tgv")
    dg.solution = U
    dt = 0.1 * 6.28318530717958623200 / (4 * 4) / 11.0   # acoustic CFL 0.1 (|v| + c ~ 11)
    ode = RungeKuttaODESolver(dg)
    for step in range(6):
        orc.rk_step(U, dt)
        ode.step_in_time(dt)
        st = dg.status()
        Ug = dg.solution
        err = rel_max_err(Ug, U)
        print(f"{rk} visc={visc} step {step}: rel err {err:.3e} status {st}")
        assert st == 0
        assert err <= 1e-12


@pytest.mark.gpu
def test_graph_replayed_steps_match_direct_steps():
    """ph_rk_step on a caller-given stream replays one captured RK step; the result is bitwise
    the directly launched steps'."""
    import torch
    kw = dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2")
    prm = Parameters.from_dict(prm_dict(**kw))
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    U0 = orc.initial_condition("tgv")
    dt = 0.1 * 6.28318530717958623200 / 16 / 11.0
    direct = DGStrong(prm)                       # legacy default stream: direct launches
    direct.solution = U0
    RungeKuttaODESolver(direct).step_in_time(dt, nsteps=5)
    s = torch.cuda.Stream()
    graphed = DGStrong(prm, stream=s.cuda_stream)
    graphed.solution = U0
    RungeKuttaODESolver(graphed).step_in_time(dt, nsteps=5)
    RungeKuttaODESolver(graphed).step_in_time(dt, nsteps=3)    # replays the cached graph
    RungeKuttaODESolver(direct).step_in_time(dt, nsteps=3)
    s.synchronize()
    assert np.array_equal(graphed.solution, direct.solution)
