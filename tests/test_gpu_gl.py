"""Uncollocated flux nodes on the GPU: Gauss-Legendre flux nodes (the reference's default
flux_nodes_type, all_parameters.cpp:77-80) and overintegration, where the interpolation,
entropy projection, flux-node differentiation and FR mass inverse are dense 1-D operators.

Bars (as the collocated path's): residual relative max-norm 1e-12 against the oracle, the
inverse mass and RK steps 1e-11, and the reference's own golden energy checks on GL nodes
(viscous_taylor_green_vortex_energy_check_strong_quick.prm:66-67 and
..._nsfr_gl_flux_nodes_quick.prm:59-60, taylor_green_vortex_energy_check.cpp:37-44) within 1e-10
through the C-ABI.
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200.dg import DGStrong, FlowSolver, RungeKuttaODESolver
from philip_b200.prm import Parameters

from helpers import perturbed_tgv, prm_dict, rel_max_err


def _gl(flux_nodes="GL", overintegration=0, **kw):
    d = prm_dict(**kw)
    d["flux_nodes_type"] = flux_nodes
    d["overintegration"] = overintegration
    return Parameters.from_dict(d)


CASES = [
    ("ns_strong_roe_sipg_p2", dict(poly_degree=2, n_cells=3, pde="navier_stokes", split=False, conv="roe")),
    ("ns_nsfr_ir_sipg_p2", dict(poly_degree=2, n_cells=3, pde="navier_stokes", two_point="IR", conv="two_point_flux")),
    ("euler_ch_roe_p3", dict(poly_degree=3, n_cells=2)),
    ("euler_ch_roe_p5", dict(poly_degree=5, n_cells=2)),
    ("ns_ch_roe_br2_p3", dict(poly_degree=3, n_cells=2, pde="navier_stokes", diss="bassi_rebay_2")),
    ("ns_ra_lxf_central_p4", dict(poly_degree=4, n_cells=2, pde="navier_stokes", two_point="Ra",
                                  conv="two_point_flux_with_lax_friedrichs_dissipation", diss="central_visc_flux")),
    ("euler_kg_ec_p1", dict(poly_degree=1, n_cells=3, two_point="KG", conv="two_point_flux")),
    ("euler_conservative_lxf_chu_p3", dict(poly_degree=3, n_cells=2, split=False, conv="lax_friedrichs", fr="cHU")),
    ("ns_conservative_central_cplus_p2", dict(poly_degree=2, n_cells=3, pde="navier_stokes", split=False,
                                             conv="central_flux", fr="cPlus")),
    ("euler_ch_p6", dict(poly_degree=6, n_cells=1)),
]
OVER = [
    ("gll_overint1_euler_ch_p2", "GLL", 1, dict(poly_degree=2, n_cells=3)),
    ("gll_overint2_ns_ch_br2_p3", "GLL", 2, dict(poly_degree=3, n_cells=2, pde="navier_stokes", diss="bassi_rebay_2")),
    ("gl_overint1_ns_strong_sipg_p3", "GL", 1, dict(poly_degree=3, n_cells=2, pde="navier_stokes", split=False,
                                                   conv="roe")),
    ("gl_overint2_euler_ir_p4", "GL", 2, dict(poly_degree=4, n_cells=2, two_point="IR", conv="two_point_flux")),
]


def _check_residual(prm, seed):
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm)
    U = perturbed_tgv(orc, seed=seed)
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    return err, orc, dg, U


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_gl_residual_matches_oracle(name, kw):
    err, *_ = _check_residual(_gl(**kw), seed=len(name))
    print(f"{name}: residual rel max err {err:.3e}")
    assert err <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name,nodes,over,kw", OVER, ids=[c[0] for c in OVER])
def test_overintegration_residual_matches_oracle(name, nodes, over, kw):
    err, *_ = _check_residual(_gl(nodes, over, **kw), seed=len(name))
    print(f"{name}: residual rel max err {err:.3e}")
    assert err <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("fr", ["cDG", "cHU", "cSD"])
def test_gl_inverse_mass_and_rk_steps_match_oracle(fr):
    prm = _gl(poly_degree=3, n_cells=2, pde="navier_stokes", fr=fr, split=False, conv="roe")
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm)
    U = perturbed_tgv(orc, seed=7)
    R = orc.residual(U)
    out = np.zeros_like(R)
    dg.apply_inverse_global_mass_matrix(R, out)
    e_m = rel_max_err(out, orc.inverse_mass(R))
    dt = 1e-3
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    Uo = U.copy()
    for _ in range(3):
        ode.step_in_time(dt)
        orc.rk_step(Uo, dt)
    e_rk = rel_max_err(dg.solution, Uo)
    print(f"GL {fr}: inverse mass {e_m:.3e}, three RK4 steps {e_rk:.3e}")
    assert e_m <= 1e-11 and e_rk <= 1e-11


GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tgv_energy_check.json")))
GL_GOLDEN = ["viscous_taylor_green_vortex_energy_check_strong_quick",
             "viscous_taylor_green_vortex_energy_check_nsfr_gl_flux_nodes_quick"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GL_GOLDEN)
def test_gpu_reproduces_reference_golden_gl(case):
    p = GOLDEN[case]["params"]
    prm = Parameters.from_dict(p)
    assert prm.get("flux_nodes_type") == "GL"
    fs = FlowSolver(prm)
    fs.run()
    ke, _, eps, _ = fs.dg.integrals()
    ke_ref = float(p["flow_solver/taylor_green_vortex/expected_kinetic_energy_at_final_time"])
    eps_ref = float(p["flow_solver/taylor_green_vortex/expected_theoretical_dissipation_rate_at_final_time"])
    print(f"{case}: KE rel err {abs(ke - ke_ref) / ke_ref:.3e}, eps rel err {abs(eps - eps_ref) / eps_ref:.3e}")
    assert abs(ke - ke_ref) / ke_ref <= 1e-10
    assert abs(eps - eps_ref) / eps_ref <= 1e-10
