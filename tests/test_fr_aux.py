"""FR auxiliary correction (flux_reconstruction_aux, all_parameters.cpp:141, :635-642): the
auxiliary equation's inverse mass is (M + K_aux)^-1 with K_aux = k (D^p)^T M D^p
(local_Flux_Reconstruction_operator_aux, operators.cpp:1796-1860) instead of M^-1, applied in
each direction of the affine cell (dg_base.cpp:4089-4219).

CPU: the oracle's lifted gradient with K_aux equals its kDG gradient carried through
(M + K_aux)^-1 M in each direction, with M, D and k built here independently in numpy
(k from get_Huynh_g2_parameter, get_spectral_difference_parameter, get_c_negative_FR_parameter,
get_c_negative_divided_by_two_FR_parameter and get_c_plus_parameter, operators.cpp:1560-1624).
GPU: the residual against the oracle within 1e-12 relative max-norm on collocated GLL nodes
(every order 1..6, so both forms of the auxiliary kernel), on GL flux nodes and with
overintegration; the precision form within 1e-5; three RK4 steps within 1e-11.

k10Thousand makes M + k K ill-conditioned (condition number 5.8e6 at p = 2, 1.3e9 at p = 3):
two correct inverses then differ by about cond * eps, so its cases take the bar
10 * cond * eps (the condition number computed here) instead of 1e-12.
"""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.prm import Parameters

from helpers import perturbed_tgv, prm_dict, rel_max_err


def _params(fr_aux, nodes="GLL", overintegration=0, **kw):
    d = prm_dict(fr_aux=fr_aux, **kw)
    d["flux_nodes_type"] = nodes
    d["overintegration"] = overintegration
    return Parameters.from_dict(d)


def _k(name, p):
    pf = math.factorial(p)
    cp = math.factorial(2 * p) / pf ** 2
    neg = -2.0 / ((2.0 * p + 1.0) * (pf * cp) ** 2) / 2.0
    return {
        "kDG": 0.0,
        "kSD": 2.0 * p / ((p + 1.0) * ((2.0 * p + 1.0) * (pf * cp) ** 2)) / 2.0,
        "kHU": 2.0 * (p + 1) / (p * ((2.0 * p + 1.0) * (pf * cp) ** 2)) / 2.0,
        "kNegative": neg,
        "kNegative2": neg / 2.0,
        "kPlus": {2: 0.186, 3: 3.67e-3, 4: 4.79e-5, 5: 4.24e-7}.get(p, float("nan")) / 2.0 / (2.0 ** p) ** 2,
        "k10Thousand": 10000.0,
    }[name]


def _lagrange(nodes, x):
    """Values and derivatives of the Lagrange basis on `nodes` at the points x."""
    n = len(nodes)
    V = np.ones((len(x), n))
    dV = np.zeros((len(x), n))
    for j in range(n):
        for m in range(n):
            if m == j:
                continue
            term = np.ones(len(x)) / (nodes[j] - nodes[m])
            for l in range(n):
                if l != j and l != m:
                    term *= (x - nodes[l]) / (nodes[j] - nodes[l])
            dV[:, j] += term
            V[:, j] *= (x - nodes[m]) / (nodes[j] - nodes[m])
    return V, dV


def _aux_mass(orc, k, p):
    """M and M + k K on the oracle's 1-D support points and flux nodes."""
    xs, xq, wq = orc.ops()
    chi, dchi = _lagrange(xs, xq)
    M = chi.T @ (wq[:, None] * chi)
    D = np.linalg.solve(M, chi.T @ (wq[:, None] * dchi))
    Dp = np.linalg.matrix_power(D, p)
    return M, M + k * (Dp.T @ M @ Dp)


def _bar(orc, aux, p):
    M, Ma = _aux_mass(orc, _k(aux, p), p)
    return max(1e-12, 10.0 * np.linalg.cond(Ma) * np.finfo(float).eps)


AUX_CASES = [
    ("gll_kHU_p3", "kHU", "GLL", 0, dict(poly_degree=3, n_cells=2)),
    ("gll_kSD_p4", "kSD", "GLL", 0, dict(poly_degree=4, n_cells=2, split=False, conv="roe")),
    ("gll_k10Thousand_p2", "k10Thousand", "GLL", 0, dict(poly_degree=2, n_cells=3)),
    ("gl_kPlus_p3", "kPlus", "GL", 0, dict(poly_degree=3, n_cells=2)),
    ("gl_overint1_kNegative2_p2", "kNegative2", "GL", 1, dict(poly_degree=2, n_cells=2, diss="bassi_rebay_2")),
]


@pytest.mark.parametrize("name,aux,nodes,over,kw", AUX_CASES, ids=[c[0] for c in AUX_CASES])
def test_oracle_aux_gradient_is_the_dg_gradient_through_the_aux_fr_mass(name, aux, nodes, over, kw):
    kw = dict(kw, pde="navier_stokes")
    p = kw["poly_degree"]
    base = _params("kDG", nodes, over, **kw)
    corr = _params(aux, nodes, over, **kw)
    o0 = Oracle(base.oracle_cfg(), base.n_cells, *base.grid_bounds)
    ok = Oracle(corr.oracle_cfg(), corr.n_cells, *corr.grid_bounds)
    U = perturbed_tgv(o0, seed=len(name))
    o0.residual(U)
    ok.residual(U)
    n = p + 1
    q0 = o0.aux().reshape(3, -1, 5, n, n, n)        # [d][cell][state][z][y][x]
    qk = ok.aux().reshape(3, -1, 5, n, n, n)
    M, Ma = _aux_mass(ok, _k(aux, p), p)
    B = np.linalg.solve(Ma, M)
    expect = np.einsum("xa,yb,zc,dkscba->dkszyx", B, B, B, q0)
    err = rel_max_err(qk, expect)
    change = rel_max_err(qk, q0)
    bar = _bar(ok, aux, p)
    print(f"{name}: oracle vs restated transfer {err:.3e}, bar {bar:.1e} "
          f"(the correction changes q by {change:.3e})")
    assert err <= bar
    assert change > 1e-8


# ------------------------------------------------------------------------------- GPU
GPU_CASES = [
    ("gll_p1_kHU", "kHU", "GLL", 0, dict(poly_degree=1, n_cells=4)),
    ("gll_p2_kSD_roe_sipg", "kSD", "GLL", 0, dict(poly_degree=2, n_cells=3)),
    ("gll_p3_kHU_conservative_br2", "kHU", "GLL", 0, dict(poly_degree=3, n_cells=3, split=False, conv="roe",
                                                          diss="bassi_rebay_2")),
    ("gll_p2_k10Thousand", "k10Thousand", "GLL", 0, dict(poly_degree=2, n_cells=2)),
    ("gll_p4_kPlus_IR_central", "kPlus", "GLL", 0, dict(poly_degree=4, n_cells=2, two_point="IR",
                                                        conv="two_point_flux", diss="central_visc_flux")),
    ("gll_p5_kNegative", "kNegative", "GLL", 0, dict(poly_degree=5, n_cells=2)),
    ("gll_p6_kNegative2_cHU", "kNegative2", "GLL", 0, dict(poly_degree=6, n_cells=1, fr="cHU")),
    ("gl_p3_kHU_roe_sipg", "kHU", "GL", 0, dict(poly_degree=3, n_cells=2, split=False, conv="roe")),
    ("gl_overint1_p2_kSD_br2", "kSD", "GL", 1, dict(poly_degree=2, n_cells=3, diss="bassi_rebay_2")),
    ("gll_overint1_p3_kPlus", "kPlus", "GLL", 1, dict(poly_degree=3, n_cells=2)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,aux,nodes,over,kw", GPU_CASES, ids=[c[0] for c in GPU_CASES])
def test_gpu_fr_aux_residual_matches_oracle(name, aux, nodes, over, kw):
    from philip_b200.dg import DGStrong
    prm = _params(aux, nodes, over, pde="navier_stokes", **kw)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm)
    U = perturbed_tgv(orc, seed=len(name))
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    bar = _bar(orc, aux, kw["poly_degree"])
    print(f"{name}: residual rel max err {err:.3e}, bar {bar:.1e}")
    assert err <= bar


@pytest.mark.gpu
def test_gpu_fr_aux_precision_form_close_to_oracle():
    from philip_b200.dg import DGStrong
    prm = _params("kHU", poly_degree=3, n_cells=3, pde="navier_stokes", diss="bassi_rebay_2")
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL)
    U = perturbed_tgv(orc, seed=5)
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    print(f"kHU precision form: residual rel err {err:.3e}")
    assert err <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nodes", ["GLL", "GL"])
def test_gpu_fr_aux_rk_steps_match_oracle(nodes):
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    prm = _params("kSD", nodes, poly_degree=3, n_cells=2, pde="navier_stokes")
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm)
    U = perturbed_tgv(orc, seed=9)
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    Uo = U.copy()
    for _ in range(3):
        ode.step_in_time(1e-3)
        orc.rk_step(Uo, 1e-3)
    err = rel_max_err(dg.solution, Uo)
    print(f"kSD {nodes}: three RK4 steps rel err {err:.3e}")
    assert err <= 1e-11
