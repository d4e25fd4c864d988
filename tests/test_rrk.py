"""Relaxation Runge-Kutta, root-finding form for the Euler / Navier-Stokes entropy
(RootFindingRRKODESolver, root_finding_rrk_ode_solver.cpp; RKNumEntropy,
runge_kutta_store_entropy.cpp; RungeKuttaODESolver::adjust_time_step,
runge_kutta_ode_solver.cpp:102-110).

The reference has no golden value for it. The oracle's restatement is pinned by the property
the method exists for: with an entropy-conservative semi-discretisation (split form with the
Chandrashekar flux and the entropy-conserving face flux, no dissipation, periodic) the
relaxed step conserves the integrated numerical entropy to rounding, where plain RK4 drifts by
its time-integration error; with dissipation the entropy decays by gamma times the
estimate.

The CUDA path is held to the oracle with bounds set by the conditioning of the root, not by
the arithmetic: r(gamma) = eta(u_n + gamma d) - eta(u_n) - gamma est is a difference of two
integrated entropies of magnitude 1e3 whose rounding (summation order, the log and pow of two
math libraries) is about 1e-13, while r changes with gamma only by about 1e-7 per unit near
its root for these small steps (the entropy changes by 1e-5 or less per step). Two correct
evaluations therefore place the root about 1e-6 apart (measured on B200: at most 4.0e-6), and
the states differ by that times d = dt sum b_i k_i. The bounds below are 1e-5 for gamma and,
for the state, a sum over the steps taken of 2e-9 plus twice the roots' relative difference
times the step's relative size (the runs are not re-synchronised, so differences carry over);
the entropy-conservation tests hold the method itself to rounding.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200.prm import Parameters

from helpers import prm_dict

EC = dict(two_point="CH", conv="two_point_flux")


WARP = 0.1   # the sine-warped curvilinear cube: x_i += 0.1 sin x sin y sin z on [0, 2 pi]^3


def _oracle(rrk, nodes="GLL", overintegration=0, warp=0.0, **kw):
    d = prm_dict(**kw)
    d["flux_nodes_type"] = nodes
    d["overintegration"] = overintegration
    prm = Parameters.from_dict(d)
    cfg = prm.oracle_cfg()
    cfg["use_relaxation_runge_kutta"] = rrk
    if warp:
        return Oracle(cfg, prm.n_cells, *prm.grid_bounds, warp=warp)
    return Oracle(cfg, prm.n_cells, *prm.grid_bounds)


def _entropy_drift(rrk, steps=5, dt=0.02, **kw):
    o = _oracle(rrk, **kw)
    U = o.initial_condition("tgv")
    e0 = o.numerical_entropy(U)
    for _ in range(steps):
        o.rk_step(U, dt)
    return (o.numerical_entropy(U) - e0) / abs(e0), o.rrk_gamma()


def test_oracle_rrk_conserves_entropy_of_the_entropy_conservative_scheme():
    plain, g_plain = _entropy_drift(False, poly_degree=3, n_cells=3, **EC)
    relaxed, g = _entropy_drift(True, poly_degree=3, n_cells=3, **EC)
    print(f"entropy drift over 5 steps: plain RK4 {plain:.3e}, relaxed {relaxed:.3e} (gamma {g:.12f})")
    assert abs(plain) > 1e-11
    assert abs(relaxed) <= 1e-13
    assert g_plain == 1.0 and abs(g - 1.0) < 0.05 and g != 1.0


@pytest.mark.parametrize("nodes,over", [("GL", 0), ("GL", 1), ("GLL", 2)])
def test_oracle_rrk_on_uncollocated_nodes_conserves_entropy(nodes, over):
    """Uncollocated flux nodes: the estimate sum_i b_i v_hat_i^T M k_i with the entropy variables
    projected on the solution basis and M = chi^T W J chi vanishes for the entropy-conserving split
    form (its v_hat^T R is zero), so the relaxed steps keep the numerical entropy integrated at the
    flux nodes."""
    plain, _ = _entropy_drift(False, poly_degree=3, n_cells=2, nodes=nodes, overintegration=over, **EC)
    relaxed, g = _entropy_drift(True, poly_degree=3, n_cells=2, nodes=nodes, overintegration=over, **EC)
    print(f"{nodes} overint {over}: entropy drift over 5 steps: plain {plain:.3e}, relaxed {relaxed:.3e} "
          f"(gamma {g:.12f})")
    assert abs(plain) > 1e-11
    assert abs(relaxed) <= 1e-13
    assert abs(g - 1.0) < 0.05 and g != 1.0


@pytest.mark.parametrize("nodes", ["GLL", "GL"])
def test_oracle_rrk_on_a_curvilinear_mesh_conserves_entropy(nodes):
    """The sine-warped cube: the estimate's mass is chi^T W det(J) chi at the flux nodes. Without
    overintegration the weight-adjusted inverse mass of the curved cells equals the inverse of that
    mass (GLL: both diagonal; GL: chi is square), so the relaxed entropy-conservative steps keep
    the numerical entropy. (With overintegration the two differ and the relaxed steps do not
    conserve it exactly: a property of the method, which the GPU reproduces step by step.)"""
    plain, _ = _entropy_drift(False, poly_degree=3, n_cells=2, nodes=nodes, warp=WARP, **EC)
    relaxed, g = _entropy_drift(True, poly_degree=3, n_cells=2, nodes=nodes, warp=WARP, **EC)
    print(f"warped {nodes}: entropy drift over 5 steps: plain {plain:.3e}, relaxed {relaxed:.3e} (gamma {g:.12f})")
    assert abs(plain) > 1e-11
    assert abs(relaxed) <= 1e-13


def test_oracle_rrk_with_dissipation_and_the_gamma_scaled_time():
    o = _oracle(True, poly_degree=2, n_cells=3, rk="ssprk3_ex")
    U = o.initial_condition("tgv")
    e0 = o.numerical_entropy(U)
    o.rk_step(U, 0.02)
    assert o.numerical_entropy(U) < e0          # Roe dissipation: entropy decays
    assert 0.5 < o.rrk_gamma() < 1.5


def test_relaxation_parameters_follow_the_reference_keys():
    d = prm_dict(poly_degree=2, n_cells=2)
    assert not Parameters.from_dict(d).use_relaxation_runge_kutta
    d["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true"
    d["ODE solver/rrk root solver/relaxation_runge_kutta_root_tolerance"] = "1e-11"
    p = Parameters.from_dict(d)
    q = p.to_ph_params()
    assert q.use_relaxation_runge_kutta == 1 and q.relaxation_runge_kutta_root_tolerance == 1e-11
    d2 = prm_dict(poly_degree=2, n_cells=2)
    d2["ODE solver/ode_solver_type"] = "rrk_explicit"      # the deprecated spelling
    assert Parameters.from_dict(d2).use_relaxation_runge_kutta


# ------------------------------------------------------------------------------- GPU

CASES = [
    ("euler_ec_rk4_p3", dict(poly_degree=3, n_cells=3, **EC), 0.02),
    ("euler_roe_ssprk3_p2", dict(poly_degree=2, n_cells=4, rk="ssprk3_ex"), 0.02),
    ("ns_br2_rk4_p3", dict(poly_degree=3, n_cells=3, pde="navier_stokes", diss="bassi_rebay_2"), 0.01),
    ("euler_ec_heun_p4", dict(poly_degree=4, n_cells=2, rk="heun2_ex", **EC), 0.01),
    # uncollocated flux nodes; the first is the reference's 3D_navier_stokes_RRK_check.prm setting
    # (GL, cPlus, Ranocha two-point flux, SIPG, SSPRK3, p = 2, 4^3 cells)
    ("gl_ns_cplus_ra_sipg_ssprk3_p2", dict(poly_degree=2, n_cells=4, pde="navier_stokes", fr="cPlus", two_point="Ra",
                                          conv="two_point_flux", rk="ssprk3_ex", nodes="GL"), 0.01),
    ("gl_euler_ec_rk4_p3", dict(poly_degree=3, n_cells=2, nodes="GL", **EC), 0.02),
    ("gll_overint1_euler_roe_rk4_p2", dict(poly_degree=2, n_cells=3, nodes="GLL", overintegration=1), 0.02),
]


def _pair(kw):
    from philip_b200.dg import DGStrong
    kw = dict(kw)
    nodes, over = kw.pop("nodes", "GLL"), kw.pop("overintegration", 0)
    d = prm_dict(**kw)
    d["flux_nodes_type"] = nodes
    d["overintegration"] = over
    d["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true"
    prm = Parameters.from_dict(d)
    cfg = prm.oracle_cfg()
    orc = Oracle(cfg, prm.n_cells, *prm.grid_bounds)
    return prm, orc, DGStrong(prm)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,dt", CASES, ids=[c[0] for c in CASES])
def test_rrk_steps_match_the_oracle(name, kw, dt):
    from philip_b200.dg import RungeKuttaODESolver
    prm, orc, dg = _pair(kw)
    U = orc.initial_condition("tgv")
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    t_orc = 0.0
    bound = 0.0
    for step in range(4):
        U_prev = U.copy()
        orc.rk_step(U, dt)
        t_orc += orc.rrk_gamma() * dt
        ode.step_in_time(dt)
        g_err = abs(ode.relaxation_parameter - orc.rrk_gamma()) / orc.rrk_gamma()
        Ug = dg.solution
        err = float(np.max(np.abs(Ug - U)) / np.max(np.abs(U)))
        # a relative difference g_err of the two roots moves the state by g_err gamma d, d the
        # step direction (u_{n+1} = u_n + gamma d): each step adds that plus the stages' own 2e-9
        # to the bound, since the two runs are not re-synchronised between steps
        rel_step = float(np.max(np.abs(U - U_prev)) / np.max(np.abs(U)))
        bound += 2e-9 + 2.0 * g_err * rel_step
        print(f"{name} step {step}: gamma {ode.relaxation_parameter:.15f} (oracle {orc.rrk_gamma():.15f}, "
              f"rel {g_err:.2e}), state rel err {err:.2e} (bound {bound:.1e})")
        assert g_err <= 1e-5
        assert err <= bound
        assert dg.status() == 0
    assert abs(ode.current_time - t_orc) <= 1e-5 * t_orc


@pytest.mark.gpu
@pytest.mark.parametrize("nodes,over", [("GLL", 0), ("GL", 0), ("GLL", 1)], ids=["gll", "gl", "gll_overint1"])
def test_rrk_conserves_entropy_on_the_gpu(nodes, over):
    """The entropy-conservative split form relaxed on the GPU conserves the numerical entropy
    (at the solution nodes when they are the flux nodes, at the flux nodes otherwise) to
    rounding over ten steps; unrelaxed RK4 does not."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    res = {}
    for rrk in (False, True):
        d = prm_dict(poly_degree=3, n_cells=4, **EC)
        d["flux_nodes_type"] = nodes
        d["overintegration"] = over
        d["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true" if rrk else "false"
        prm = Parameters.from_dict(d)
        orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
        dg = DGStrong(prm)
        dg.solution = orc.initial_condition("tgv")
        e0 = orc.numerical_entropy(dg.solution)
        RungeKuttaODESolver(dg).step_in_time(0.02, nsteps=10)
        res[rrk] = (orc.numerical_entropy(dg.solution) - e0) / abs(e0)
    print(f"{nodes} overintegration {over}: entropy drift over 10 steps: plain {res[False]:.3e}, "
          f"relaxed {res[True]:.3e}")
    assert abs(res[False]) > 1e-11
    assert abs(res[True]) <= 1e-12


WARPED_CASES = [
    ("warped_gll_euler_ec_rk4_p3", dict(poly_degree=3, n_cells=2, **EC), 0.02),
    ("warped_gl_euler_ec_rk4_p3", dict(poly_degree=3, n_cells=2, nodes="GL", **EC), 0.02),
    ("warped_gll_overint1_euler_roe_rk4_p2", dict(poly_degree=2, n_cells=3, nodes="GLL", overintegration=1), 0.02),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,dt", WARPED_CASES, ids=[c[0] for c in WARPED_CASES])
def test_rrk_on_a_curvilinear_mesh_matches_the_oracle(name, kw, dt):
    """Relaxation RK on the sine-warped cube (cDG): the GPU's roots and states follow the oracle's
    within the bounds of the affine comparison, and (without overintegration) the entropy-
    conservative scheme's relaxed steps conserve the numerical entropy on the GPU."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    kw = dict(kw)
    nodes, over = kw.pop("nodes", "GLL"), kw.pop("overintegration", 0)
    orc = _oracle(True, nodes=nodes, overintegration=over, warp=WARP, **kw)
    d = prm_dict(**kw)
    d["flux_nodes_type"] = nodes
    d["overintegration"] = over
    d["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true"
    dg = DGStrong(Parameters.from_dict(d), warp=WARP)
    U = orc.initial_condition("tgv")
    e0 = orc.numerical_entropy(U)
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    bound = 0.0
    for step in range(4):
        U_prev = U.copy()
        orc.rk_step(U, dt)
        ode.step_in_time(dt)
        g_err = abs(ode.relaxation_parameter - orc.rrk_gamma()) / orc.rrk_gamma()
        err = float(np.max(np.abs(dg.solution - U)) / np.max(np.abs(U)))
        rel_step = float(np.max(np.abs(U - U_prev)) / np.max(np.abs(U)))
        bound += 2e-9 + 2.0 * g_err * rel_step
        print(f"{name} step {step}: gamma {ode.relaxation_parameter:.15f} (oracle {orc.rrk_gamma():.15f}, "
              f"rel {g_err:.2e}), state rel err {err:.2e} (bound {bound:.1e})")
        assert g_err <= 1e-5
        assert err <= bound
        assert dg.status() == 0
    drift = (orc.numerical_entropy(dg.solution) - e0) / abs(e0)
    print(f"{name}: GPU entropy change over 4 relaxed steps {drift:.3e}")
    if kw.get("conv") == "two_point_flux" and over == 0:
        assert abs(drift) <= 1e-12
