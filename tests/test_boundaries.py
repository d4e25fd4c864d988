"""Boundary conditions of non-periodic meshes (assemble_boundary_term_strong, strong_dg.cpp:1582-2366;
the auxiliary boundary term, :725-866; Euler::boundary_face_values, euler.cpp:1096-1560;
NavierStokes::boundary_face_values_viscous_flux, navier_stokes.cpp:1354-1432; the numerical fluxes'
on_boundary branches, viscous_numerical_flux.cpp:66-328).

CPU: the oracle's boundary states against an independent numpy restatement of the reference's
formulas (every boundary type, Navier-Stokes wall adiabatic and isothermal); the oracle's slip-wall
residual on [0, L]^3 equal to the periodic residual of the mirror-symmetric flow on [-L, L]^3
restricted to [0, L]^3 (the reflected exterior state is the mirrored neighbour's state, so the whole
boundary term is pinned to the periodic path, which the golden energy values pin); the free stream
kept by farfield boundaries and a fluid at rest by Navier-Stokes walls.
GPU: residuals against the oracle within 1e-12 relative max-norm (Euler: every boundary type, split
and conservative, FR; Navier-Stokes: BR2 / SIPG / central, adiabatic and isothermal walls, slip walls,
FR auxiliary corrections, p = 1..6; collocated GLL nodes, GL flux nodes and overintegration, with and
without use_projected_entropy_variables_for_nsfr_boundary_term), the precision form within 1e-5,
three RK steps within 1e-11.
On GL nodes the mirror test holds for the conservative form, and for the split form with
use_projected_entropy_variables_for_nsfr_boundary_term; by default the split form's boundary flux
takes the interpolated face state and the interior faces the projected one (pinned below).
"""
import inspect
import math

import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.prm import Parameters

from helpers import perturbed_tgv, prm_dict, rel_max_err

GAMMA = 1.4


def _params(**kw):
    """prm_dict's keywords, plus any .prm key given by its name (e.g. flux_nodes_type,
    "euler/angle_of_attack")."""
    named = inspect.signature(prm_dict).parameters
    extra = {k: kw.pop(k) for k in list(kw) if k not in named}
    d = prm_dict(**kw)
    d.update(extra)
    return Parameters.from_dict(d)


# ------------------------------------------------------------------ numpy restatement of the states
def _prim(u):
    rho = u[0]
    v = u[1:4] / rho
    p = (GAMMA - 1) * (u[4] - 0.5 * rho * np.dot(v, v))
    return rho, v, p


def _cons(rho, v, p):
    return np.array([rho, *(rho * v), p / (GAMMA - 1) + 0.5 * rho * np.dot(v, v)])


def _free_stream(mach, aoa_deg):
    a = aoa_deg * math.pi / 180.0
    return 1.0, np.array([math.cos(a), math.sin(a), 0.0]), 1.0 / (GAMMA * mach * mach)


def _restated_state(bt, n, u, mach, aoa):
    """Euler::boundary_face_values for outward unit normal n (euler.cpp:1096-1560)."""
    g1 = GAMMA - 1
    rho, v, p = _prim(u)
    rho_f, v_f, p_f = _free_stream(mach, aoa)
    t_f = GAMMA * p_f / rho_f * mach * mach
    total_p = p_f * (1 + 0.5 * g1 * mach * mach) ** (GAMMA / g1)
    total_t = t_f * (total_p / p_f) ** (g1 / GAMMA)
    if bt in (1001, 1006):                         # slip wall: reflect the normal velocity
        return _cons(rho, v - 2.0 * np.dot(v, n) * n, p)
    if bt == 1005:
        return _cons(rho_f, v_f, p_f)
    if bt == 1007:
        return u.copy()
    if bt == 1004:                                 # Riemann invariants
        c, cf = math.sqrt(GAMMA * p / rho), math.sqrt(GAMMA * p_f / rho_f)
        r_out = np.dot(v, n) + 2 * c / g1
        r_inc = np.dot(v_f, n) - 2 * cf / g1
        vn, cb = 0.5 * (r_out + r_inc), 0.25 * g1 * (r_out - r_inc)
        if abs(vn) >= abs(cb):
            return _cons(rho_f, v_f, p_f) if vn < 0 else u.copy()
        rs, vs, ps = (rho_f, v_f, p_f) if vn < 0 else (rho, v, p)
        rb = (cb * cb / GAMMA / (ps * rs ** -GAMMA)) ** (1 / g1)
        return _cons(rb, vs - np.dot(vs, n) * n + vn * n, cb * cb * rb / GAMMA)
    if bt == 1002:                                 # back pressure 0.99 of the inlet static pressure
        mach_i = np.linalg.norm(v) / math.sqrt(GAMMA * p / rho)
        if mach_i > 1:
            return u.copy()
        p_b = 0.99 * total_p * (1 + 0.5 * g1 * mach * mach) ** (-GAMMA / g1)
        t_i = GAMMA * mach * mach * p / rho
        return _cons(GAMMA * mach * mach * p_b / t_i, v, p_b)
    if bt == 1003:                                 # inflow along -n
        m = -n
        if mach < 1:
            r_pos = np.dot(v, m) + 2 * math.sqrt(GAMMA * p / rho) / g1
            H = u[4] / rho + p / rho
            a, b, c = 1 + 2 / g1, -2 * r_pos, 0.5 * g1 * (r_pos * r_pos - 2 * H)
            cb = max(-b / (2 * a) + math.sqrt(b * b - 4 * a * c) / (2 * a),
                     -b / (2 * a) - math.sqrt(b * b - 4 * a * c) / (2 * a))
            vmag = r_pos - 2 * cb / g1
            rad = 1 + 0.5 * g1 * (vmag / cb) ** 2
            p_b, t_b = total_p * rad ** (-GAMMA / g1), total_t / rad
            return _cons(GAMMA * mach * mach * p_b / t_b, vmag * m, p_b)
        rad = 1 + 0.5 * g1 * mach * mach
        p_b, t_b = total_p * rad ** (-GAMMA / g1), total_t / rad
        rho_b = GAMMA * mach * mach * p_b / t_b
        return _cons(rho_b, -mach * math.sqrt(GAMMA * p_b / rho_b) * n, p_b)
    raise ValueError(bt)


def _restated_viscous_state(bt, u, g, mach, thermal, t_wall):
    """NavierStokes::boundary_face_values_viscous_flux (navier_stokes.cpp:1354-1432)."""
    if bt == 1006:
        return u.copy(), g.copy()
    ub = np.array([u[0], -u[1], -u[2], -u[3], u[4]])
    gb = g.copy()
    if thermal == "adiabatic":
        gb[4] = 0.0
    else:
        rho, v, p = _prim(u)
        t_ext = 2 * t_wall - GAMMA * mach * mach * p / rho
        ub = _cons(rho, -v, rho * t_ext / (GAMMA * mach * mach))
    return ub, gb


@pytest.mark.parametrize("mach,aoa", [(0.3, 10.0), (1.7, -25.0)])
def test_oracle_boundary_states_match_restatement(mach, aoa):
    rng = np.random.default_rng(int(mach * 10))
    errs = {}
    for thermal, t_wall in (("adiabatic", 1.0), ("isothermal", 1.3)):
        prm = _params(pde="navier_stokes", mach=mach, **{"euler/angle_of_attack": aoa,
                      "navier_stokes/thermal_boundary_condition_type": thermal,
                      "navier_stokes/nondimensionalized_isothermal_wall_temperature": t_wall})
        orc = Oracle(prm.oracle_cfg(), 2, 0.0, 1.0)
        for trial in range(40):
            n = rng.standard_normal(3)
            n /= np.linalg.norm(n)
            rho = 0.5 + rng.random()
            speed = mach * math.sqrt(GAMMA * (1.0 / (GAMMA * mach * mach)) / 1.0)
            v = rng.standard_normal(3) * speed * (0.2 + 2.0 * rng.random())
            p = (1.0 / (GAMMA * mach * mach)) * (0.5 + rng.random())
            u = _cons(rho, v, p)
            g = rng.standard_normal((5, 3))
            for bt in (1001, 1002, 1003, 1004, 1005, 1006, 1007):
                uc, uv, gv = orc.boundary_values(bt, n, u, g)
                ref = _restated_state(bt, n, u, mach, aoa)
                errs[bt] = max(errs.get(bt, 0.0), rel_max_err(uc, ref))
                if bt in (1001, 1006):
                    rv, rg = _restated_viscous_state(bt, u, g, mach, thermal, t_wall)
                    key = (bt, thermal)
                    errs[key] = max(errs.get(key, 0.0), rel_max_err(uv, rv), rel_max_err(gv, rg))
    print({str(k): f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) <= 1e-13


def _mirror(U, n, N1):
    """The state on [0, L]^3 (n^3 cells, lexicographic) reflected into the 2n^3-cell cube [-L, L]^3:
    a reflection across x_d = 0 reverses the nodes along d and negates the momentum along d."""
    Us = U.reshape(n, n, n, 5, N1, N1, N1)          # [k][j][i][s][z][y][x]
    B = np.zeros((2 * n, 2 * n, 2 * n, 5, N1, N1, N1))
    for K in range(2 * n):
        for J in range(2 * n):
            for I in range(2 * n):
                src = [A - n if A >= n else n - 1 - A for A in (I, J, K)]
                c = Us[src[2], src[1], src[0]].copy()
                if I < n:
                    c = c[:, :, :, ::-1]; c[1] *= -1
                if J < n:
                    c = c[:, :, ::-1, :]; c[2] *= -1
                if K < n:
                    c = c[:, ::-1, :, :]; c[3] *= -1
                B[K, J, I] = c
    return B.reshape(-1)


PROJ = "use_projected_entropy_variables_for_nsfr_boundary_term"
MIRROR_CASES = [
    ("split_CH_roe_p2", dict(poly_degree=2, split=True, two_point="CH", conv="roe"), "wall"),
    ("split_IR_ec_p3", dict(poly_degree=3, split=True, two_point="IR", conv="two_point_flux"), "slip_wall"),
    ("conservative_roe_p3", dict(poly_degree=3, split=False, conv="roe"), "wall"),
    ("conservative_lxf_cHU_p2", dict(poly_degree=2, split=False, conv="lax_friedrichs", fr="cHU"), "slip_wall"),
    ("gl_conservative_roe_p2", dict(poly_degree=2, split=False, conv="roe", flux_nodes_type="GL"), "wall"),
    ("gll_overint1_conservative_roe_p2", dict(poly_degree=2, split=False, conv="roe", overintegration=1), "wall"),
    # the uncollocated split form's interior faces take the projected entropy variables' face
    # state: a boundary mirrors them only with the flag that gives its flux the same state
    ("gl_split_CH_roe_p3_projected", dict(poly_degree=3, split=True, conv="roe", flux_nodes_type="GL",
                                          **{PROJ: "true"}), "slip_wall"),
    ("gl_overint1_split_IR_ec_p2_projected", dict(poly_degree=2, split=True, two_point="IR", conv="two_point_flux",
                                                  flux_nodes_type="GL", overintegration=1, **{PROJ: "true"}), "wall"),
]


@pytest.mark.parametrize("name,kw,bt", MIRROR_CASES, ids=[c[0] for c in MIRROR_CASES])
def test_oracle_slip_wall_is_the_mirrored_periodic_flow(name, kw, bt):
    prm = _params(pde="euler", **kw)
    cfg = prm.oracle_cfg()
    n, N1, L = 2, kw["poly_degree"] + 1, 1.0
    walls = Oracle(cfg, n, 0.0, L, "lexicographic", boundaries=[bt] * 6)
    cube = Oracle(cfg, 2 * n, -L, L, "lexicographic")
    U = perturbed_tgv(walls, seed=len(name), amp=0.05)
    Rw = walls.residual(U)
    Rc = cube.residual(_mirror(U, n, N1)).reshape(2 * n, 2 * n, 2 * n, 5, N1 ** 3)[n:, n:, n:].reshape(-1)
    err = rel_max_err(Rw, Rc)
    print(f"{name}: walls vs mirrored periodic cube {err:.2e}")
    assert err <= 1e-13


def test_oracle_uncollocated_split_boundary_takes_the_interpolated_state_by_default():
    """Without use_projected_entropy_variables_for_nsfr_boundary_term the boundary flux of the GL
    split form takes the interpolated face state (strong_dg.cpp:2255-2273), which differs from the
    projected one of the interior faces: the mirror no longer holds."""
    prm = _params(pde="euler", poly_degree=3, split=True, conv="roe", flux_nodes_type="GL")
    cfg = prm.oracle_cfg()
    n, N1 = 2, 4
    walls = Oracle(cfg, n, 0.0, 1.0, "lexicographic", boundaries=["slip_wall"] * 6)
    cube = Oracle(cfg, 2 * n, -1.0, 1.0, "lexicographic")
    U = perturbed_tgv(walls, seed=2, amp=0.05)
    Rc = cube.residual(_mirror(U, n, N1)).reshape(2 * n, 2 * n, 2 * n, 5, N1 ** 3)[n:, n:, n:].reshape(-1)
    err = rel_max_err(walls.residual(U), Rc)
    print(f"GL split, interpolated boundary state: differs from the mirror by {err:.2e}")
    assert err > 1e-5


def _uniform(orc, rho, v, p):
    U = np.zeros(orc.ndofs).reshape(-1, 5, orc.nd ** 3)
    for s, val in enumerate(_cons(rho, np.asarray(v, dtype=float), p)):
        U[:, s, :] = val
    return U.reshape(-1)


@pytest.mark.parametrize("bt", ["farfield", "riemann_farfield"])
def test_oracle_farfield_keeps_the_free_stream(bt):
    mach, aoa = 0.4, 30.0
    prm = _params(pde="euler", poly_degree=3, split=False, conv="roe", mach=mach, **{"euler/angle_of_attack": aoa})
    orc = Oracle(prm.oracle_cfg(), 2, 0.0, 1.0, boundaries=[bt] * 6)
    U = _uniform(orc, *_free_stream(mach, aoa))
    R = orc.residual(U)
    scale = 1.0 / (GAMMA * mach * mach)     # the pressure flux
    print(f"{bt}: max |R| / p_inf = {np.max(np.abs(R)) / scale:.2e}")
    assert np.max(np.abs(R)) <= 1e-13 * scale


@pytest.mark.parametrize("thermal", ["adiabatic", "isothermal"])
def test_oracle_navier_stokes_wall_keeps_a_fluid_at_rest(thermal):
    mach = 0.1
    p = 1.0 / (GAMMA * mach * mach)
    prm = _params(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2", mach=mach,
                  **{"navier_stokes/thermal_boundary_condition_type": thermal,
                     "navier_stokes/nondimensionalized_isothermal_wall_temperature": 1.0})
    orc = Oracle(prm.oracle_cfg(), 2, 0.0, 1.0, boundaries=["wall"] * 6)
    U = _uniform(orc, 1.0, [0.0, 0.0, 0.0], p)    # temperature gam M^2 p / rho = 1 = T_wall
    R = orc.residual(U)
    print(f"{thermal}: max |R| / p = {np.max(np.abs(R)) / p:.2e}")
    assert np.max(np.abs(R)) <= 1e-13 * p


# curvilinear cells (the sine-warped cube: the warp vanishes on the cube's sides, so boundary faces
# stay flat while the metric varies along them)
def _curved(kw, warp, bnd):
    prm = _params(**kw)
    return prm, Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, warp=warp, boundaries=bnd)


CURVED_PIN = [
    ("euler_split_riemann_walls", dict(pde="euler", poly_degree=3, n_cells=3),
     ["riemann_farfield", "riemann_farfield", "wall", "wall", "periodic", "periodic"]),
    ("ns_br2_walls", dict(pde="navier_stokes", poly_degree=2, n_cells=3, diss="bassi_rebay_2"),
     ["periodic", "periodic", "wall", "wall", "slip_wall", "slip_wall"]),
    ("ns_central_isothermal", dict(pde="navier_stokes", poly_degree=3, n_cells=2, diss="central_visc_flux",
                                   **{"navier_stokes/thermal_boundary_condition_type": "isothermal"}), ["wall"] * 6),
    ("gl_ns_br2_walls", dict(pde="navier_stokes", poly_degree=2, n_cells=3, diss="bassi_rebay_2",
                             flux_nodes_type="GL"), ["slip_wall"] * 2 + ["wall"] * 2 + ["periodic"] * 2),
    ("gl_euler_conservative_riemann", dict(pde="euler", poly_degree=3, n_cells=2, split=False, conv="roe",
                                           flux_nodes_type="GL"), ["riemann_farfield"] * 2 + ["wall"] * 4),
]


@pytest.mark.parametrize("name,kw,bnd", CURVED_PIN, ids=[c[0] for c in CURVED_PIN])
def test_oracle_curvilinear_boundaries_vanishing_warp(name, kw, bnd):
    """The curvilinear boundary terms (normals and |C n| from the face metric) reduce to the affine
    ones as the warp vanishes."""
    _, affine = _curved(kw, 0.0, bnd)
    _, curved = _curved(kw, 1e-300, bnd)
    U = _flow_state(affine, seed=3)
    err = rel_max_err(curved.residual(U), affine.residual(U))
    print(f"{name}: vanishing warp vs affine {err:.2e}")
    assert err <= 1e-13


@pytest.mark.parametrize("bt,nodes", [("farfield", "GLL"), ("riemann_farfield", "GLL"), ("riemann_farfield", "GL")])
def test_oracle_curvilinear_farfield_keeps_the_free_stream(bt, nodes):
    mach, aoa = 0.4, 30.0
    prm, orc = _curved(dict(pde="euler", poly_degree=3, n_cells=3, split=False, conv="roe", mach=mach,
                            flux_nodes_type=nodes, **{"euler/angle_of_attack": aoa}), 0.1, [bt] * 6)
    R = orc.residual(_uniform(orc, *_free_stream(mach, aoa)))
    scale = 1.0 / (GAMMA * mach * mach)
    print(f"{bt}, curvilinear: max |R| / p_inf = {np.max(np.abs(R)) / scale:.2e}")
    assert np.max(np.abs(R)) <= 1e-12 * scale


def test_oracle_curvilinear_walls_keep_a_parallel_uniform_flow():
    """Walls on the y sides (flat: the warp vanishes there) and a uniform flow with v_y = 0: the slip
    wall's exterior state is the interior one, and the warped interior keeps the free stream."""
    prm, orc = _curved(dict(pde="euler", poly_degree=3, n_cells=3), 0.1, WALLS_Y)
    p = 1.0 / (GAMMA * 0.01)
    R = orc.residual(_uniform(orc, 1.0, [0.6, 0.0, -0.3], p))
    print(f"curvilinear walls, parallel uniform flow: max |R| / p = {np.max(np.abs(R)) / p:.2e}")
    assert np.max(np.abs(R)) <= 1e-12 * p


# ------------------------------------------------------------------------------- GPU
def _flow_state(orc, seed):
    """Perturbed TGV with a mean flow along x (so that inflow and outflow boundaries see one)."""
    U = perturbed_tgv(orc, seed=seed, amp=0.02).reshape(-1, 5, orc.nd ** 3)
    rho = U[:, 0].copy()
    ke_old = 0.5 * (U[:, 1] ** 2 + U[:, 2] ** 2 + U[:, 3] ** 2) / rho
    U[:, 1] += 0.5 * rho
    U[:, 4] += 0.5 * (U[:, 1] ** 2 + U[:, 2] ** 2 + U[:, 3] ** 2) / rho - ke_old
    return U.reshape(-1)


GPU_CASES = [
    ("euler_split_CHroe_p3_walls_y", dict(pde="euler", poly_degree=3),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("euler_conservative_roe_p2_riemann_x", dict(pde="euler", poly_degree=2, split=False, conv="roe"),
     ["riemann_farfield", "riemann_farfield", "slip_wall", "slip_wall", "periodic", "periodic"]),
    ("euler_split_IR_ec_p4_mixed", dict(pde="euler", poly_degree=4, two_point="IR", conv="two_point_flux"),
     ["farfield", "farfield", "extrapolation", "extrapolation", "wall", "wall"]),
    ("euler_conservative_lxf_cHU_p5_in_out", dict(pde="euler", poly_degree=5, split=False, conv="lax_friedrichs",
                                                  fr="cHU"),
     ["inflow", "pressure_outflow", "slip_wall", "slip_wall", "slip_wall", "slip_wall"]),
    ("euler_split_KG_lxf_p1_all_riemann", dict(pde="euler", poly_degree=1, two_point="KG",
                                               conv="two_point_flux_with_lax_friedrichs_dissipation"),
     ["riemann_farfield"] * 6),
    ("ns_br2_split_p3_channel", dict(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2"),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("ns_sipg_conservative_p2_isothermal", dict(pde="navier_stokes", poly_degree=2, split=False, conv="roe",
                                                **{"navier_stokes/thermal_boundary_condition_type": "isothermal",
                                                   "navier_stokes/nondimensionalized_isothermal_wall_temperature": 1.1}),
     ["periodic", "periodic", "wall", "wall", "slip_wall", "slip_wall"]),
    ("ns_central_split_p4_box", dict(pde="navier_stokes", poly_degree=4, diss="central_visc_flux"),
     ["wall"] * 6),
    ("ns_br2_kSD_p2_walls_x", dict(pde="navier_stokes", poly_degree=2, diss="bassi_rebay_2", fr_aux="kSD"),
     ["wall", "wall", "periodic", "periodic", "periodic", "periodic"]),
    ("ns_sipg_split_p5_slip", dict(pde="navier_stokes", poly_degree=5),
     ["slip_wall", "slip_wall", "wall", "wall", "periodic", "periodic"]),
    ("ns_br2_split_p6_walls_z", dict(pde="navier_stokes", poly_degree=6, diss="bassi_rebay_2", n_cells=2),
     ["periodic", "periodic", "periodic", "periodic", "wall", "wall"]),
    ("ns_sipg_split_p1_box", dict(pde="navier_stokes", poly_degree=1, n_cells=4), ["wall"] * 6),
    # GL flux nodes (the reference's default) and overintegration
    ("gl_euler_split_CHroe_p3_walls_y", dict(pde="euler", poly_degree=3, flux_nodes_type="GL"),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("gl_euler_conservative_roe_p2_mixed", dict(pde="euler", poly_degree=2, split=False, conv="roe",
                                                flux_nodes_type="GL"),
     ["inflow", "pressure_outflow", "riemann_farfield", "riemann_farfield", "farfield", "extrapolation"]),
    ("gl_euler_split_IR_p2_projected", dict(pde="euler", poly_degree=2, two_point="IR", conv="two_point_flux",
                                            flux_nodes_type="GL", **{PROJ: "true"}),
     ["slip_wall", "slip_wall", "riemann_farfield", "riemann_farfield", "periodic", "periodic"]),
    ("gl_ns_br2_split_p3_channel", dict(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2",
                                        flux_nodes_type="GL"),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("gl_ns_sipg_conservative_p2_isothermal", dict(pde="navier_stokes", poly_degree=2, split=False, conv="roe",
                                                   flux_nodes_type="GL",
                                                   **{"navier_stokes/thermal_boundary_condition_type": "isothermal",
                                                      "navier_stokes/nondimensionalized_isothermal_wall_temperature": 0.9}),
     ["wall", "wall", "slip_wall", "slip_wall", "periodic", "periodic"]),
    ("gll_overint1_ns_central_split_p2_box", dict(pde="navier_stokes", poly_degree=2, diss="central_visc_flux",
                                                  overintegration=1), ["wall"] * 6),
    ("gl_ns_br2_split_p4_projected_kHU", dict(pde="navier_stokes", poly_degree=4, diss="bassi_rebay_2",
                                              flux_nodes_type="GL", fr_aux="kHU", n_cells=2, **{PROJ: "true"}),
     ["wall", "wall", "periodic", "periodic", "slip_wall", "slip_wall"]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,bnd", GPU_CASES, ids=[c[0] for c in GPU_CASES])
def test_gpu_boundary_residual_matches_oracle(name, kw, bnd):
    from philip_b200.dg import DGStrong
    kw = dict(kw)
    kw.setdefault("n_cells", 3)
    prm = _params(**kw)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, boundaries=bnd)
    dg = DGStrong(prm, boundaries=bnd)
    U = _flow_state(orc, seed=len(name))
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    print(f"{name}: residual rel max err {err:.3e}")
    assert err <= 1e-12


CURVED_GPU = [
    ("curved_euler_split_CHroe_p3_walls_y", dict(pde="euler", poly_degree=3),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("curved_euler_conservative_roe_p2_riemann", dict(pde="euler", poly_degree=2, split=False, conv="roe"),
     ["riemann_farfield", "riemann_farfield", "periodic", "periodic", "slip_wall", "slip_wall"]),
    ("curved_euler_split_IR_p4_inflow_outflow", dict(pde="euler", poly_degree=4, two_point="IR",
                                                     conv="two_point_flux", n_cells=2),
     ["inflow", "pressure_outflow", "slip_wall", "slip_wall", "farfield", "extrapolation"]),
    ("curved_ns_br2_split_p3_channel", dict(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2"),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("curved_ns_central_split_p2_isothermal_box", dict(pde="navier_stokes", poly_degree=2, diss="central_visc_flux",
                                                       **{"navier_stokes/thermal_boundary_condition_type":
                                                          "isothermal"}), ["wall"] * 6),
    ("curved_ns_br2_split_p5_slip", dict(pde="navier_stokes", poly_degree=5, diss="bassi_rebay_2", n_cells=2),
     ["slip_wall", "slip_wall", "wall", "wall", "periodic", "periodic"]),
    # GL flux nodes and overintegration on curved cells
    ("curved_gl_euler_split_CHroe_p3_walls_y", dict(pde="euler", poly_degree=3, flux_nodes_type="GL"),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("curved_gl_euler_conservative_roe_p2_mixed", dict(pde="euler", poly_degree=2, split=False, conv="roe",
                                                       flux_nodes_type="GL"),
     ["inflow", "pressure_outflow", "riemann_farfield", "riemann_farfield", "slip_wall", "slip_wall"]),
    ("curved_gl_ns_br2_split_p3_channel", dict(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2",
                                               flux_nodes_type="GL"),
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("curved_gll_overint1_ns_central_split_p2_isothermal", dict(pde="navier_stokes", poly_degree=2,
                                                                diss="central_visc_flux", overintegration=1,
                                                                **{"navier_stokes/thermal_boundary_condition_type":
                                                                   "isothermal"}), ["wall"] * 6),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,bnd", CURVED_GPU, ids=[c[0] for c in CURVED_GPU])
def test_gpu_curvilinear_boundary_residual_matches_oracle(name, kw, bnd):
    from philip_b200.dg import DGStrong
    kw = dict(kw)
    kw.setdefault("n_cells", 3)
    prm, orc = _curved(kw, 0.1, bnd)
    dg = DGStrong(prm, warp=0.1, boundaries=bnd)
    U = _flow_state(orc, seed=len(name))
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    print(f"{name}: residual rel max err {err:.3e}")
    assert err <= 1e-12


@pytest.mark.gpu
def test_gpu_curvilinear_boundary_steps_and_precision_form():
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    bnd = ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]
    prm, orc = _curved(dict(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2"), 0.1, bnd)
    U = _flow_state(orc, seed=8)
    dg32 = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL, warp=0.1, boundaries=bnd)
    err32 = rel_max_err(dg32.residual_of(U), orc.residual(U))
    dg = DGStrong(prm, warp=0.1, boundaries=bnd)
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    Uo = U.copy()
    for _ in range(3):
        ode.step_in_time(1e-3)
        orc.rk_step(Uo, 1e-3)
    err = rel_max_err(dg.solution, Uo)
    print(f"curvilinear channel: precision form {err32:.3e}, three RK4 steps {err:.3e}")
    assert err32 <= 1e-5 and err <= 1e-11


@pytest.mark.gpu
def test_gpu_boundary_precision_form_close_to_oracle():
    from philip_b200.dg import DGStrong
    bnd = ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]
    prm = _params(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2")
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, boundaries=bnd)
    dg = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL, boundaries=bnd)
    U = _flow_state(orc, seed=4)
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    print(f"channel walls, precision form: residual rel err {err:.3e}")
    assert err <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ns_channel", "euler_riemann", "gl_ns_channel"])
def test_gpu_boundary_rk_steps_match_oracle(case):
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    if case in ("ns_channel", "gl_ns_channel"):
        prm = _params(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2",
                      flux_nodes_type="GL" if case == "gl_ns_channel" else "GLL")
        bnd = ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]
    else:
        prm = _params(pde="euler", poly_degree=3, split=False, conv="roe", rk="ssprk3_ex")
        bnd = ["riemann_farfield", "riemann_farfield", "slip_wall", "slip_wall", "farfield", "farfield"]
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, boundaries=bnd)
    dg = DGStrong(prm, boundaries=bnd)
    U = _flow_state(orc, seed=7)
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    Uo = U.copy()
    for _ in range(3):
        ode.step_in_time(1e-3)
        orc.rk_step(Uo, 1e-3)
    err = rel_max_err(dg.solution, Uo)
    print(f"{case}: three RK steps rel err {err:.3e}")
    assert err <= 1e-11


# ------------------------------------------------------------------ refusals (no GPU needed)
def _mesh(prm, bnd, **kw):
    m = _lib.PhMeshDesc(prm.n_cells, 0, *prm.grid_bounds)
    m.grid_degree = prm.poly_degree
    for f, t in enumerate(_lib.boundary_ids(bnd)):
        m.boundary_type[f] = t
    for k, v in kw.items():
        setattr(m, k, v)
    return m


WALLS_Y = ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]
REFUSED = [
    ("navier_stokes_farfield", dict(pde="navier_stokes", diss="bassi_rebay_2"),
     ["riemann_farfield", "riemann_farfield", "periodic", "periodic", "periodic", "periodic"], None, {},
     _lib.PH_ERR_UNSUPPORTED, "1006"),
    ("unpaired_periodic_side", dict(), ["wall", "periodic", "periodic", "periodic", "periodic", "periodic"], None, {},
     _lib.PH_ERR_INVALID, "periodic on both sides"),
    ("unknown_boundary_id", dict(), [1000, 1000, 0, 0, 0, 0], None, {}, _lib.PH_ERR_INVALID, "1001..1007"),
    ("side_slip", dict(), WALLS_Y, lambda p: setattr(p, "side_slip_angle", 2.0), {}, _lib.PH_ERR_INVALID,
     "side_slip_angle"),
]


@pytest.mark.parametrize("name,prm_kw,bnd,edit,mesh_kw,code,text", REFUSED, ids=[r[0] for r in REFUSED])
def test_boundary_configurations_outside_the_path_are_refused(name, prm_kw, bnd, edit, mesh_kw, code, text):
    import ctypes
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict(**prm_kw))
    p = prm.to_ph_params()
    if edit:
        edit(p)
    m = _mesh(prm, bnd, **mesh_kw)
    h = ctypes.c_void_p()
    rc = L.ph_ctx_create(ctypes.byref(m), ctypes.byref(p), None, ctypes.byref(h))
    msg = L.ph_last_error().decode()
    print(f"{name}: rc {rc}, {msg}")
    assert rc == code and text in msg


def test_entry_points_and_non_periodic_meshes():
    """The no-allocation residual takes periodic meshes; a batch takes boundaries on its split-form
    Euler solves (their slot holds one boundary type per boundary face besides the periodic
    slot's arrays) and refuses a Navier-Stokes farfield as contexts do."""
    import ctypes
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict())
    p = prm.to_ph_params()
    m = _mesh(prm, WALLS_Y)
    dummy = ctypes.c_void_p(16)   # never dereferenced: the checks come first
    assert L.ph_residual_noalloc(ctypes.byref(m), ctypes.byref(p), dummy, dummy, None) == _lib.PH_ERR_UNSUPPORTED
    assert b"periodic" in L.ph_last_error()
    walls, periodic = ctypes.c_size_t(), ctypes.c_size_t()
    assert L.ph_batch_bytes(ctypes.byref(m), ctypes.byref(p), ctypes.byref(walls)) == _lib.PH_OK
    mp = _mesh(prm, ["periodic"] * 6)
    assert L.ph_batch_bytes(ctypes.byref(mp), ctypes.byref(p), ctypes.byref(periodic)) == _lib.PH_OK
    nb = 2 * prm.n_cells ** 2
    assert walls.value - periodic.value == (nb * 4 + 255) // 256 * 256
    ns = Parameters.from_dict(prm_dict(pde="navier_stokes", diss="bassi_rebay_2"))
    q = ns.to_ph_params()
    mf = _mesh(ns, ["riemann_farfield", "riemann_farfield", "periodic", "periodic", "periodic", "periodic"])
    assert L.ph_batch_bytes(ctypes.byref(mf), ctypes.byref(q), ctypes.byref(walls)) == _lib.PH_ERR_UNSUPPORTED


BATCH_BND = [
    ("walls_y", ["periodic", "periodic", "wall", "wall", "periodic", "periodic"]),
    ("slip_farfield_outflow", ["slip_wall", "slip_wall", "farfield", "farfield", "pressure_outflow", "inflow"]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("warp", [0.0, 0.1], ids=["affine", "warped"])
@pytest.mark.parametrize("precision", [_lib.PH_FP64, _lib.PH_FP32_RESIDUAL], ids=["fp64", "fp32"])
def test_batched_solves_with_boundaries_match_single_solves(precision, warp):
    """Split-form Euler solves with boundary faces inside a batch, beside a periodic solve of the
    same order: the bounded solves' group runs the boundary-face instance of the batched kernel on
    all its tiles (a context runs it on the tiles that touch a boundary and the periodic kernel on
    the rest). The two instances evaluate an interior face alike: the results are bitwise the
    single-solve contexts' in FP64, affine and curved (in the precision form measured bitwise on
    affine cells and within 2.5e-9 on curved ones, where the compiler contracts FP32 products
    differently in the two kernel bodies; held to 1e-6, as the periodic batch is)."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.serve import Batch
    prm = _params(poly_degree=3, n_cells=4)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    U0 = orc.initial_condition("tgv")
    dt, nsteps = 2e-3, 6
    b = Batch(1 << 30, precision)
    cases = BATCH_BND + [("periodic", ["periodic"] * 6)]
    slots = [b.admit(_mesh(prm, bnd, warp=warp), prm.to_ph_params(precision), U0, dt, nsteps) for _, bnd in cases]
    b.step(10 ** 6)
    assert b.active == 0
    tol = 0.0 if precision == _lib.PH_FP64 else 1e-6
    for (name, bnd), s in zip(cases, slots):
        Ub = b.state(s, U0.size)
        dg = DGStrong(prm, precision=precision, warp=warp, boundaries=None if name == "periodic" else bnd)
        dg.solution = U0
        RungeKuttaODESolver(dg).step_in_time(dt, nsteps=nsteps)
        Ua = dg.solution
        err = float(np.max(np.abs(Ub - Ua)) / np.max(np.abs(Ua)))
        print(f"{name} warp {warp}: batch vs context rel max err {err:.3e} (bitwise {np.array_equal(Ub, Ua)})")
        assert b.status(s) == 0 and dg.status() == 0
        if precision == _lib.PH_FP64:
            assert np.array_equal(Ub, Ua)
        assert err <= tol
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["RK4_3_5_3SStar", "RK3_2_5F_3SStarPlus", "relaxation"])
def test_gpu_boundary_low_storage_and_relaxation_steps_match_oracle(method):
    """The low-storage (3S* / 3S*+) and relaxation RK solvers on a wall-bounded mesh: the stage
    kernels' epilogues are the periodic ones, the boundary tiles run the boundary-face instances."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    kw = dict(pde="navier_stokes", poly_degree=3, diss="bassi_rebay_2", two_point="CH", conv="two_point_flux")
    if method == "relaxation":
        kw["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true"
    else:
        kw["rk"] = method
    prm = _params(**kw)
    bnd = ["periodic", "periodic", "wall", "wall", "slip_wall", "slip_wall"]
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, boundaries=bnd)
    dg = DGStrong(prm, boundaries=bnd)
    U = _flow_state(orc, seed=5)
    dg.solution = U
    ode = RungeKuttaODESolver(dg)
    Uo = U.copy()
    for _ in range(3):
        ode.step_in_time(1e-3)
        orc.rk_step(Uo, 1e-3)
    err = rel_max_err(dg.solution, Uo)
    extra = ""
    if method == "relaxation":
        g_err = abs(ode.relaxation_parameter - orc.rrk_gamma()) / orc.rrk_gamma()
        extra = f", gamma rel err {g_err:.2e}"
        assert g_err <= 1e-5
    print(f"walls, {method}: three steps rel err {err:.3e}{extra}")
    assert err <= (5e-9 if method == "relaxation" else 1e-11)


@pytest.mark.gpu
def test_gpu_slip_walls_run_the_mirrored_periodic_taylor_green_vortex():
    """The inviscid Taylor-Green vortex is mirror-symmetric about the planes x, y, z = 0 and pi: on
    [0, pi]^3 with slip walls all around it must stay the octant of the periodic run on
    [-pi, pi]^3 (the same cells), step after step (twenty RK4 steps)."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    n, p = 3, 3
    walls = _params(pde="euler", poly_degree=p, n_cells=n, left=0.0, right=math.pi)
    cube = _params(pde="euler", poly_degree=p, n_cells=2 * n, left=-math.pi, right=math.pi)
    ow = Oracle(walls.oracle_cfg(), n, 0.0, math.pi, "lexicographic", boundaries=["slip_wall"] * 6)
    U = ow.initial_condition("tgv")
    dw = DGStrong(walls, cell_order=1, boundaries=["slip_wall"] * 6)
    dc = DGStrong(cube, cell_order=1)
    dw.solution = U
    dc.solution = _mirror(U, n, p + 1)
    dt = 0.1 * math.pi / n / (p + 1) / 11.0
    RungeKuttaODESolver(dw).step_in_time(dt, nsteps=20)
    RungeKuttaODESolver(dc).step_in_time(dt, nsteps=20)
    N1 = p + 1
    octant = dc.solution.reshape(2 * n, 2 * n, 2 * n, 5, N1 ** 3)[n:, n:, n:].reshape(-1)
    err = rel_max_err(dw.solution, octant)
    change = rel_max_err(dw.solution, U)
    print(f"slip-walled octant vs periodic cube after 20 RK4 steps: {err:.2e} (the state changed by {change:.2e})")
    assert err <= 1e-12 and change > 1e-6
