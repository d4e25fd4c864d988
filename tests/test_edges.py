"""Edge cases of the hot path: configurations outside the GPU path are refused with a message
(before any device work, so these run without a GPU), the smallest meshes (one periodic cell,
whose six faces are its own neighbours; p = 1) match the oracle, and at the default bench
size the RK step conserves the integrals of mass, momentum and energy (periodic cube,
conservative strong form: sum over the nodes of W det J u changes only by rounding).
"""
import ctypes

import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.prm import Parameters

from helpers import perturbed_tgv, prm_dict, rel_max_err


def _create(prm_kw=None, mesh_kw=None, edit=None):
    """ph_ctx_create on a parameter set edited at the C level; returns (rc, message)."""
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict(**(prm_kw or {})))
    p = prm.to_ph_params()
    if edit:
        edit(p)
    m = _lib.PhMeshDesc()
    m.n_cells_per_direction = prm.n_cells
    m.cell_order = 0
    m.left, m.right = prm.grid_bounds
    m.warp = 0.0
    m.grid_degree = prm.poly_degree
    for k, v in (mesh_kw or {}).items():
        setattr(m, k, v)
    h = ctypes.c_void_p()
    rc = L.ph_ctx_create(ctypes.byref(m), ctypes.byref(p), None, ctypes.byref(h))
    msg = L.ph_last_error().decode()
    if rc == 0:
        L.ph_ctx_destroy(h)
    return rc, msg


REFUSED = [
    ("gl_flux_nodes_precision_form", lambda p: (setattr(p, "flux_nodes_type", 0), setattr(p, "precision", 1)),
     _lib.PH_ERR_UNSUPPORTED, "FP64"),
    ("overintegration_3", lambda p: setattr(p, "overintegration", 3), _lib.PH_ERR_UNSUPPORTED, "overintegration"),
    ("gl_flux_nodes_p6_overintegration", lambda p: (setattr(p, "flux_nodes_type", 0), setattr(p, "poly_degree", 6),
                                                    setattr(p, "overintegration", 1)),
     _lib.PH_ERR_UNSUPPORTED, "<= 7"),
    ("degree_7", lambda p: setattr(p, "poly_degree", 7), _lib.PH_ERR_UNSUPPORTED, "poly_degree"),
    ("implicit_rk", lambda p: setattr(p, "runge_kutta_method", 4), _lib.PH_ERR_INVALID, "out of range"),
    ("ec_flux_without_split_form", lambda p: (setattr(p, "use_split_form", 0), setattr(p, "conv_num_flux", 3)),
     _lib.PH_ERR_INVALID, "split form"),
    ("rrk_with_kg", lambda p: (setattr(p, "use_relaxation_runge_kutta", 1), setattr(p, "two_point_num_flux_type", 0)),
     _lib.PH_ERR_UNSUPPORTED, "KG"),
    ("rrk_with_low_storage", lambda p: (setattr(p, "use_relaxation_runge_kutta", 1), setattr(p, "runge_kutta_method", 7)),
     _lib.PH_ERR_UNSUPPORTED, "Butcher"),
    ("rrk_in_precision_form", lambda p: (setattr(p, "use_relaxation_runge_kutta", 1), setattr(p, "precision", 1)),
     _lib.PH_ERR_UNSUPPORTED, "FP64"),
    ("kplus_aux_at_degree_6", lambda p: (setattr(p, "poly_degree", 6), setattr(p, "flux_reconstruction_aux", 5)),
     _lib.PH_ERR_UNSUPPORTED, "flux_reconstruction_aux"),
    ("aux_fr_type_7", lambda p: setattr(p, "flux_reconstruction_aux", 7), _lib.PH_ERR_INVALID, "out of range"),
]


@pytest.mark.parametrize("name,edit,code,text", REFUSED, ids=[r[0] for r in REFUSED])
def test_configurations_outside_the_path_are_refused(name, edit, code, text):
    rc, msg = _create(edit=edit)
    print(f"{name}: rc {rc}, {msg}")
    assert rc == code and text in msg


def test_curvilinear_navier_stokes_with_sipg_is_refused():
    """Curvilinear Navier-Stokes takes BR2 or the central viscous flux: the SIPG penalty uses the
    cell's extent along the face normal (dg_base.cpp:397-413), not restated on curved cells."""
    rc, msg = _create(prm_kw=dict(pde="navier_stokes"), mesh_kw=dict(warp=0.1))
    assert rc == _lib.PH_ERR_UNSUPPORTED and "bassi_rebay_2" in msg
    rc, msg = _create(prm_kw=dict(pde="navier_stokes", diss="bassi_rebay_2"), mesh_kw=dict(warp=0.1),
                      edit=lambda p: setattr(p, "flux_reconstruction_aux", 2))
    assert rc == _lib.PH_ERR_UNSUPPORTED and "kDG" in msg


def test_curvilinear_gl_navier_stokes_with_sipg_is_refused():
    """GL flux nodes on curvilinear cells, like GLL ones, take BR2 or the central viscous flux
    (an FR auxiliary correction is taken there: the uncollocated auxiliary kernel's weight-adjusted
    projection carries (M + K_aux)^-1)."""
    rc, msg = _create(prm_kw=dict(pde="navier_stokes"), mesh_kw=dict(warp=0.1),
                      edit=lambda p: setattr(p, "flux_nodes_type", 0))
    assert rc == _lib.PH_ERR_UNSUPPORTED and "bassi_rebay_2" in msg


def test_entry_points_without_contexts_refuse_gl_flux_nodes():
    """The batch, the server and the no-allocation residual run the collocated kernels only."""
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict())
    p = prm.to_ph_params()
    p.flux_nodes_type = 0
    m = _lib.PhMeshDesc(prm.n_cells, 0, *prm.grid_bounds)
    dummy = ctypes.c_void_p(16)
    assert L.ph_residual_noalloc(ctypes.byref(m), ctypes.byref(p), dummy, dummy, None) == _lib.PH_ERR_UNSUPPORTED
    nbytes = ctypes.c_size_t()
    assert L.ph_batch_bytes(ctypes.byref(m), ctypes.byref(p), ctypes.byref(nbytes)) == _lib.PH_ERR_UNSUPPORTED
    assert b"collocated" in L.ph_last_error()


BAD_MESHES = [
    ("recursive_order_n3", dict(n_cells_per_direction=3, cell_order=2), "power of two"),
    ("cell_order_3", dict(cell_order=3), "cell_order"),
    ("cell_order_negative", dict(cell_order=-1), "cell_order"),
    ("no_cells", dict(n_cells_per_direction=0), "bad mesh"),
]


@pytest.mark.parametrize("name,mesh_kw,text", BAD_MESHES, ids=[b[0] for b in BAD_MESHES])
def test_bad_meshes_are_refused_by_every_entry_point(name, mesh_kw, text):
    """A cell order the connectivity cannot build (the recursive-children order of a cube whose
    side is not a power of two would number cells past the mesh) is refused with
    PH_ERR_INVALID before any device work by ph_ctx_create, ph_residual_noalloc and
    ph_batch_bytes."""
    rc, msg = _create(mesh_kw=mesh_kw)
    assert rc == _lib.PH_ERR_INVALID and text in msg, (rc, msg)
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict())
    p = prm.to_ph_params()
    m = _lib.PhMeshDesc(prm.n_cells, 0, *prm.grid_bounds)
    for k, v in mesh_kw.items():
        setattr(m, k, v)
    dummy = ctypes.c_void_p(16)   # never dereferenced: the checks come first
    rc = L.ph_residual_noalloc(ctypes.byref(m), ctypes.byref(p), dummy, dummy, None)
    assert rc == _lib.PH_ERR_INVALID and text in L.ph_last_error().decode()
    nbytes = ctypes.c_size_t()
    rc = L.ph_batch_bytes(ctypes.byref(m), ctypes.byref(p), ctypes.byref(nbytes))
    assert rc == _lib.PH_ERR_INVALID and text in L.ph_last_error().decode()


def test_noalloc_refuses_what_the_context_refuses():
    """ph_residual_noalloc applies ph_ctx_create's parameter checks before any launch."""
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict())
    m = _lib.PhMeshDesc(prm.n_cells, 0, *prm.grid_bounds)
    dummy = ctypes.c_void_p(16)
    for field, value in (("pde_type", 2), ("two_point_num_flux_type", 7), ("conv_num_flux", 9), ("precision", 3),
                         ("poly_degree", 7)):
        p = prm.to_ph_params()
        setattr(p, field, value)
        rc = L.ph_residual_noalloc(ctypes.byref(m), ctypes.byref(p), dummy, dummy, None)
        assert rc in (_lib.PH_ERR_INVALID, _lib.PH_ERR_UNSUPPORTED), field


# ------------------------------------------------------------------------------- GPU

SMALL = [
    ("one_cell_euler_p3", dict(poly_degree=3, n_cells=1)),
    ("one_cell_ns_br2_p2", dict(poly_degree=2, n_cells=1, pde="navier_stokes", diss="bassi_rebay_2")),
    ("one_cell_ns_sipg_p5", dict(poly_degree=5, n_cells=1, pde="navier_stokes")),
    ("two_cells_p1", dict(poly_degree=1, n_cells=2)),
    ("two_cells_ns_p6", dict(poly_degree=6, n_cells=2, pde="navier_stokes", diss="bassi_rebay_2")),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", SMALL, ids=[s[0] for s in SMALL])
def test_smallest_meshes_match_the_oracle(name, kw):
    from philip_b200.dg import DGStrong
    prm = Parameters.from_dict(prm_dict(**kw))
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm)
    U = perturbed_tgv(orc, seed=len(name))
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    print(f"{name}: residual rel max err {err:.3e}")
    assert err <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(_lib.PH_FP64, 1e-12), (_lib.PH_FP32_RESIDUAL, 1e-10)],
                         ids=["fp64", "precision_form"])
def test_conservation_at_the_bench_size(precision, tol):
    """24^3 cells, p = 5, viscous TGV (14.9 M DOF): three RK4 steps leave the integrals of the
    five conserved variables unchanged to rounding (relative to the integral's magnitude; the
    momenta, whose integrals vanish on the TGV, relative to the mass)."""
    from philip_b200.dg import FlowSolver, RungeKuttaODESolver
    d = prm_dict(poly_degree=5, n_cells=24, pde="navier_stokes", diss="bassi_rebay_2")
    d["flow_solver/adaptive_time_step"] = "true"
    prm = Parameters.from_dict(d)
    fs = FlowSolver(prm, precision=precision)
    dt = fs.adaptive_time_step()
    ops = _gll_weights(prm.poly_degree)
    W = np.einsum("i,j,k->kji", ops, ops, ops).reshape(-1)          # node weight, x fastest
    h = (prm.grid_bounds[1] - prm.grid_bounds[0]) / prm.n_cells
    N1 = prm.poly_degree + 1

    def integrals(U):
        u = U.reshape(-1, 5, N1 ** 3)
        return np.einsum("csn,n->s", u, W) * h ** 3

    q0 = integrals(fs.dg.solution)
    RungeKuttaODESolver(fs.dg).step_in_time(dt, nsteps=3)
    q1 = integrals(fs.dg.solution)
    assert fs.dg.status() == 0
    scale = np.array([abs(q0[0]), abs(q0[0]), abs(q0[0]), abs(q0[0]), abs(q0[4])])
    change = np.abs(q1 - q0) / scale
    print(f"conserved-integral changes over 3 steps: {change}")
    assert np.all(change <= tol)


def _gll_weights(p):
    """GLL weights on [0, 1] for p + 1 points: the nodes are +-1 and the roots of P_p', the weights
    2 / (p (p + 1) P_p(x)^2) on [-1, 1]."""
    n = p + 1
    from numpy.polynomial import legendre as Lg
    c = np.zeros(n); c[-1] = 1.0                       # P_p
    interior = Lg.legroots(Lg.legder(c)) if n > 2 else np.array([])
    x = np.concatenate(([-1.0], interior, [1.0]))
    Pp = Lg.legval(x, c)
    w = 2.0 / (p * (p + 1) * Pp ** 2)
    return 0.5 * w


@pytest.mark.gpu
def test_device_time_loop_refuses_relaxed_steps():
    from philip_b200.dg import DGStrong
    d = prm_dict(poly_degree=2, n_cells=2)
    d["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true"
    dg = DGStrong(Parameters.from_dict(d))
    rows = np.zeros((2, 4))
    rc = dg.L.ph_run(dg.handle, 1e-3, 4, 2, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == _lib.PH_ERR_UNSUPPORTED and b"relaxation" in dg.L.ph_last_error()


@pytest.mark.gpu
def test_roe_entropy_fix_with_vanishing_wave_speed_differences():
    """A z-extruded isentropic vortex in the precision form: at the z faces the normal
    velocities and their differences are below FP32's normal range, where the Harten fix's
    eps^-1 (an approximate reciprocal that flushes to zero) is infinite; the fix then keeps
    eps / 2 (the quotient it drops is smaller than eps), so the step stays finite and close to
    the FP64 step (before this guard two nodes per corner cell turned NaN after one step)."""
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.serve import SolveRequest
    req = SolveRequest("isentropic_vortex", n_cells=3, poly_degree=4, mach=0.4, final_time=0.02)
    U0, dt, nsteps = req.prepare()
    out = {}
    for prec in (_lib.PH_FP64, _lib.PH_FP32_RESIDUAL):
        dg = DGStrong(req.parameters(), precision=prec)
        dg.solution = U0
        RungeKuttaODESolver(dg).step_in_time(dt, nsteps=nsteps)
        out[prec] = dg.solution
        assert dg.status() == 0
    assert np.all(np.isfinite(out[_lib.PH_FP32_RESIDUAL]))
    assert rel_max_err(out[_lib.PH_FP32_RESIDUAL], out[_lib.PH_FP64]) <= 1e-5
