"""All nine integrated quantities of PeriodicTurbulence::compute_and_update_integrated_quantities
(periodic_turbulence.cpp:439-672, IntegratedQuantitiesEnum order of periodic_turbulence.h:176-186).

The reference's golden values pin the kinetic energy and the vorticity-based dissipation
rate only (taylor_green_vortex_energy_check.cpp). The oracle's other seven are pinned by the
analytic values of the Taylor-Green initial field on [0, 2 pi]^3, to which the interpolated
state converges with the mesh: rho = 1 makes the incompressible and compressible kinetic
energy and enstrophy equal (1/8 and 3/8); the field is solenoidal, so the pressure dilatation
vanishes and the deviatoric strain rate equals the strain rate, whose squared magnitude
averages to half the mean squared vorticity (3/8, times a constant viscosity of 1);
the vorticity's gradient gives a palinstrophy of 9/8; the angular momentum 0.5 |x|^2 |omega|
is checked against a midpoint sum of the analytic field. The CUDA path is then held to the
oracle within 1e-12 relative (affine and curvilinear cells, Sutherland and constant viscosity).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.prm import Parameters

from helpers import TWO_PI, perturbed_tgv, prm_dict

NAMES = _lib.INTEGRATED_QUANTITIES


def _setup(const_visc=True, warp=0.0, **kw):
    d = prm_dict(**kw)
    if const_visc:
        d["navier_stokes/use_constant_viscosity"] = "true"
    prm = Parameters.from_dict(d)
    left, right = prm.grid_bounds
    return prm, Oracle(prm.oracle_cfg(), prm.n_cells, left, right, warp=warp)


def _midpoint_angular_momentum(m=96):
    x = (np.arange(m) + 0.5) * TWO_PI / m
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    ox = -np.cos(X) * np.sin(Y) * np.sin(Z)
    oy = -np.sin(X) * np.cos(Y) * np.sin(Z)
    oz = 2.0 * np.sin(X) * np.sin(Y) * np.cos(Z)
    return float(np.mean(0.5 * (X ** 2 + Y ** 2 + Z ** 2) * np.sqrt(ox ** 2 + oy ** 2 + oz ** 2)))


def test_oracle_tgv_initial_field_analytic_values():
    _, orc = _setup(poly_degree=5, n_cells=4, pde="navier_stokes")
    q = orc.integrated_quantities(orc.initial_condition("tgv"))
    v = dict(zip(NAMES, q[:9]))
    for k, exact in [("kinetic_energy", 0.125), ("enstrophy", 0.375), ("incompressible_kinetic_energy", 0.125),
                     ("incompressible_enstrophy", 0.375),
                     ("viscosity_times_strain_rate_tensor_magnitude_sqr", 0.375),
                     ("viscosity_times_deviatoric_strain_rate_tensor_magnitude_sqr", 0.375)]:
        assert abs(v[k] - exact) <= 1e-7 * exact, (k, v[k])
    assert abs(v["pressure_dilatation"]) <= 1e-14
    assert abs(v["incompressible_palinstrophy"] - 1.125) <= 2e-3 * 1.125
    am = _midpoint_angular_momentum()
    assert abs(v["angular_momentum"] - am) <= 2e-3 * am
    # the last entry is the maximum wave speed, the same as the four-value subset's
    assert q[9] == orc.integrals(orc.initial_condition("tgv"))[3]


def test_oracle_palinstrophy_converges_with_the_mesh():
    errs = []
    for n in (2, 4):
        _, orc = _setup(poly_degree=4, n_cells=n, pde="navier_stokes")
        errs.append(abs(orc.integrated_quantities(orc.initial_condition("tgv"))[7] - 1.125))
    assert errs[1] < errs[0] / 8


def test_oracle_sutherland_viscosity_near_one_at_freestream_temperature():
    # T = gamma M^2 p / rho = 1 + O(M^2) on the TGV initial field: mu(T) close to 1
    _, orc = _setup(const_visc=False, poly_degree=4, n_cells=3, pde="navier_stokes", mach=0.1)
    q = orc.integrated_quantities(orc.initial_condition("tgv"))
    assert abs(q[4] / q[6] - 1.0) < 0.02


def test_oracle_vanishing_warp_matches_affine_path():
    kw = dict(poly_degree=3, n_cells=3, pde="navier_stokes")
    _, affine = _setup(**kw)
    _, curved = _setup(warp=1e-300, **kw)
    U = perturbed_tgv(affine, seed=4)
    qa, qc = affine.integrated_quantities(U), curved.integrated_quantities(U)
    assert np.allclose(qc, qa, rtol=1e-12, atol=1e-14 * np.max(np.abs(qa)))


def test_unsteady_table_columns_follow_the_reference():
    import inspect
    from philip_b200.dg import FlowSolver
    src = inspect.getsource(FlowSolver.unsteady_data_row)
    for col in ("eps_vorticity", "eps_pressure", "eps_strain", "eps_dev_strain", "incompressible_kinetic_energy",
                "incompressible_enstrophy", "incompressible_palinstrophy", "angular_momentum"):
        assert f'"{col}"' in src


# ------------------------------------------------------------------------------- GPU parity

CASES = [
    ("euler_p2", dict(poly_degree=2, n_cells=4), True, 0.0),
    ("ns_const_visc_p3", dict(poly_degree=3, n_cells=4, pde="navier_stokes"), True, 0.0),
    ("ns_sutherland_p5", dict(poly_degree=5, n_cells=2, pde="navier_stokes"), False, 0.0),
    ("ns_sutherland_p6", dict(poly_degree=6, n_cells=2, pde="navier_stokes"), False, 0.0),
    # the integrands are the Navier-Stokes physics' whatever the PDE, so the viscous quantities
    # are computed on the Euler context too
    ("curved_p3", dict(poly_degree=3, n_cells=3), False, 0.1),
    ("curved_ns_br2_p4", dict(poly_degree=4, n_cells=2, pde="navier_stokes", diss="bassi_rebay_2"), False, 0.1),
    ("curved_p6", dict(poly_degree=6, n_cells=2), True, 0.1),
]


def _close(a, b, scale):
    return abs(a - b) <= 1e-12 * max(abs(b), scale)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,const_visc,warp", CASES, ids=[c[0] for c in CASES])
def test_integrated_quantities_parity(name, kw, const_visc, warp):
    from philip_b200.dg import DGStrong
    prm, orc = _setup(const_visc=const_visc, warp=warp, **kw)
    dg = DGStrong(prm, warp=warp)
    U = perturbed_tgv(orc, seed=len(name), amp=0.01)
    dg.solution = U
    q_gpu = dg.integrated_quantities()
    q_orc = orc.integrated_quantities(U)
    scale = np.max(np.abs(q_orc[:9]))
    for i, k in enumerate(NAMES):
        print(f"{name} {k}: gpu {q_gpu[i]:.15e} oracle {q_orc[i]:.15e}")
        assert _close(q_gpu[i], q_orc[i], 1e-3 * scale), k
    # the four-value subset agrees with the full set
    q4 = dg.integrals()
    assert _close(q4[0], q_gpu[0], 0.0) and _close(q4[1], q_gpu[1], 0.0)
    assert _close(q4[3], q_orc[9], 0.0)


@pytest.mark.gpu
def test_flow_solver_unsteady_row():
    from philip_b200.dg import FlowSolver
    d = prm_dict(poly_degree=3, n_cells=4, pde="navier_stokes", final_time=0.05)
    d["flow_solver/dipole_wall_collision/do_compute_angular_momentum"] = "true"
    prm = Parameters.from_dict(d)
    fs = FlowSolver(prm)
    fs.run()
    row = fs.unsteady_data_row()
    left, right = prm.grid_bounds
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, left, right)
    q = orc.integrated_quantities(fs.dg.solution)
    re = float(prm.get("navier_stokes/reynolds_number_inf"))
    assert _close(row["eps_pressure"], -q[2], 1e-3 * q[0])
    assert _close(row["eps_strain"], 2.0 * q[4] / re, 0.0)
    assert _close(row["eps_dev_strain"], 2.0 * q[3] / re, 0.0)
    assert _close(row["incompressible_palinstrophy"], q[7], 0.0)
    assert _close(row["angular_momentum"], q[8], 0.0)
    assert abs(row["time"] - 0.05) < 1e-12
