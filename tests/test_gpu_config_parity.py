"""Parity of the CUDA path with the CPU oracle at the benchmark configurations' real sizes.

The smaller parity cases (1-4 cells per direction) cover every flux and option; these cover
the index maps, cell orders and kernel variants that only run at full size, with the
correctness bar of the hot path:
  residual, relative max-norm ........................................ 1e-12
      (max over DOFs of |R_gpu - R_oracle| over max |R_oracle|, globally and per conserved
      variable)
  kinetic-energy and enstrophy histories, relative, every step ....... 1e-10
      (the reference's energy-check bar, taylor_green_vortex_energy_check.cpp:37-44; the
      quantities of periodic_turbulence.cpp:439-672)
  precision form residual against the FP64 oracle .................... 1e-5 (stated, printed)

Configurations (viscous cases: Re 1600, Pr 0.71, Sutherland viscosity, BR2; all: Mach 0.1,
Chandrashekar split form with Roe dissipation, cDG, RK4):
  8^3 cells p = 3 inviscid to t = 1; 24^3 cells p = 5; 32^3 cells p = 3.
The reference's constant TGV step at CFL 0.1 is acoustically unstable at Mach 0.1 (the state
turns non-physical within ten RK4 steps, in the oracle too), so the histories use the
adaptive step CFL 0.1 x spacing / max wave speed of the initial state, held constant.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.dg import DGStrong, FlowSolver, RungeKuttaODESolver
from philip_b200.prm import Parameters

from helpers import prm_dict, rel_max_err

Oracle.set_threads(os.cpu_count() or 8)


def _per_variable_err(a, b, N1):
    a = a.reshape(-1, 5, N1 ** 3)
    b = b.reshape(-1, 5, N1 ** 3)
    return max(float(np.max(np.abs(a[:, s] - b[:, s])) / np.max(np.abs(b[:, s]))) for s in range(5))


def _setup(**kw):
    d = prm_dict(**kw)
    d["flow_solver/adaptive_time_step"] = "true"
    prm = Parameters.from_dict(d)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    return prm, orc


def _histories(prm, orc, nsteps=None, final_time=None, precision=_lib.PH_FP64):
    """Steps the GPU (FlowSolver's discretisation, through the C-ABI) and the oracle with the
    same constant step; returns the per-step relative errors of KE and enstrophy and the
    final states."""
    fs = FlowSolver(prm, precision=precision)
    U = orc.initial_condition("tgv")
    assert rel_max_err(fs.dg.solution, U) <= 1e-14
    fs.dg.solution = U          # the same initial state, bit for bit
    dt = fs.adaptive_time_step()
    if nsteps is None:
        nsteps = int(np.ceil(final_time / dt - 1e-12))
    ode = RungeKuttaODESolver(fs.dg)
    errs = []
    t = 0.0
    for n in range(nsteps):
        step = dt if final_time is None else min(dt, final_time - t)
        ode.step_in_time(step)
        orc.rk_step(U, step)
        t += step
        g = fs.dg.integrals()
        o = orc.integrals(U)
        errs.append((abs(g[0] - o[0]) / abs(o[0]), abs(g[1] - o[1]) / abs(o[1])))
    assert fs.dg.status() == 0 and orc.status() == 0
    return np.array(errs), fs.dg.solution, U, t


@pytest.mark.gpu
def test_c1_inviscid_8_p3_histories_to_t1():
    prm, orc = _setup(poly_degree=3, n_cells=8)
    errs, Ug, Uo, t = _histories(prm, orc, final_time=1.0)
    print(f"8^3 p3 inviscid: {len(errs)} RK4 steps to t = {t:.6f}; max rel err KE {errs[:, 0].max():.3e}, "
          f"enstrophy {errs[:, 1].max():.3e}; final state {rel_max_err(Ug, Uo):.3e}")
    assert abs(t - 1.0) <= 1e-12
    assert errs[:, 0].max() <= 1e-10
    assert errs[:, 1].max() <= 1e-10


@pytest.mark.gpu
def test_c2_viscous_24_p5_residual_step_and_histories():
    prm, orc = _setup(poly_degree=5, n_cells=24, pde="navier_stokes", diss="bassi_rebay_2")
    dg = DGStrong(prm)
    U = orc.initial_condition("tgv")
    rng = np.random.default_rng(24)
    Up = U * (1.0 + 0.01 * rng.standard_normal(U.shape))
    Rg, Ro = dg.residual_of(Up), orc.residual(Up)
    e_glob, e_var = rel_max_err(Rg, Ro), _per_variable_err(Rg, Ro, 6)
    print(f"24^3 p5 residual: rel err {e_glob:.3e} (per variable {e_var:.3e})")
    assert e_glob <= 1e-12 and e_var <= 1e-12
    del dg
    errs, Ug, Uo, _ = _histories(prm, orc, nsteps=20)
    e1 = rel_max_err(Ug, Uo)
    print(f"24^3 p5: 20 RK4 steps, KE {errs[:, 0].max():.3e}, enstrophy {errs[:, 1].max():.3e}; state {e1:.3e}")
    assert errs[:, 0].max() <= 1e-10
    assert errs[:, 1].max() <= 1e-10
    assert e1 <= 1e-11


@pytest.mark.gpu
def test_c3_viscous_32_p3_residual_fp64_and_precision_form():
    prm, orc = _setup(poly_degree=3, n_cells=32, pde="navier_stokes", diss="bassi_rebay_2")
    U = orc.initial_condition("tgv")
    rng = np.random.default_rng(32)
    Up = U * (1.0 + 0.01 * rng.standard_normal(U.shape))
    Ro = orc.residual(Up)
    dg = DGStrong(prm)
    Rg = dg.residual_of(Up)
    e_glob, e_var = rel_max_err(Rg, Ro), _per_variable_err(Rg, Ro, 4)
    print(f"32^3 p3 residual FP64: rel err {e_glob:.3e} (per variable {e_var:.3e})")
    assert e_glob <= 1e-12 and e_var <= 1e-12
    del dg
    dg32 = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL)
    e32 = rel_max_err(dg32.residual_of(Up), Ro)
    print(f"32^3 p3 residual, precision form against the FP64 oracle: rel err {e32:.3e}")
    assert e32 <= 1e-5
