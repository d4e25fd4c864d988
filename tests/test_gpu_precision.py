"""Precision form: FP32 residual arithmetic, FP64 state with a compensated final sum,
FP64 positivity checks and metric scaling.

Tolerances (stated here, measured against the FP64 oracle / FP64 GPU path):
  residual, relative max-norm vs the FP64 oracle ............ 1e-5
  TGV kinetic energy history over 200 steps, relative ....... 2e-7
  vorticity-based dissipation rate history, relative ........ 1e-6
(the history bounds hold with the flow's mean pressure taken out of the FP32 momentum
fluxes, ph_params.pressure_shift, which the flow-case parameters set; without it they were
3e-6 and 1e-6)
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from philip_b200 import _lib
from philip_b200.dg import DGStrong, FlowSolver
from philip_b200.prm import Parameters

from helpers import prm_dict, perturbed_tgv, rel_max_err


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"),
                                dict(poly_degree=5, n_cells=2), dict(poly_degree=2, n_cells=3, two_point="IR",
                                                                     conv="two_point_flux")])
def test_fp32_residual_close_to_fp64_oracle(kw):
    prm = Parameters.from_dict(prm_dict(**kw))
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    dg = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL)
    U = perturbed_tgv(orc, seed=4)
    err = rel_max_err(dg.residual_of(U), orc.residual(U))
    print(f"fp32 residual rel err {err:.3e}")
    assert err <= 1e-5


@pytest.mark.gpu
def test_fp32_tgv_energy_history():
    d = prm_dict(poly_degree=3, n_cells=8, pde="navier_stokes", diss="bassi_rebay_2", cfl=0.009,
                 final_time=0.354)
    hist = {}
    for prec in (_lib.PH_FP64, _lib.PH_FP32_RESIDUAL):
        fs = FlowSolver(Parameters.from_dict(d), precision=prec)
        fs.run()
        assert fs.dg.status() == 0
        hist[prec] = np.array(fs.unsteady_data)
    h64, h32 = hist[_lib.PH_FP64], hist[_lib.PH_FP32_RESIDUAL]
    assert h64.shape == h32.shape and len(h64) > 150
    ke_err = np.max(np.abs(h32[:, 1] - h64[:, 1])) / np.max(np.abs(h64[:, 1]))
    eps_err = np.max(np.abs(h32[:, 3] - h64[:, 3])) / np.max(np.abs(h64[:, 3]))
    print(f"fp32 KE rel err {ke_err:.3e}, dissipation-rate rel err {eps_err:.3e}")
    # with the mean pressure taken out of the FP32 momentum fluxes (ph_params.pressure_shift)
    assert ke_err <= 2e-7
    assert eps_err <= 1e-6


@pytest.mark.gpu
def test_kinetic_energy_rate_from_the_time_derivative():
    """ph_kinetic_energy_rate: dKE/dt from the state and M^-1 R(u) equals the derivative of the
    kinetic energy along that direction, by central differences at two step sizes and Richardson
    extrapolation (tolerance 1e-8: the differences' rounding over the step), in FP64; the
    precision form's rate at the same state is stated (its FP32 residual carries about 1e-6 of
    the momentum and energy fluxes, and dKE/dt is a small difference of such terms)."""
    prm = Parameters.from_dict(prm_dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"))
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    U = perturbed_tgv(orc, seed=9, amp=0.01)
    dg = DGStrong(prm)
    dg.solution = U
    rate = dg.kinetic_energy_rate()
    K = orc.inverse_mass(orc.residual(U))

    def central(eps):
        ke = []
        for sgn in (1.0, -1.0):
            dg.solution = U + sgn * eps * K
            ke.append(dg.integrals()[0])
        return (ke[0] - ke[1]) / (2.0 * eps)

    eps = 1e-3 / np.max(np.abs(K))
    d1, d2 = central(eps), central(eps / 2)
    fd = (4.0 * d2 - d1) / 3.0
    dg32 = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL)
    dg32.solution = U
    rate32 = dg32.kinetic_energy_rate()
    print(f"dKE/dt {rate:.12e}, central differences {d1:.12e} {d2:.12e} -> {fd:.12e}, "
          f"precision form {rate32:.12e} (rel {abs(rate32 - rate) / abs(rate):.2e})")
    assert abs(rate - fd) <= 1e-8 * abs(rate)
    assert abs(rate32 - rate) <= 1e-3 * abs(rate)
