"""ph_residual_noalloc: R(U) on caller-owned device buffers with no device allocation.

Callers that cannot call cudaMalloc (inside CUDA-graph capture, in loops that must not
synchronise the device, or under a framework that owns all device memory) use this entry
point; its scratch is a fixed file-scope device array. It must give the same residual as
ph_residual (tolerance 1e-12 relative max-norm, as the other parity tests), on two calls
in a row (the shared scratch keeps the previous call's contents), and reject meshes above
its fixed limits with an error. Collected last on purpose (file name).
"""
import ctypes

import numpy as np
import pytest

from philip_b200 import _lib
from philip_b200.dg import DGStrong
from philip_b200.prm import Parameters

from helpers import prm_dict, rel_max_err

CASES = [
    ("ns_CH_roe_br2_p3", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2")),
    ("ns_IR_sipg_p2_lex", dict(poly_degree=2, n_cells=3, pde="navier_stokes", two_point="IR", conv="two_point_flux")),
    ("euler_CH_roe_p5", dict(poly_degree=5, n_cells=2)),
    ("ns_conservative_cHU_p4", dict(poly_degree=4, n_cells=3, pde="navier_stokes", split=False, conv="roe",
                                    fr="cHU")),
]


def _state(dg, seed):
    from philip_b200.dg import conservative_state, tgv_primitive
    X = dg.node_coordinates()
    U = conservative_state(dg, tgv_primitive(X[..., 0], X[..., 1], X[..., 2], 1.4, 0.1))
    rng = np.random.default_rng(seed)
    return U * (1.0 + 0.02 * rng.standard_normal(U.shape))


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_noalloc_residual_matches_context_residual(name, kw):
    import torch
    prm = Parameters.from_dict(prm_dict(**kw))
    dg = DGStrong(prm)
    L = dg.L
    for call in range(2):
        U = _state(dg, seed=call + len(name))
        R_ref = dg.residual_of(U)
        dU = torch.from_numpy(U).cuda()
        dR = torch.full_like(dU, float("nan"))
        rc = L.ph_residual_noalloc(ctypes.byref(dg.mesh), ctypes.byref(dg.params), ctypes.c_void_p(dU.data_ptr()),
                                   ctypes.c_void_p(dR.data_ptr()), None)
        _lib.check(rc)
        torch.cuda.synchronize()
        err = rel_max_err(dR.cpu().numpy(), R_ref)
        print(f"{name} call {call}: no-alloc vs context residual rel err {err:.3e}")
        assert err <= 1e-12


@pytest.mark.gpu
def test_noalloc_rejects_meshes_above_its_limits():
    import torch
    L = _lib.load()
    # 14^3 cells at p = 5: 2744 x (4 x 216 + 24 x 36) doubles of viscous terms > 4 Mi
    prm = Parameters.from_dict(prm_dict(poly_degree=5, n_cells=14, pde="navier_stokes", diss="bassi_rebay_2"))
    p = prm.to_ph_params()
    mesh = _lib.PhMeshDesc(14, 0, 0.0, 6.28318530717958623200)
    dU = torch.zeros(5 * 216 * 14 ** 3, dtype=torch.float64, device="cuda")
    dR = torch.zeros_like(dU)
    rc = L.ph_residual_noalloc(ctypes.byref(mesh), ctypes.byref(p), ctypes.c_void_p(dU.data_ptr()),
                               ctypes.c_void_p(dR.data_ptr()), None)
    assert rc == 1
    assert b"viscous-term scratch" in L.ph_last_error()
    mesh.n_cells_per_direction = 40
    rc = L.ph_residual_noalloc(ctypes.byref(mesh), ctypes.byref(p), ctypes.c_void_p(dU.data_ptr()),
                               ctypes.c_void_p(dR.data_ptr()), None)
    assert rc == 1
    assert b"cells exceed" in L.ph_last_error()
