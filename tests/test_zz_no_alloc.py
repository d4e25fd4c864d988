"""ph_residual_noalloc: R(U) on caller-owned device buffers with no device allocation.

Some callers of this library cannot allocate device memory: a solver loop that must never
synchronise the device (cudaMalloc and cudaFree may synchronise), or a host framework that
reserves all device memory for its own pool up front and forbids allocations behind its
back. They call this entry point; its scratch is fixed file-scope device arrays shared by
every call.

Checked here, through the C-ABI: the same residual as ph_residual on a context (tolerance
1e-12 relative max-norm in FP64, the other parity tests' bound; 1e-5 in the precision form,
the precision tests' bound) on two calls in a row (the shared scratch keeps the previous
call's contents), on the default stream and on a side stream; free device memory unchanged
by a warm call; the non-physical flag of the last call readable through
ph_residual_noalloc_status and cleared by the next call; meshes above the fixed limits
rejected with an error. Collected last on purpose (file name).
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
    ("ns_CH_kSD_aux_p3", dict(poly_degree=3, n_cells=3, pde="navier_stokes", fr_aux="kSD")),
]


def _state(dg, seed):
    from philip_b200.dg import conservative_state, tgv_primitive
    X = dg.node_coordinates()
    U = conservative_state(dg, tgv_primitive(X[..., 0], X[..., 1], X[..., 2], 1.4, 0.1))
    rng = np.random.default_rng(seed)
    return U * (1.0 + 0.02 * rng.standard_normal(U.shape))


def _noalloc(dg, dU, dR, stream=None):
    rc = dg.L.ph_residual_noalloc(ctypes.byref(dg.mesh), ctypes.byref(dg.params), ctypes.c_void_p(dU.data_ptr()),
                                  ctypes.c_void_p(dR.data_ptr()), stream)
    _lib.check(rc)


def _status(L, stream=None):
    flags = ctypes.c_uint32(0xFFFFFFFF)
    _lib.check(L.ph_residual_noalloc_status(stream, ctypes.byref(flags)))
    return flags.value


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_noalloc_residual_matches_context_residual(name, kw):
    import torch
    prm = Parameters.from_dict(prm_dict(**kw))
    dg = DGStrong(prm)
    for call in range(2):
        U = _state(dg, seed=call + len(name))
        R_ref = dg.residual_of(U)
        dU = torch.from_numpy(U).cuda()
        dR = torch.full_like(dU, float("nan"))
        _noalloc(dg, dU, dR)
        torch.cuda.synchronize()
        err = rel_max_err(dR.cpu().numpy(), R_ref)
        print(f"{name} call {call}: no-alloc vs context residual rel err {err:.3e}")
        assert err <= 1e-12
        assert _status(dg.L) == 0


@pytest.mark.gpu
def test_noalloc_precision_form_matches_context_residual():
    import torch
    prm = Parameters.from_dict(prm_dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"))
    dg = DGStrong(prm, precision=_lib.PH_FP32_RESIDUAL)
    for call in range(2):
        U = _state(dg, seed=11 + call)
        R_ref = dg.residual_of(U)
        dU = torch.from_numpy(U).cuda()
        dR = torch.full_like(dU, float("nan"))
        _noalloc(dg, dU, dR)
        torch.cuda.synchronize()
        err = rel_max_err(dR.cpu().numpy(), R_ref)
        print(f"precision form call {call}: no-alloc vs context residual rel err {err:.3e}")
        assert err <= 1e-5


@pytest.mark.gpu
def test_noalloc_on_a_side_stream_allocates_nothing():
    import torch
    prm = Parameters.from_dict(prm_dict(poly_degree=4, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"))
    dg = DGStrong(prm)
    U = _state(dg, seed=5)
    R_ref = dg.residual_of(U)
    side = torch.cuda.Stream()
    dU = torch.from_numpy(U).cuda()
    dR = torch.full_like(dU, float("nan"))
    torch.cuda.synchronize()
    handle = ctypes.c_void_p(side.cuda_stream)
    _noalloc(dg, dU, dR, handle)        # warm call: the device's first call resolves the arrays' addresses
    side.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    dR.fill_(float("nan"))
    torch.cuda.synchronize()
    _noalloc(dg, dU, dR, handle)
    side.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    err = rel_max_err(dR.cpu().numpy(), R_ref)
    print(f"side stream: rel err {err:.3e}, free memory {free_before} -> {free_after}")
    assert err <= 1e-12
    assert free_after == free_before


@pytest.mark.gpu
def test_noalloc_reports_a_non_physical_state():
    import torch
    prm = Parameters.from_dict(prm_dict(poly_degree=3, n_cells=2))
    dg = DGStrong(prm)
    U = _state(dg, seed=3)
    bad = U.copy()
    bad[0] = -abs(bad[0])               # density of node 0 of cell 0
    dU = torch.from_numpy(bad).cuda()
    dR = torch.zeros_like(dU)
    _noalloc(dg, dU, dR)
    assert _status(dg.L) & 1
    dU.copy_(torch.from_numpy(U))
    _noalloc(dg, dU, dR)                # the next call clears the flag
    assert _status(dg.L) == 0


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
