"""Batch of solves (ph_batch_*): a solve's result is bitwise the same alone in a batch and
inside a running mix, whatever else shares the batch and whenever it joins; it matches the
single-solve context (ph_rk_step) bitwise in FP64 and within 1e-6 relative max-norm in the
precision form (the two kernels are the same source, but the compiler may contract FP32
products into FMAs differently in the two kernel bodies); admission respects the HBM budget;
the tile-shape autotuner runs; the vortex solve converges to the exact translated vortex."""
import numpy as np
import pytest

from philip_b200 import _lib
from philip_b200.dg import DGStrong, RungeKuttaODESolver
from philip_b200.serve import Batch, SnapshotServer, SolveRequest, autotune, solve_bytes

pytestmark = pytest.mark.gpu

TWO_PI = 6.28318530717958623200

MIX = [
    SolveRequest("isentropic_vortex", n_cells=4, poly_degree=2, mach=0.3, beta=2.0, direction=(0.6, 0.8, 0.0),
                 final_time=0.05),
    SolveRequest("taylor_green_vortex", n_cells=3, poly_degree=3, left=0.0, right=TWO_PI, warp=0.1, mach=0.2,
                 final_time=0.02),
    SolveRequest("isentropic_vortex", n_cells=2, poly_degree=4, warp=0.1, mach=0.4, beta=3.0,
                 direction=(0.0, 0.6, 0.8), final_time=0.05),
    SolveRequest("taylor_green_vortex", n_cells=2, poly_degree=5, left=0.0, right=TWO_PI, mach=0.1,
                 final_time=0.01, two_point="IR", conv="two_point_flux"),
]


FP32_RTOL = 1e-6


def _same_as_single(Ub, Ua, precision):
    if precision == _lib.PH_FP64:
        return np.array_equal(Ub, Ua)
    return np.max(np.abs(Ub - Ua)) <= FP32_RTOL * np.max(np.abs(Ua))


def _alone_in_batch(req, precision):
    b = Batch(1 << 28, precision)
    U0 = req.initial_state()
    dt, nsteps = req.time_step(U0)
    s = b.admit(req.mesh(), req.parameters().to_ph_params(precision), U0, dt, nsteps)
    b.step(nsteps)
    U = b.state(s, req.ndofs)
    b.close()
    return U


def _alone(req, precision):
    """The same solve through the single-solve context (ph_rk_step)."""
    dg = DGStrong(req.parameters(), precision=precision, warp=req.warp)
    U0 = req.initial_state()
    dt, nsteps = req.time_step(U0)
    dg.solution = U0
    RungeKuttaODESolver(dg).step_in_time(dt, nsteps=nsteps)
    return dg.solution, dg.status()


@pytest.mark.parametrize("precision", [_lib.PH_FP64, _lib.PH_FP32_RESIDUAL])
def test_batch_matches_single_solves_bitwise(precision):
    b = Batch(1 << 30, precision)
    slots = []
    for req in MIX:
        U0 = req.initial_state()
        dt, nsteps = req.time_step(U0)
        slots.append(b.admit(req.mesh(), req.parameters().to_ph_params(precision), U0, dt, nsteps))
    b.step(10 ** 6)
    assert b.active == 0
    for req, s in zip(MIX, slots):
        Ub = b.state(s, req.ndofs)
        Ua, st = _alone(req, precision)
        print(f"{req.flow_case} p={req.poly_degree} warp={req.warp}: max |batch - alone| {np.max(np.abs(Ub - Ua)):.3e}")
        assert st == 0 and b.status(s) == 0
        assert _same_as_single(Ub, Ua, precision)
    assert b.launches > 0
    b.close()


def test_same_result_alone_and_joining_a_running_mix():
    prec = _lib.PH_FP32_RESIDUAL
    req = MIX[0]
    U0 = req.initial_state()
    dt, nsteps = req.time_step(U0)
    prm = req.parameters().to_ph_params(prec)
    U_alone = _alone_in_batch(req, prec)

    mix = Batch(1 << 30, prec)
    others = []
    for r in MIX[1:]:
        V0 = r.initial_state()
        d, n = r.time_step(V0)
        others.append((r, mix.admit(r.mesh(), r.parameters().to_ph_params(prec), V0, d, n)))
    mix.step(2)                         # the mix is running when the solve arrives
    s = mix.admit(req.mesh(), prm, U0, dt, nsteps)
    mix.step(3)
    late = SolveRequest("isentropic_vortex", n_cells=3, poly_degree=3, mach=0.2, beta=1.5, final_time=0.03)
    V0 = late.initial_state()
    d, n = late.time_step(V0)
    mix.admit(late.mesh(), late.parameters().to_ph_params(prec), V0, d, n)   # and another joins mid-way
    mix.step(10 ** 6)
    assert np.array_equal(mix.state(s, req.ndofs), U_alone)
    mix.close()


def test_admission_respects_the_budget():
    prec = _lib.PH_FP32_RESIDUAL
    req = SolveRequest("isentropic_vortex", n_cells=4, poly_degree=3, final_time=0.01)
    U0 = req.initial_state()
    dt, nsteps = req.time_step(U0)
    prm = req.parameters().to_ph_params(prec)
    need = solve_bytes(req.mesh(), prm)
    b = Batch(2 * need + need // 2, prec)
    s0 = b.admit(req.mesh(), prm, U0, dt, nsteps)
    s1 = b.admit(req.mesh(), prm, U0, dt, nsteps)
    assert s0 is not None and s1 is not None
    assert b.admit(req.mesh(), prm, U0, dt, nsteps) is None
    b.step(nsteps)
    U = b.state(s0, req.ndofs)
    b.release(s0)
    s2 = b.admit(req.mesh(), prm, U0, dt, nsteps)
    assert s2 is not None
    b.step(nsteps)
    assert np.array_equal(b.state(s2, req.ndofs), U)
    b.close()


def test_served_mix_and_vortex_error():
    prec = _lib.PH_FP32_RESIDUAL
    rng = np.random.default_rng(20261203)
    reqs = []
    for i in range(12):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        reqs.append((0.002 * i, SolveRequest("isentropic_vortex", n_cells=int(rng.choice([3, 4])),
                                             poly_degree=int(rng.integers(2, 5)), mach=float(rng.uniform(0.1, 0.5)),
                                             beta=float(rng.uniform(1.0, 5.0)), direction=tuple(d),
                                             final_time=0.1, warp=0.1 if i % 2 else 0.0)))
    srv = SnapshotServer(Batch(1 << 30, prec), chunk=8, keep_states=True)
    stats = srv.run(reqs)
    assert len(stats.completed) == 12 and stats.max_in_flight > 1
    for c in stats.completed:
        assert c.status == 0
        exact = c.request.exact_state()
        err = np.max(np.abs(c.state - exact)) / np.max(np.abs(exact))
        print(f"p={c.request.poly_degree} n={c.request.n_cells} beta={c.request.beta:.2f}: rel max error {err:.3e}, "
              f"latency {c.latency * 1e3:.1f} ms")
        assert err < 0.1
        assert np.array_equal(c.state, _alone_in_batch(c.request, prec))
        assert _same_as_single(c.state, _alone(c.request, prec)[0], prec)


@pytest.mark.parametrize("p", [2, 3])
def test_batched_vortex_converges_at_the_design_order(p):
    """h-refinement of the translated isentropic vortex in one FP64 batch (all meshes together):
    the RMS nodal error against the exact solution falls by at least 2^(p + 1/2) per halving of
    the cell size (DG of degree p on a smooth solution: order p + 1, here measured between the
    two finest meshes), so a wrong-but-stable solve fails."""
    prec = _lib.PH_FP64
    ns = [6, 12, 24]
    reqs = [SolveRequest("isentropic_vortex", n_cells=n, poly_degree=p, mach=0.3, beta=3.0,
                         direction=(0.6, 0.8, 0.0), final_time=0.5, cfl=0.05) for n in ns]
    b = Batch(4 << 30, prec)
    slots = []
    for r in reqs:
        U0 = r.initial_state()
        dt, nsteps = r.time_step(U0)
        slots.append(b.admit(r.mesh(), r.parameters().to_ph_params(prec), U0, dt, nsteps))
    b.step(10 ** 6)
    errs = []
    for r, s in zip(reqs, slots):
        U = b.state(s, r.ndofs)
        ex = r.exact_state()
        errs.append(float(np.sqrt(np.mean((U - ex) ** 2)) / np.sqrt(np.mean(ex ** 2))))
    b.close()
    orders = [np.log2(errs[i] / errs[i + 1]) for i in range(len(ns) - 1)]
    print(f"p={p}: RMS errors {['%.3e' % e for e in errs]}, observed orders {['%.2f' % o for o in orders]}")
    assert orders[-1] >= p + 0.5
    assert all(e2 < e1 for e1, e2 in zip(errs, errs[1:]))


def test_autotuner_picks_a_variant():
    best, ms = autotune(3, _lib.PH_FP32_RESIDUAL, False)
    print("p=3 variants ms:", ms, "best", best)
    assert len(ms) >= 1 and 0 <= best < len(ms) and all(t > 0 for t in ms)
