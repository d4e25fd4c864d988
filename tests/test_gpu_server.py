"""Native server (ph_server_*): the continuous-batching loop of the batch of solves behind a
thread-safe submission queue. A served solve's final state is bitwise the single-solve
context's in FP64 (the batch's guarantee, kept through admission order, chunking and
retirement); submissions from several threads at once all complete; a solve larger than the
whole budget fails with the batch's message instead of waiting for ever; a Poisson stream
completes with its latencies recorded."""
import threading

import numpy as np
import pytest

from philip_b200 import _lib
from philip_b200.dg import DGStrong, RungeKuttaODESolver
from philip_b200.serve import Server, SolveRequest, poisson_arrivals, serve_native

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


def test_server_refuses_bad_arguments_without_a_gpu():
    import ctypes
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.ph_server_create(ctypes.c_size_t(1 << 20), _lib.PH_FP64, 0, 0.004, ctypes.byref(h)) == _lib.PH_ERR_INVALID
    assert L.ph_server_create(ctypes.c_size_t(0), _lib.PH_FP64, 4, 0.004, ctypes.byref(h)) == _lib.PH_ERR_INVALID
    assert L.ph_server_create(ctypes.c_size_t(1 << 20), 7, 4, 0.004, ctypes.byref(h)) == _lib.PH_ERR_INVALID
    assert L.ph_server_create(ctypes.c_size_t(1 << 20), _lib.PH_FP64, 4, -1.0, ctypes.byref(h)) == _lib.PH_ERR_INVALID


def _alone(req):
    dg = DGStrong(req.parameters(), precision=_lib.PH_FP64, warp=req.warp)
    U0, dt, nsteps = req.prepare()
    dg.solution = U0
    RungeKuttaODESolver(dg).step_in_time(dt, nsteps=nsteps)
    return dg.solution


@pytest.mark.gpu
def test_served_solves_are_the_single_solves_bitwise():
    srv = Server(1 << 30, _lib.PH_FP64, chunk=3)
    tickets = [srv.submit_request(r) for r in MIX]
    for req, t in zip(MIX, tickets):
        assert srv.wait(t, 120.0) == _lib.PH_SOLVE_DONE
        U, flags, (t_adm, t_done) = srv.result(t, req.ndofs)
        Ua = _alone(req)
        print(f"{req.flow_case} p={req.poly_degree}: max |served - alone| {np.max(np.abs(U - Ua)):.3e}, "
              f"admitted after {t_adm * 1e3:.1f} ms, done after {t_done * 1e3:.1f} ms")
        assert flags == 0 and 0.0 <= t_adm <= t_done
        assert np.array_equal(U, Ua)
    srv.close()


@pytest.mark.gpu
def test_submissions_from_several_threads():
    srv = Server(1 << 30, _lib.PH_FP32_RESIDUAL, chunk=8)
    tickets, lock = [], threading.Lock()

    def client(k):
        for j in range(4):
            req = SolveRequest("isentropic_vortex", n_cells=2 + (j % 2), poly_degree=2 + (k + j) % 3, mach=0.2 + 0.1 * k,
                               final_time=0.02)
            t = srv.submit_request(req)
            with lock:
                tickets.append((t, req))

    th = [threading.Thread(target=client, args=(k,)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert len({t for t, _ in tickets}) == 12
    for t, req in tickets:
        assert srv.wait(t, 120.0) == _lib.PH_SOLVE_DONE
        U, flags, _ = srv.result(t, req.ndofs)
        assert flags == 0 and np.all(np.isfinite(U))
    with pytest.raises(_lib.PhError, match="unknown ticket"):
        srv.poll(tickets[0][0])
    srv.close()


@pytest.mark.gpu
def test_a_solve_larger_than_the_budget_fails():
    srv = Server(8 << 20, _lib.PH_FP64)
    big = SolveRequest("taylor_green_vortex", n_cells=8, poly_degree=5, left=0.0, right=TWO_PI, final_time=0.01)
    t = srv.submit_request(big)
    assert srv.wait(t, 60.0) == _lib.PH_SOLVE_FAILED
    with pytest.raises(_lib.PhError):
        srv.result(t, big.ndofs)
    small = SolveRequest("isentropic_vortex", n_cells=2, poly_degree=2, final_time=0.01)
    t2 = srv.submit_request(small)
    assert srv.wait(t2, 60.0) == _lib.PH_SOLVE_DONE
    srv.result(t2, small.ndofs)
    srv.close()


@pytest.mark.gpu
def test_a_poisson_stream_through_the_native_server():
    rng = np.random.default_rng(20261203)
    times = poisson_arrivals(200.0, 16, rng)
    reqs = [SolveRequest("isentropic_vortex", n_cells=int(rng.integers(2, 5)), poly_degree=int(rng.integers(2, 5)),
                         mach=float(rng.uniform(0.1, 0.4)), final_time=0.05) for _ in times]
    srv = Server(1 << 30, _lib.PH_FP32_RESIDUAL, chunk=8)
    stats = serve_native(srv, list(zip(times, reqs)))
    srv.close()
    assert len(stats.completed) == 16
    assert all(c.latency > 0 and c.status == 0 for c in stats.completed)
    assert stats.max_in_flight >= 1 and stats.percentile(99) >= stats.percentile(50)
