"""Batched and served solves: many independent periodic-cube Euler solves resident on one
GPU, stepped together (the parameter-swept snapshot solves of the reference's
AdaptiveSamplingBase::solveSnapshotFOM, src/reduced_order/adaptive_sampling_base.cpp:255-265,
each of which runs FlowSolver::run, src/flow_solver/flow_solver.cpp:427-600).

  Batch .............. ctypes view of the ph_batch_* C-ABI (arena budget, admission,
                       graph-replayed steps, completion polling, read-back, release)
  SolveRequest ....... one solve: flow case, mesh (affine or sine-warped), order, Mach number,
                       vortex parameters, final time; builds the initial state and time step
  SnapshotServer ..... continuous batching: requests that arrive while others run are admitted
                       as the HBM budget frees up, stepped in chunks with a bounded amount of
                       work in flight, retired as they finish; records per-solve latency
  Server ............. the same loop in native code behind a thread-safe submission queue
                       (ph_server_*): submit from any thread, poll / wait, collect results
  serve_native ....... a stream of timed arrivals through a Server, with per-solve latency
  autotune ........... the tile-shape autotuner of the batched stage kernel
"""
from __future__ import annotations

import ctypes
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .dg import isentropic_vortex_primitive, tgv_primitive
from .prm import Parameters

TWO_PI = 6.28318530717958623200


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def autotune(poly_degree: int, precision: int = _lib.PH_FP32_RESIDUAL, curvilinear: bool = False):
    """Times the tile-shape variants of the batched stage kernel for (order, mesh kind) and keeps
    the fastest for this process. Returns (best variant, [ms per stage launch of each variant])."""
    L = _lib.load()
    best, nv = ctypes.c_int(0), ctypes.c_int(0)
    ms = (ctypes.c_double * 4)()
    _lib.check(L.ph_batch_autotune(poly_degree, precision, int(curvilinear), ctypes.byref(best), ms, ctypes.byref(nv)))
    return int(best.value), [float(ms[i]) for i in range(nv.value)]


def mesh_node_xyz(mesh: _lib.PhMeshDesc, poly_degree: int) -> np.ndarray:
    n1 = poly_degree + 1
    out = np.empty((mesh.n_cells_per_direction ** 3, n1 ** 3, 3))
    _lib.check(_lib.load().ph_mesh_node_xyz(ctypes.byref(mesh), poly_degree, _dp(out)))
    return out


def solve_bytes(mesh: _lib.PhMeshDesc, params: _lib.PhParams) -> int:
    """Device bytes one solve takes from a batch's HBM budget."""
    v = ctypes.c_size_t(0)
    _lib.check(_lib.load().ph_batch_bytes(ctypes.byref(mesh), ctypes.byref(params), ctypes.byref(v)))
    return int(v.value)


class Batch:
    """A batch of solves sharing one device arena of `budget_bytes` (ph_batch_*)."""

    def __init__(self, budget_bytes: int, precision: int = _lib.PH_FP32_RESIDUAL):
        self.L = _lib.load()
        self.precision = precision
        h = ctypes.c_void_p()
        _lib.check(self.L.ph_batch_create(ctypes.c_size_t(int(budget_bytes)), precision, None, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None:
            self.L.ph_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def bytes_for(self, mesh, params) -> int:
        return solve_bytes(mesh, params)

    def admit(self, mesh, params, U0: np.ndarray, dt: float, nsteps: int):
        """Slot id, or None when the budget has no room now."""
        U0 = np.ascontiguousarray(U0, dtype=np.float64)
        slot = ctypes.c_int(-1)
        rc = self.L.ph_batch_admit(self._h, ctypes.byref(mesh), ctypes.byref(params), _dp(U0), dt, nsteps,
                                   ctypes.byref(slot))
        if rc == _lib.PH_ERR_NOMEM:
            return None
        _lib.check(rc)
        return int(slot.value)

    def step(self, nsteps: int):
        _lib.check(self.L.ph_batch_step(self._h, nsteps))

    def poll(self, slot: int) -> bool:
        v = ctypes.c_int(0)
        _lib.check(self.L.ph_batch_poll(self._h, slot, ctypes.byref(v)))
        return bool(v.value)

    def progress(self, slot: int):
        d, n = ctypes.c_int(0), ctypes.c_int(0)
        _lib.check(self.L.ph_batch_progress(self._h, slot, ctypes.byref(d), ctypes.byref(n)))
        return int(d.value), int(n.value)

    @property
    def active(self) -> int:
        v = ctypes.c_int(0)
        _lib.check(self.L.ph_batch_active(self._h, ctypes.byref(v)))
        return int(v.value)

    def state(self, slot: int, ndofs: int) -> np.ndarray:
        U = np.empty(ndofs)
        _lib.check(self.L.ph_batch_get_state(self._h, slot, _dp(U)))
        return U

    def status(self, slot: int) -> int:
        v = ctypes.c_uint32(0)
        _lib.check(self.L.ph_batch_status(self._h, slot, ctypes.byref(v)))
        return int(v.value)

    def release(self, slot: int):
        _lib.check(self.L.ph_batch_release(self._h, slot))

    def fence(self) -> int:
        t = ctypes.c_longlong(0)
        _lib.check(self.L.ph_batch_fence(self._h, ctypes.byref(t)))
        return int(t.value)

    def wait(self, ticket: int):
        _lib.check(self.L.ph_batch_fence_wait(self._h, ticket))

    @property
    def launches(self) -> int:
        v = ctypes.c_longlong(0)
        _lib.check(self.L.ph_batch_launches(self._h, ctypes.byref(v)))
        return int(v.value)


@dataclass
class SolveRequest:
    """One periodic-cube Euler solve (split form, CH two-point flux + Roe dissipation, RK4)."""
    flow_case: str = "isentropic_vortex"          # or "taylor_green_vortex"
    n_cells: int = 4
    poly_degree: int = 3
    left: float = 0.0
    right: float = 10.0
    warp: float = 0.0
    mach: float = 0.5
    beta: float = 5.0                             # vortex strength (velocity perturbation beta/(2 pi) e^{(1-r^2)/2})
    direction: tuple = (1.0, 0.0, 0.0)
    center: tuple = (5.0, 5.0)
    final_time: float = 1.0
    cfl: float = 0.1
    two_point: str = "CH"
    conv: str = "two_point_flux_with_roe_dissipation"
    rk: str = "rk4_ex"
    gamma: float = 1.4
    tag: object = None

    def parameters(self) -> Parameters:
        return Parameters.from_dict({
            "dimension": 3, "pde_type": "euler", "use_weak_form": False, "flux_nodes_type": "GLL",
            "use_split_form": True, "two_point_num_flux_type": self.two_point, "conv_num_flux": self.conv,
            "flux_reconstruction": "cDG", "all_boundaries_are_periodic": True,
            "ODE solver/ode_solver_type": "runge_kutta", "ODE solver/runge_kutta_method": self.rk,
            "euler/mach_infinity": self.mach, "euler/gamma_gas": self.gamma,
            "flow_solver/flow_case_type": self.flow_case, "flow_solver/poly_degree": self.poly_degree,
            "flow_solver/final_time": self.final_time, "flow_solver/courant_friedrichs_lewy_number": self.cfl,
            "flow_solver/grid/grid_left_bound": self.left, "flow_solver/grid/grid_right_bound": self.right,
            "flow_solver/grid/number_of_grid_elements_per_dimension": self.n_cells,
        })

    def mesh(self) -> _lib.PhMeshDesc:
        return _lib.PhMeshDesc(self.n_cells, 0, self.left, self.right, self.warp, self.poly_degree)

    @property
    def ndofs(self) -> int:
        return self.n_cells ** 3 * 5 * (self.poly_degree + 1) ** 3

    def primitive(self, X: np.ndarray, t: float = 0.0):
        x, y, z = X[..., 0], X[..., 1], X[..., 2]
        if self.flow_case == "taylor_green_vortex":
            return tgv_primitive(x, y, z, self.gamma, self.mach)
        # beta is the vortex strength of the usual convention (velocity perturbation
        # beta/(2 pi) e^{(1-r^2)/2}); the reference's form takes the amplitude beta e^{1/2}/(2 pi)
        amp = self.beta * math.exp(0.5) / (2.0 * math.pi)
        return isentropic_vortex_primitive(x, y, z, self.gamma, amp, self.mach, self.direction,
                                           self.center, t, self.right - self.left)

    def conservative(self, X: np.ndarray, t: float = 0.0) -> np.ndarray:
        rho, u, v, w, p = self.primitive(X, t)
        E = p / (self.gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
        return np.ascontiguousarray(np.stack([rho, rho * u, rho * v, rho * w, E], axis=1).reshape(-1))

    def node_xyz(self) -> np.ndarray:
        return mesh_node_xyz(self.mesh(), self.poly_degree)

    def initial_state(self) -> np.ndarray:
        return self.conservative(self.node_xyz())

    def time_step(self, U0: np.ndarray):
        """CFL x node spacing / max(|v| + c) of the initial state (the reference's
        adaptive_time_step formula, periodic_turbulence.cpp:361-369), shortened so that an
        integer number of steps ends at final_time. Returns (dt, nsteps)."""
        n1 = self.poly_degree + 1
        U = U0.reshape(-1, 5, n1 ** 3)
        rho = U[:, 0]
        v2 = (U[:, 1] ** 2 + U[:, 2] ** 2 + U[:, 3] ** 2) / (rho * rho)
        p = (self.gamma - 1.0) * (U[:, 4] - 0.5 * rho * v2)
        wave = float(np.max(np.sqrt(v2) + np.sqrt(self.gamma * p / rho)))
        dx = (self.right - self.left) / (self.n_cells * n1)
        dt = self.cfl * dx / wave
        nsteps = max(1, int(math.ceil(self.final_time / dt - 1e-12)))
        return self.final_time / nsteps, nsteps

    def prepare(self):
        """Initial state and time step, computed once (the request's payload)."""
        if getattr(self, "_prepared", None) is None:
            U0 = self.initial_state()
            self._prepared = (U0, *self.time_step(U0))
        return self._prepared

    def exact_state(self) -> np.ndarray:
        """Exact solution at final_time (the vortex translated with the free stream)."""
        if self.flow_case != "isentropic_vortex":
            raise ValueError("exact solution only for the isentropic vortex")
        return self.conservative(self.node_xyz(), self.final_time)


@dataclass
class Completed:
    request: SolveRequest
    arrival: float
    admitted: float
    done: float
    steps: int
    state: np.ndarray | None = None
    status: int = 0

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeStats:
    completed: list = field(default_factory=list)
    makespan: float = 0.0
    max_in_flight: int = 0
    admissions_deferred: int = 0

    def percentile(self, q: float) -> float:
        lat = sorted(c.latency for c in self.completed)
        if not lat:
            return float("nan")
        k = min(len(lat) - 1, max(0, int(math.ceil(q / 100.0 * len(lat))) - 1))
        return lat[k]

    @property
    def solves_per_s(self) -> float:
        return len(self.completed) / self.makespan if self.makespan > 0 else float("nan")


class SnapshotServer:
    """Continuous batching over a Batch.

    Each loop iteration: admit every arrived request the budget can hold (FIFO: a request that
    does not fit waits, and blocks the ones behind it, so large requests are not starved),
    enqueue `chunk` RK steps of all resident solves (one graph replay per step), and wait for
    the chunk before last so at most two chunks are in flight; then retire the solves whose
    last step the GPU has completed. Latency = completion time - arrival time.
    """

    def __init__(self, batch, chunk: int = 16, keep_states: bool = False, clock=time.perf_counter,
                 precision: int = _lib.PH_FP32_RESIDUAL, admit_slice: float = 0.004):
        self.batch = batch
        self.chunk = chunk
        self.keep_states = keep_states
        self.clock = clock
        self.precision = precision
        self.admit_slice = admit_slice   # host time per loop spent admitting while solves are resident

    def _prepare(self, req: SolveRequest):
        U0, dt, nsteps = req.prepare()
        return req.mesh(), req.parameters().to_ph_params(self.precision), U0, dt, nsteps

    def run(self, arrivals):
        """arrivals: list of (arrival time in s from start, SolveRequest). Returns ServeStats."""
        pending = deque(sorted(arrivals, key=lambda a: a[0]))
        queue = deque()
        resident = {}          # slot -> (request, arrival, admitted, nsteps)
        stats = ServeStats()
        t0 = self.clock()
        tickets = deque()
        while pending or queue or resident:
            now = self.clock() - t0
            while pending and pending[0][0] <= now:
                queue.append(pending.popleft())
            # admit in FIFO order; while solves are resident, only for a slice of host time, so
            # the queued GPU work keeps running while the host sets up the newcomers
            t_end = self.clock() + self.admit_slice if resident else float("inf")
            while queue and self.clock() < t_end:
                arr, req = queue[0]
                mesh, prm, U0, dt, nsteps = self._prepare(req)
                slot = self.batch.admit(mesh, prm, U0, dt, nsteps)
                if slot is None:
                    stats.admissions_deferred += 1
                    break
                queue.popleft()
                resident[slot] = (req, arr, self.clock() - t0, nsteps)
                if len(resident) == 1:
                    t_end = self.clock() + self.admit_slice
            stats.max_in_flight = max(stats.max_in_flight, len(resident))
            if not resident:
                if pending:
                    time.sleep(max(0.0, min(pending[0][0] - (self.clock() - t0), 0.01)))
                continue
            if self.batch.active > 0:
                self.batch.step(self.chunk)
                tickets.append(self.batch.fence())
                if len(tickets) > 2:
                    self.batch.wait(tickets.popleft())
            for slot in list(resident):
                if self.batch.poll(slot):
                    req, arr, adm, nsteps = resident.pop(slot)
                    done = self.clock() - t0
                    st = self.batch.state(slot, req.ndofs) if self.keep_states else None
                    flags = self.batch.status(slot)
                    self.batch.release(slot)
                    stats.completed.append(Completed(req, arr, adm, done, nsteps, st, flags))
            if self.batch.active == 0 and resident:
                # every resident solve has been enqueued to its end: wait for the GPU
                while tickets:
                    self.batch.wait(tickets.popleft())
        stats.makespan = self.clock() - t0
        return stats


class Server:
    """ph_server_*: a worker thread of the library runs the continuous-batching loop over its
    own batch; submissions return a ticket at once and may come from any thread."""

    def __init__(self, budget_bytes: int, precision: int = _lib.PH_FP32_RESIDUAL, chunk: int = 16,
                 admit_slice: float = 0.004):
        self.L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self.L.ph_server_create(ctypes.c_size_t(int(budget_bytes)), precision, chunk, admit_slice,
                                           ctypes.byref(h)))
        self._h = h
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None) is not None:
            self.L.ph_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit(self, mesh, params, U0: np.ndarray, dt: float, nsteps: int) -> int:
        t = ctypes.c_longlong(0)
        U0 = np.ascontiguousarray(U0, dtype=np.float64)
        _lib.check(self.L.ph_server_submit(self._h, ctypes.byref(mesh), ctypes.byref(params), _dp(U0), dt, nsteps,
                                           ctypes.byref(t)))
        return int(t.value)

    def submit_request(self, req: SolveRequest) -> int:
        U0, dt, nsteps = req.prepare()
        return self.submit(req.mesh(), req.parameters().to_ph_params(self.precision), U0, dt, nsteps)

    def poll(self, ticket: int) -> int:
        st = ctypes.c_int(0)
        _lib.check(self.L.ph_server_poll(self._h, ticket, ctypes.byref(st)))
        return int(st.value)

    def wait(self, ticket: int, timeout: float = 3600.0) -> int:
        st = ctypes.c_int(0)
        _lib.check(self.L.ph_server_wait(self._h, ticket, timeout, ctypes.byref(st)))
        return int(st.value)

    def result(self, ticket: int, ndofs: int):
        """(final state, status word, (seconds to admission, seconds to completion)); raises
        PhError for a failed solve."""
        U = np.empty(ndofs)
        flags = ctypes.c_uint32(0)
        sec = (ctypes.c_double * 2)()
        _lib.check(self.L.ph_server_result(self._h, ticket, _dp(U), ctypes.byref(flags), sec))
        return U, int(flags.value), (float(sec[0]), float(sec[1]))

    def stats(self):
        out = (ctypes.c_longlong * 4)()
        _lib.check(self.L.ph_server_stats(self._h, out))
        return {"queued": int(out[0]), "admissions_deferred": int(out[1]), "max_resident": int(out[2]),
                "launches": int(out[3])}


def serve_native(server: Server, arrivals, keep_states: bool = False, clock=time.perf_counter):
    """arrivals: list of (arrival time in s from start, SolveRequest). Each request is prepared
    (initial state, time step) and submitted at its arrival time; the results are collected as
    they finish. Latency = completion - arrival. Returns ServeStats."""
    import threading
    stats = ServeStats()
    order = sorted(arrivals, key=lambda a: a[0])
    submitted = []                 # (ticket, request, arrival, seconds after start at submission)
    lock = threading.Lock()
    t0 = clock()

    def submitter():
        for arr, req in order:
            delay = arr - (clock() - t0)
            if delay > 0:
                time.sleep(delay)
            ticket = server.submit_request(req)
            with lock:
                submitted.append((ticket, req, arr, clock() - t0))

    th = threading.Thread(target=submitter)
    th.start()
    done = 0
    while done < len(order):
        with lock:
            pending = list(submitted)
            submitted.clear()
        if not pending:
            time.sleep(0.001)
            continue
        for ticket, req, arr, t_sub in pending:
            server.wait(ticket)
            U, flags, (t_adm, t_done) = server.result(ticket, req.ndofs)
            _, _, nsteps = req.prepare()
            stats.completed.append(Completed(req, arr, t_sub + t_adm, t_sub + t_done, nsteps,
                                             U if keep_states else None, flags))
            done += 1
    th.join()
    stats.makespan = max(c.done for c in stats.completed) if stats.completed else 0.0
    s = server.stats()
    stats.max_in_flight = s["max_resident"]
    stats.admissions_deferred = s["admissions_deferred"]
    return stats


def poisson_arrivals(rate: float, count: int, rng: np.random.Generator):
    """Arrival times of a Poisson process of `rate` per second."""
    return np.cumsum(rng.exponential(1.0 / rate, size=count))
