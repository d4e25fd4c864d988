"""Host-side mirror of the reference's DGBase/DGStrong, RungeKuttaODESolver and
FlowSolver surface over the C-ABI library.

Reference interfaces mirrored (same names and argument meaning):
  DGBase::solution / right_hand_side ............ src/dg/dg_base.hpp:396, :409
  DGBase::assemble_residual ..................... src/dg/dg_base.hpp:571
  DGBase::apply_inverse_global_mass_matrix ...... src/dg/dg_base.hpp:267
  DGBase::set_current_time ...................... src/dg/dg_base.hpp
  ODESolverBase::step_in_time / advance_solution_time  src/ode_solver/ode_solver_base.h:70, .cpp:262-322
  FlowSolver::run (unsteady loop) ............... src/flow_solver/flow_solver.cpp:427-600
  PeriodicTurbulence::get_constant_time_step .... src/flow_solver/flow_solver_cases/periodic_turbulence.cpp:115-127
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .prm import Parameters


def _ptr(a: np.ndarray) -> int:
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def gll_nodes(n: int) -> np.ndarray:
    """Gauss-Lobatto nodes on [0,1] (the FE_DGQ support points)."""
    if n == 1:
        return np.array([0.5])
    m = n - 1
    z = -np.cos(np.pi * np.arange(n) / m)
    for _ in range(100):
        # Newton on P_m'(z) at the interior points
        p0, p1 = np.ones_like(z), z.copy()
        for k in range(2, m + 1):
            p0, p1 = p1, ((2 * k - 1) * z * p1 - (k - 1) * p0) / k
        with np.errstate(divide="ignore", invalid="ignore"):
            dp = m * (z * p1 - p0) / (z * z - 1.0)
            d2p = (2.0 * z * dp - m * (m + 1.0) * p1) / (1.0 - z * z)
            dz = np.where(np.abs(np.abs(z) - 1.0) < 1e-15, 0.0, dp / d2p)
        z = z - dz
        if np.max(np.abs(dz)) < 1e-16:
            break
    x = 0.5 * (z + 1.0)
    x[0], x[-1] = 0.0, 1.0
    return x


class DGStrong:
    """Strong-form DG/FR discretisation on a periodic cube, evaluated on the B200."""

    def __init__(self, parameters: Parameters, precision: int = _lib.PH_FP64, cell_order: int = 0,
                 stream: int | None = None, warp: float = 0.0, mapping_support_points: np.ndarray | None = None,
                 slab: tuple[int, int] | None = None, halo=None, dist=None, boundaries=None):
        """boundaries: six boundary conditions, for the sides x-, x+, y-, y+, z-, z+ (names of
        _lib.BOUNDARY such as "wall", "riemann_farfield", or boundary_id values; "periodic" / 0
        keeps a periodic pair). None: the periodic cube.
        warp != 0 gives the sine-warped (curvilinear) cube: every coordinate moves by
        warp (L/2pi) sin(2pi(x-l)/L) sin(2pi(y-l)/L) sin(2pi(z-l)/L), mapping degree = p.
        mapping_support_points ([cell][3][(p+1)^3], GLL points) gives any other curved mapping.
        slab = (z_first, z_count): this process's layers of a mesh shared by several GPUs
        (philip_b200.slab); halo: the object whose `callback` exchanges the partition faces
        (and whose `sum_callback`, when present, sums the relaxation RK entropy integrals over
        the ranks);
        dist: the torch.distributed module (initialised) over which the integrals, maxima and
        error norms of the slabs are combined into the mesh's (None: this slab's share)."""
        self.L = _lib.load()
        self.parameters = parameters
        self.params = parameters.to_ph_params(precision)
        left, right = parameters.grid_bounds
        self.warp = float(warp)
        self.mesh = _lib.PhMeshDesc(parameters.n_cells, cell_order, left, right, self.warp, parameters.poly_degree)
        if mapping_support_points is not None:
            self._support = np.ascontiguousarray(mapping_support_points, dtype=np.float64)
            self.mesh.mapping_support_points = self._support.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if boundaries is not None:
            for f, t in enumerate(_lib.boundary_ids(boundaries)):
                self.mesh.boundary_type[f] = t
        h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream) if stream else None
        if slab is None:
            _lib.check(self.L.ph_ctx_create(ctypes.byref(self.mesh), ctypes.byref(self.params), st, ctypes.byref(h)))
        else:
            _lib.check(self.L.ph_ctx_create_slab(ctypes.byref(self.mesh), ctypes.byref(self.params), int(slab[0]),
                                                 int(slab[1]), st, ctypes.byref(h)))
        self._h = h
        self.slab = slab
        self.halo = halo
        self.dist = dist if (slab is not None and dist is not None and dist.is_initialized()
                             and dist.get_world_size() > 1) else None
        if halo is not None:
            _lib.check(self.L.ph_set_halo_exchange(h, halo.callback, None))
            if getattr(halo, "sum_callback", None) is not None:   # relaxation RK: the mesh's entropy sums
                _lib.check(self.L.ph_set_rank_sum(h, halo.sum_callback, None))
        self.n_dofs = int(self.L.ph_ndofs(h))
        self.poly_degree = parameters.poly_degree
        self.n_cells = parameters.n_cells ** 2 * (slab[1] if slab is not None else parameters.n_cells)
        self.n_shape = (self.poly_degree + 1) ** 3
        self.right_hand_side = np.zeros(self.n_dofs)
        self.current_time = 0.0

    def __del__(self):
        if getattr(self, "_h", None) is not None:
            self.L.ph_ctx_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # -- state
    @property
    def solution(self) -> np.ndarray:
        U = np.empty(self.n_dofs)
        _lib.check(self.L.ph_get_state(self._h, _ptr(U), _lib.PH_HOST))
        return U

    @solution.setter
    def solution(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.size != self.n_dofs:
            raise ValueError("state size mismatch")
        _lib.check(self.L.ph_set_state(self._h, _ptr(U), _lib.PH_HOST))

    def set_current_time(self, t: float):
        self.current_time = t

    # -- residual and mass inverse
    def assemble_residual(self, compute_dRdW: bool = False, compute_dRdX: bool = False,
                          compute_d2R: bool = False, CFL_mass: float = 0.0):
        if compute_dRdW or compute_dRdX or compute_d2R:
            raise NotImplementedError("implicit/adjoint derivatives are outside the explicit path")
        U = self.solution
        _lib.check(self.L.ph_residual(self._h, _ptr(U), _ptr(self.right_hand_side), _lib.PH_HOST))

    def residual_of(self, U: np.ndarray) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.empty(self.n_dofs)
        _lib.check(self.L.ph_residual(self._h, _ptr(U), _ptr(R), _lib.PH_HOST))
        return R

    def apply_inverse_global_mass_matrix(self, input_vector: np.ndarray, output_vector: np.ndarray,
                                         use_auxiliary_eq: bool = False):
        if use_auxiliary_eq:
            raise NotImplementedError("the auxiliary mass inverse is applied inside the residual")
        inp = np.ascontiguousarray(input_vector, dtype=np.float64)
        if not (output_vector.dtype == np.float64 and output_vector.flags["C_CONTIGUOUS"]):
            raise ValueError("output_vector must be a contiguous float64 array")
        _lib.check(self.L.ph_apply_inverse_mass(self._h, _ptr(inp), _ptr(output_vector), _lib.PH_HOST))

    # -- geometry
    def cell_ijk(self) -> np.ndarray:
        out = np.empty((self.n_cells, 3), dtype=np.int32)
        _lib.check(self.L.ph_cell_ijk(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return out

    def node_coordinates(self) -> np.ndarray:
        """Physical coordinates of the solution support points, [cell][node][3]."""
        out = np.empty((self.n_cells, self.n_shape, 3))
        _lib.check(self.L.ph_node_xyz(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    # -- reductions over the slabs of a shared mesh (identity on a whole mesh)
    def _allreduce(self, values, op: str) -> np.ndarray:
        if self.dist is None:
            return np.asarray(values, dtype=np.float64)
        import torch
        dev = "cuda" if self.dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor(np.asarray(values, dtype=np.float64), device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM if op == "sum" else self.dist.ReduceOp.MAX)
        return t.cpu().numpy()

    def global_max(self, value: float) -> float:
        return float(self._allreduce([value], "max")[0])

    def global_sum(self, value: float) -> float:
        return float(self._allreduce([value], "sum")[0])

    # -- diagnostics
    def integrals(self) -> np.ndarray:
        """Kinetic energy, enstrophy, vorticity-based dissipation rate (volume averages) and the
        maximum wave speed; a slab's share of the first three without `dist`."""
        out = np.zeros(4)
        _lib.check(self.L.ph_integrals(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        if self.dist is not None:
            out = np.concatenate([self._allreduce(out[:3], "sum"), self._allreduce(out[3:], "max")])
        return out

    def integrated_quantities(self) -> np.ndarray:
        """The nine quantities of PeriodicTurbulence::compute_and_update_integrated_quantities
        (periodic_turbulence.cpp:439-672) in IntegratedQuantitiesEnum order
        (_lib.INTEGRATED_QUANTITIES), each over the domain volume."""
        out = np.zeros(len(_lib.INTEGRATED_QUANTITIES))
        _lib.check(self.L.ph_integrated_quantities(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return self._allreduce(out, "sum") if self.dist is not None else out

    def kinetic_energy_rate(self) -> float:
        """dKE/dt of the current solution from its time derivative M^-1 R (ph_kinetic_energy_rate)."""
        v = ctypes.c_double(0.0)
        _lib.check(self.L.ph_kinetic_energy_rate(self._h, ctypes.byref(v)))
        return float(v.value)

    def apply_limiter(self, dt: float):
        """BoundPreservingLimiter::limit on the current solution for a stage of time step dt
        (the context's positivity-preserving limiter, limiter/bound_preserving_limiter)."""
        _lib.check(self.L.ph_limit(self._h, dt))

    def status(self) -> int:
        v = ctypes.c_uint32(0)
        _lib.check(self.L.ph_status(self._h, ctypes.byref(v)))
        return int(v.value)


class RungeKuttaODESolver:
    """Explicit RK stepping on the device-resident state: the Butcher methods of
    RungeKuttaODESolver and the low-storage methods of LowStorageRungeKuttaODESolver
    (src/ode_solver/low_storage_runge_kutta_ode_solver.cpp), with the latter's error-based
    step-size control."""

    def __init__(self, dg: DGStrong):
        self.dg = dg
        self.current_time = 0.0
        self.current_iteration = 0
        self.epsilon = [1.0, 1.0, 1.0]   # step-size controller history (low_storage_runge_kutta_ode_solver.cpp:11)
        self.relaxation_parameter = 1.0  # relaxation RK: the last step's gamma

    def step_in_time(self, dt: float, pseudotime: bool = False, nsteps: int = 1):
        if pseudotime:
            raise NotImplementedError("pseudotime stepping belongs to the steady solvers")
        _lib.check(self.dg.L.ph_rk_step(self.dg.handle, dt, nsteps))
        if self.dg.parameters.use_relaxation_runge_kutta:
            # each step advanced gamma dt (RungeKuttaODESolver::adjust_time_step)
            g, elapsed = ctypes.c_double(1.0), ctypes.c_double(0.0)
            _lib.check(self.dg.L.ph_rk_relaxation(self.dg.handle, ctypes.byref(g), ctypes.byref(elapsed)))
            self.relaxation_parameter = float(g.value)
            self.current_iteration += nsteps
            self.current_time += float(elapsed.value)
        else:
            for _ in range(nsteps):
                self.current_iteration += 1
                self.current_time += dt
        self.dg.set_current_time(self.current_time)

    def step_in_time_with_records(self, dt: float, nsteps: int, record_every: int):
        """nsteps steps of dt with the four ph_integrals values reduced on the device after
        every record_every-th step (ph_run); returns [(time, KE, enstrophy, eps, wave)] with
        the times this solver's clock shows after those steps."""
        nrec = nsteps // record_every if record_every > 0 else 0
        rows = np.zeros((max(nrec, 1), 4))
        _lib.check(self.dg.L.ph_run(self.dg.handle, dt, nsteps, record_every,
                                    rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        out = []
        for s in range(nsteps):
            self.current_iteration += 1
            self.current_time += dt
            if record_every > 0 and (s + 1) % record_every == 0 and (s + 1) // record_every <= nrec:
                out.append((self.current_time, *rows[(s + 1) // record_every - 1]))
        self.dg.set_current_time(self.current_time)
        return out

    def error_norm(self) -> float:
        """Weighted RMS error estimate of the last low-storage step (over the whole mesh when
        the slabs of a shared mesh combine their sums)."""
        w = ctypes.c_double(0.0)
        _lib.check(self.dg.L.ph_rk_error_norm(self.dg.handle, ctypes.byref(w)))
        if self.dg.dist is None:
            return float(w.value)
        s = self.dg._allreduce([w.value ** 2 * self.dg.n_dofs, float(self.dg.n_dofs)], "sum")
        return float(math.sqrt(s[0] / s[1]))

    def get_automatic_error_adaptive_step_size(self, dt: float) -> float:
        """LowStorageRungeKuttaODESolver::get_automatic_error_adaptive_step_size
        (low_storage_runge_kutta_ode_solver.cpp:80-110): PID controller on eps = 1 / w."""
        from .prm import RK_ORDER
        prm = self.dg.parameters
        order = RK_ORDER[prm.get("ODE solver/runge_kutta_method")]
        b1, b2, b3 = (float(prm.get(f"ODE solver/low-storage rk solver/beta{i}")) for i in (1, 2, 3))
        w = self.error_norm()
        self.epsilon = [1.0 / w, self.epsilon[0], self.epsilon[1]]
        e0, e1, e2 = self.epsilon
        return e0 ** (b1 / order) * e1 ** (b2 / order) * e2 ** (b3 / order) * dt

    def get_automatic_initial_step_size(self, dt: float = 0.0) -> float:
        """LowStorageRungeKuttaODESolver::get_automatic_initial_step_size
        (low_storage_runge_kutta_ode_solver.cpp:112-175)."""
        u_n = self.dg.solution
        n = u_n.size
        rhs = np.empty(n)
        self.dg.apply_inverse_global_mass_matrix(self.dg.residual_of(u_n), rhs)
        gmax = self.dg.global_max
        d0 = gmax(float(np.max(np.abs(u_n))))
        d1 = gmax(float(np.max(np.abs(rhs))))
        h0 = 1e-6 if (d0 < 1e-5 or d1 < 1e-5) else 0.01 * d0 / d1
        u1 = u_n + h0 * rhs
        rhs1 = np.empty(n)
        self.dg.apply_inverse_global_mass_matrix(self.dg.residual_of(u1), rhs1)
        d2 = gmax(float(np.max(np.abs(rhs1 - rhs)))) / h0
        h1 = max(1e-6, h0 * 1e-3) if max(d1, d2) <= 1e-15 else 0.01 / max(d1, d2)
        self.dg.solution = u_n
        return min(100.0 * h0, h1)

    def advance_solution_time(self, time_advance: float, dt: float):
        """ODESolverBase::advance_solution_time: steps of dt, the last one clipped."""
        final = self.current_time + time_advance
        while self.current_time < final:
            step = min(dt, final - self.current_time)
            self.step_in_time(step)


# --------------------------------------------------------------------------------
# Flow cases (periodic cube): Taylor-Green vortex and isentropic vortex
# --------------------------------------------------------------------------------
def tgv_primitive(x, y, z, gamma, mach):
    """InitialConditionFunction_TaylorGreenVortex (initial_condition_function.cpp:261-310)."""
    rho = np.ones_like(x)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    p = 1.0 / (gamma * mach * mach) + (1.0 / 16.0) * (np.cos(2.0 * x) + np.cos(2.0 * y)) * (np.cos(2.0 * z) + 2.0)
    return rho, u, v, w, p


def isentropic_vortex_primitive(x, y, z, gamma, beta, mach, direction, center=(0.0, 0.0), t=0.0, period=0.0):
    """Isentropic vortex translated with the free stream (initial_condition_function.cpp:643-690,
    with strength, Mach number and direction as parameters)."""
    dx = x - center[0] - mach * direction[0] * t
    dy = y - center[1] - mach * direction[1] * t
    if period > 0.0:
        dx = dx - period * np.round(dx / period)
        dy = dy - period * np.round(dy / period)
    om = beta * np.exp(-0.5 * (dx * dx + dy * dy))
    dT = -(gamma - 1.0) / 2.0 * om * om
    rho = (1.0 + dT) ** (1.0 / (gamma - 1.0))
    u = mach * direction[0] - dy * om
    v = mach * direction[1] + dx * om
    w = mach * direction[2] * np.ones_like(x)
    p = 1.0 / gamma * (1.0 + dT) ** (gamma / (gamma - 1.0))
    return rho, u, v, w, p


def conservative_state(dg: DGStrong, prim) -> np.ndarray:
    """Nodal interpolation (VectorTools::interpolate) into the reference DoF layout."""
    rho, u, v, w, p = prim
    gamma = dg.params.gamma_gas
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    cons = np.stack([rho, rho * u, rho * v, rho * w, E], axis=1)   # [cell][state][node]
    return np.ascontiguousarray(cons.reshape(-1))


RESTART_MAGIC = b"PHB2RST1"


def restart_filename_without_extension(index: int) -> str:
    """FlowSolver::get_restart_filename_without_extension (flow_solver.cpp:168-180)."""
    return f"restart-{index:05d}"


def write_restart_state(path: str, U: np.ndarray, time: float, iteration: int, dt: float):
    """Device-state checkpoint: magic, DOF count, time, iteration, time step, then the state in
    the reference DoF order (little-endian float64). It stands in for deal.II's
    triangulation + SolutionTransfer serialisation, which this path does not link."""
    with open(path, "wb") as f:
        f.write(RESTART_MAGIC)
        np.array([U.size, iteration], dtype="<i8").tofile(f)
        np.array([time, dt], dtype="<f8").tofile(f)
        np.ascontiguousarray(U, dtype="<f8").tofile(f)


def read_restart_state(path: str):
    with open(path, "rb") as f:
        if f.read(8) != RESTART_MAGIC:
            raise ValueError(f"{path}: not a restart state file")
        n, iteration = np.fromfile(f, dtype="<i8", count=2)
        time, dt = np.fromfile(f, dtype="<f8", count=2)
        U = np.fromfile(f, dtype="<f8", count=int(n))
    if U.size != n:
        raise ValueError(f"{path}: truncated")
    return U, float(time), int(iteration), float(dt)


class FlowSolver:
    """FlowSolver::run for the periodic-cube cases (TGV; isentropic vortex), with the
    reference's restart files (flow_solver.cpp:240-395): restart-NNNNN.prm (the input
    parameters with the ODE solver's initial time / iteration / time step and the restart
    switches updated), the unsteady data table, and the state checkpoint."""

    def __init__(self, parameters: Parameters, precision: int = _lib.PH_FP64, cell_order: int = 0,
                 warp: float = 0.0, stream: int | None = None, slab: tuple[int, int] | None = None,
                 halo=None, dist=None, boundaries=None):
        """slab / halo / dist: this process's share of a mesh over several GPUs (DGStrong);
        the time steps, integrals and table rows are then the whole mesh's on every rank.
        boundaries: the non-periodic sides (DGStrong)."""
        self.parameters = parameters
        self.dg = DGStrong(parameters, precision=precision, cell_order=cell_order, warp=warp, stream=stream,
                           slab=slab, halo=halo, dist=dist, boundaries=boundaries)
        self.ode_solver = RungeKuttaODESolver(self.dg)
        self.flow_case = parameters.get("flow_solver/flow_case_type")
        X = self.dg.node_coordinates()
        gamma, mach = self.dg.params.gamma_gas, self.dg.params.mach_infinity
        if self.flow_case == "taylor_green_vortex":
            prim = tgv_primitive(X[..., 0], X[..., 1], X[..., 2], gamma, mach)
        elif self.flow_case == "isentropic_vortex":
            m = math.sqrt(2.0 / gamma)
            beta = m * 5 * math.sqrt(2.0) / 4.0 / math.pi * math.exp(0.5)
            prim = isentropic_vortex_primitive(X[..., 0], X[..., 1], X[..., 2], gamma, beta, m,
                                               (math.cos(math.pi / 4), math.sin(math.pi / 4), 0.0))
        else:
            raise ValueError(f"flow_case_type {self.flow_case!r} is outside the periodic-cube cases")
        self.dg.solution = conservative_state(self.dg, prim)
        # SetInitialCondition::interpolate_initial_condition limits the interpolated state with the
        # Wang 2012 limiter (set_initial_condition.cpp:54-67), for a stage of the initial time step
        if parameters.get("limiter/bound_preserving_limiter") == "positivity_preservingWang2012":
            self.dg.apply_limiter(float(parameters.get("ODE solver/initial_time_step")))
        self.unsteady_data = []
        self.restart_dt = None
        # time POD (flow_solver.cpp:110-120): the snapshot matrix stays on the device
        self.snapshot_every = int(parameters.get("reduced order/output_snapshot_every_x_timesteps"))
        self.time_pod = None
        if self.snapshot_every != 0:
            from .pod import OnlinePOD
            self.time_pod = OnlinePOD(self.dg.n_dofs, 16)
            self.time_pod.addSnapshot(self.dg)
        if parameters.get("flow_solver/restart_computation_from_file").lower() == "true":
            self._restart_from_file()

    def _restart_dir(self) -> str:
        return self.parameters.get("flow_solver/restart_files_directory_name")

    def _table_name(self, index: int) -> str:
        return (self.parameters.get("flow_solver/unsteady_data_table_filename") + "-" +
                restart_filename_without_extension(index) + ".txt")

    def _restart_from_file(self):
        """FlowSolver constructor's restart branch (flow_solver.cpp:58-100, :452-541)."""
        import os
        idx = int(self.parameters.get("flow_solver/restart_file_index"))
        base = os.path.join(self._restart_dir(), restart_filename_without_extension(idx))
        U, t, it, dt = read_restart_state(base + ".sol")
        if U.size != self.dg.n_dofs:
            raise ValueError("restart state does not match the discretisation")
        self.dg.solution = U
        self.ode_solver.current_time = float(self.parameters.get("ODE solver/initial_time"))
        self.ode_solver.current_iteration = int(self.parameters.get("ODE solver/initial_iteration"))
        self.dg.set_current_time(self.ode_solver.current_time)
        self.restart_dt = float(self.parameters.get("ODE solver/initial_time_step"))
        table = os.path.join(self._restart_dir(), self._table_name(idx))
        if os.path.exists(table):
            rows = np.loadtxt(table, skiprows=1, ndmin=2)
            self.unsteady_data = [tuple(r) for r in rows]

    def output_restart_files(self, index: int, dt: float):
        """FlowSolver::output_restart_files + write_restart_parameter_file (flow_solver.cpp:240-395)."""
        import os
        d = self._restart_dir()
        base = os.path.join(d, restart_filename_without_extension(index))
        write_restart_state(base + ".sol", self.dg.solution, self.ode_solver.current_time,
                            self.ode_solver.current_iteration, dt)
        with open(os.path.join(d, self._table_name(index)), "w") as f:
            f.write("time kinetic_energy enstrophy vorticity_based_dissipation_rate max_wave_speed\n")
            for row in self.unsteady_data:
                f.write(" ".join(repr(float(v)) for v in row) + "\n")
        prm = self.parameters.with_values({
            "ODE solver/initial_desired_time_for_output_solution_every_dt_time_intervals":
                f"{self.ode_solver.current_time:.16e}",
            "ODE solver/initial_iteration": str(self.ode_solver.current_iteration),
            "ODE solver/initial_time": f"{self.ode_solver.current_time:.16e}",
            "ODE solver/initial_time_step": f"{dt:.16e}",
            "flow_solver/output_restart_files": "true",
            "flow_solver/restart_computation_from_file": "true",
            "flow_solver/restart_file_index": str(index),
        })
        with open(base + ".prm", "w") as f:   # written last, after the data it points to
            f.write(prm.to_text())

    def unsteady_data_row(self) -> dict:
        """One row of PeriodicTurbulence's unsteady data table (compute_unsteady_data_and_write_to_table,
        periodic_turbulence.cpp:925-972): the integrated quantities and the dissipation rates
        derived from them, under the reference's column names; the viscous-only columns only
        for Navier-Stokes, the angular momentum only when asked for."""
        q = dict(zip(_lib.INTEGRATED_QUANTITIES, self.dg.integrated_quantities()))
        viscous = self.parameters.get("pde_type") != "euler"
        re = float(self.parameters.get("navier_stokes/reynolds_number_inf"))
        row = {"time": self.ode_solver.current_time,
               "kinetic_energy": q["kinetic_energy"], "enstrophy": q["enstrophy"]}
        if viscous:
            row["eps_vorticity"] = 2.0 * q["enstrophy"] / re
        row["eps_pressure"] = -q["pressure_dilatation"]
        if viscous:
            row["eps_strain"] = 2.0 * q["viscosity_times_strain_rate_tensor_magnitude_sqr"] / re
            row["eps_dev_strain"] = 2.0 * q["viscosity_times_deviatoric_strain_rate_tensor_magnitude_sqr"] / re
        for k in ("incompressible_kinetic_energy", "incompressible_enstrophy", "incompressible_palinstrophy"):
            row[k] = q[k]
        if self.parameters.get("flow_solver/dipole_wall_collision/do_compute_angular_momentum").lower() == "true":
            row["angular_momentum"] = q["angular_momentum"]
        return row

    def _grid_spacing(self) -> float:
        left, right = self.parameters.grid_bounds
        ndof_per_state = self.parameters.n_cells ** 3 * self.dg.n_shape   # the whole mesh's
        return (right - left) / ndof_per_state ** (1.0 / 3.0)

    def constant_time_step(self) -> float:
        """PeriodicTurbulence::get_constant_time_step (periodic_turbulence.cpp:115-127)."""
        cst = float(self.parameters.get("flow_solver/constant_time_step"))
        if cst > 0.0:
            return cst
        return float(self.parameters.get("flow_solver/courant_friedrichs_lewy_number")) * self._grid_spacing()

    def adaptive_time_step(self) -> float:
        """PeriodicTurbulence::get_adaptive_time_step (periodic_turbulence.cpp:361-369):
        CFL x spacing / maximum convective wave speed (|v| + c) of the current state."""
        wave = self.dg.integrals()[3]
        return float(self.parameters.get("flow_solver/courant_friedrichs_lewy_number")) * self._grid_spacing() / wave

    def time_step(self) -> float:
        if self.parameters.get("flow_solver/adaptive_time_step").lower() == "true":
            return self.adaptive_time_step()
        return self.constant_time_step()

    def run(self, record_every: int = 1):
        final_time = float(self.parameters.get("flow_solver/final_time"))
        end_exact = self.parameters.get("flow_solver/end_exactly_at_final_time").lower() == "true"
        adaptive = self.parameters.get("flow_solver/adaptive_time_step").lower() == "true"
        error_adaptive = self.parameters.get("flow_solver/error_adaptive_time_step").lower() == "true"
        if adaptive and error_adaptive:
            raise ValueError("CFL-adaptation and error-adaptation cannot be used at the same time")
        write_restart = self.parameters.get("flow_solver/output_restart_files").lower() == "true"
        if write_restart and self.dg.slab is not None:
            raise ValueError("restart files hold the whole mesh's state: not written from the slabs of a shared mesh")
        every_x = int(self.parameters.get("flow_solver/output_restart_files_every_x_steps"))
        every_dt = float(self.parameters.get("flow_solver/output_restart_files_every_dt_time_intervals"))
        restart_index = int(self.parameters.get("flow_solver/restart_file_index")) + 1 \
            if self.restart_dt is not None else 1
        next_restart_time = self.ode_solver.current_time + every_dt
        if self.restart_dt is not None:
            dt = self.restart_dt
        elif error_adaptive:   # flow_solver.cpp:495-510
            dt = self.ode_solver.get_automatic_initial_step_size()
        else:
            dt = self.time_step()
        if not self.unsteady_data:
            self.unsteady_data.append((self.ode_solver.current_time, *self.dg.integrals()))
        if (not adaptive and not error_adaptive and not write_restart and record_every > 0
                and not self.parameters.use_relaxation_runge_kutta and self.dg.slab is None
                and self.time_pod is None
                and self.ode_solver.current_iteration % record_every == 0):
            # the whole steps of dt run on the device with the records reduced there (ph_run);
            # the count follows the loop below step by step, so the clock is the same
            t, n = self.ode_solver.current_time, 0
            while t < final_time and not (end_exact and t + dt > final_time):
                t += dt
                n += 1
            # records after iterations that are multiples of record_every, as the loop below
            self.unsteady_data.extend(self.ode_solver.step_in_time_with_records(dt, n, record_every))
        while self.ode_solver.current_time < final_time:
            step = dt
            if self.ode_solver.current_time + step > final_time and end_exact:
                step = final_time - self.ode_solver.current_time
            self.ode_solver.step_in_time(step)
            if adaptive or self.ode_solver.current_iteration % record_every == 0:
                q = self.dg.integrals()
                self.unsteady_data.append((self.ode_solver.current_time, *q))
                if adaptive:
                    dt = float(self.parameters.get("flow_solver/courant_friedrichs_lewy_number")) * \
                        self._grid_spacing() / q[3]
            if error_adaptive:   # flow_solver.cpp:603-607
                dt = self.ode_solver.get_automatic_error_adaptive_step_size(step)
            if self.time_pod is not None and self.ode_solver.current_iteration % self.snapshot_every == 0:
                self.time_pod.addSnapshot(self.dg)   # flow_solver.cpp:675-679, a device copy
            if write_restart:   # flow_solver.cpp:605-632: every dt time interval, or every x steps
                if every_dt > 0.0:
                    if self.ode_solver.current_time >= next_restart_time:
                        self.output_restart_files(restart_index, dt)
                        restart_index += 1
                        next_restart_time += every_dt
                elif self.ode_solver.current_iteration % every_x == 0:
                    self.output_restart_files(self.ode_solver.current_iteration // every_x, dt)
        if self.time_pod is not None:   # flow_solver.cpp:683-688
            from .pod import write_snapshot_matrix
            write_snapshot_matrix(f"solution_snapshots_iteration_{self.ode_solver.current_iteration}.txt",
                                  self.time_pod.getSnapshotMatrix())
        return 0
