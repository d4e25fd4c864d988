#!/usr/bin/env python
"""Benchmark of the explicit strong-form DG/FR residual + RK4 stage on the B200.

Workload (default): viscous Taylor-Green vortex, Re=1600, Pr=0.71, Mach 0.1, on the
periodic cube [0, 2 pi]^3 with 24^3 hex cells, p = 5 on GLL nodes (216 nodes/cell,
14,929,920 DOFs), Chandrashekar split-form volume flux, Roe face dissipation, BR2
viscous flux, classical RK4. Synthetic data: the TGV initial condition, interpolated
at the nodes.

A "step" is one RK4 time step (4 stages). The metric is DOF-updates per second per
stage = N_DOF x stages / time, aggregated over all GPUs (each GPU integrates its own
copy of the cube: replicas, weak scaling). With --shard slab the GPUs share one cube
instead, each owning a slab of cell layers and exchanging the partition faces with its
neighbours every stage (strong scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload tgv_viscous_24_p5|tgv_inviscid_8_p3|tgv_viscous_32_p3]
                  [--precision fp64|fp32] [--shard replicas|slab]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TWO_PI = 6.28318530717958623200

WORKLOADS = {
    # name: (poly_degree, cells per direction, pde, diss flux, description)
    "tgv_viscous_24_p5": (5, 24, "navier_stokes", "bassi_rebay_2",
                          "viscous TGV Re=1600, 24^3 cells, p=5 GLL, CH split + Roe, BR2, RK4"),
    "tgv_inviscid_8_p3": (3, 8, "euler", "symm_internal_penalty",
                          "inviscid TGV, 8^3 cells, p=3 GLL, CH split + Roe, RK4"),
    "tgv_viscous_32_p3": (3, 32, "navier_stokes", "bassi_rebay_2",
                          "viscous TGV Re=1600, 32^3 cells, p=3 GLL, CH split + Roe, BR2, RK4"),
    # reduced size of the default workload, for ncu captures (still larger than L2)
    "tgv_viscous_16_p5": (5, 16, "navier_stokes", "bassi_rebay_2",
                          "viscous TGV Re=1600, 16^3 cells, p=5 GLL, CH split + Roe, BR2, RK4"),
    # the default workload on Gauss-Legendre flux nodes (the reference's default flux_nodes_type):
    # dense interpolation, entropy projection and FR operators
    "tgv_viscous_gl_24_p5": (5, 24, "navier_stokes", "bassi_rebay_2",
                             "viscous TGV Re=1600, 24^3 cells, p=5 on GL flux nodes, CH split + Roe, BR2, RK4"),
}


def prm_for(workload: str) -> dict:
    p, n, pde, diss, _ = WORKLOADS[workload]
    return {
        "dimension": 3, "pde_type": pde, "use_weak_form": False,
        "flux_nodes_type": "GL" if "_gl_" in workload else "GLL",
        "use_split_form": True, "two_point_num_flux_type": "CH",
        "conv_num_flux": "two_point_flux_with_roe_dissipation", "diss_num_flux": diss,
        "flux_reconstruction": "cDG", "use_inverse_mass_on_the_fly": True,
        "all_boundaries_are_periodic": True, "do_renumber_dofs": False,
        "ODE solver/ode_solver_type": "runge_kutta", "ODE solver/runge_kutta_method": "rk4_ex",
        "euler/mach_infinity": 0.1, "navier_stokes/reynolds_number_inf": 1600.0,
        "navier_stokes/prandtl_number": 0.71,
        "flow_solver/flow_case_type": "taylor_green_vortex", "flow_solver/poly_degree": p,
        "flow_solver/final_time": 2.0, "flow_solver/courant_friedrichs_lewy_number": 0.1,
        # CFL x spacing / max wave speed (the reference's adaptive_time_step formula); the
        # constant formula CFL x spacing ignores the sound speed and is unstable at Mach 0.1
        "flow_solver/adaptive_time_step": True,
        "flow_solver/grid/grid_left_bound": 0.0, "flow_solver/grid/grid_right_bound": TWO_PI,
        "flow_solver/grid/number_of_grid_elements_per_dimension": n,
    }


def bytes_per_dof_stage(viscous: bool, p: int = 5) -> dict:
    """Algorithmic HBM bytes per DOF of the stage kernel, averaged over the 4 RK4 stages.

    Stage kernel (FP64 state), per DOF:
      stage 1:   U_in + acc_out + next                   = 24 B
      stage 2,3: U_in + u_n + acc_in + acc_out + next    = 40 B
      stage 4:   U_in + acc_in + u_{n+1}                 = 24 B      -> mean 32 B
    Viscous: the auxiliary kernel reads U_in (8 B) and writes the viscous terms per cell:
    the divergence (4 NP doubles) and the six face blocks (24 NF doubles); the stage kernel
    reads the divergence, its own face blocks and its neighbours' (48 NF doubles). Per DOF
    (5 NP DOFs per cell). Neighbour state traces are not counted: they are re-reads of data
    the neighbouring CTA streams, served from L2.
    """
    n1 = p + 1
    NP, NF = n1 ** 3, n1 ** 2
    stage = 32.0 + ((4 * NP + 48 * NF) * 8.0 / (5 * NP) if viscous else 0.0)
    aux = (8.0 + (4 * NP + 24 * NF) * 8.0 / (5 * NP)) if viscous else 0.0
    return {"stage": stage, "aux": aux}


def flops_per_dof_stage(p: int, viscous: bool) -> dict:
    """Algorithmic FP64 operations per DOF of one stage-kernel launch (Chandrashekar split form,
    EC + Roe faces, BR2 when viscous, classical RK4 epilogue), counted from the kernel source:
    add / mul = 1, fma = 2, division / square root / logarithm = 1 each. Each unordered pair of
    nodes on a line is counted once (1.5 (n1 - 1) pair fluxes per node; the skew operator's
    diagonal is zero, operators.cpp:1466-1476) and each face once (3 n1^2 face nodes per cell).
    The viscous flux, gradient and divergence belong to the auxiliary kernel, not to this one.
      pair flux (Chandrashekar means, momentum and energy fluxes) ........ 56
      its accumulation into both nodes (2 x 5 fma) ........................ 20
      node quantities (velocity, pressure, beta, two logarithms) .......... 22
      face node: EC flux 56 + Roe-Pike dissipation with Harten's fix 118 +
        the neighbour's node quantities 22 + lift 10 (+ BR2 average 20) .. 206 (226)
      epilogue: face terms, 1/h, RK4 running sum and next stage input .... 45 per node
    """
    n1 = p + 1
    pair = 56 + 20
    face_node = 206 + (20 if viscous else 0)
    per_node = 1.5 * (n1 - 1) * pair + 22 + 3.0 * n1 * n1 * face_node / n1 ** 3 + 45
    return {"per_dof": per_node / 5.0, "pair_flux": pair, "face_node": face_node,
            "rule": "add/mul 1, fma 2, div/sqrt/log 1; each node pair and each face once"}


def measured_fp64_mix(p: int, viscous: bool, precision: str):
    """Executed FP64 operations and FP64-pipe activity of the stage kernel from an ncu capture
    (profiles/fp64_mix.json), or None."""
    path = os.path.join(ROOT, "profiles", "fp64_mix.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(f"residual_kernel/{'navier_stokes' if viscous else 'euler'}/p{p}/{precision}")


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons during the timed region:
    through NVML every 5 ms (the device found by its PCI bus id), else nvidia-smi every 50 ms.
    Reads only."""

    def __init__(self, device_index: int):
        self.idx = device_index
        self.samples = []
        self.source = "nvidia-smi"
        self._stop = threading.Event()
        self._thr = None
        self._nvml = None
        try:
            import pynvml
            import torch
            pr = torch.cuda.get_device_properties(device_index)
            pynvml.nvmlInit()
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            self._handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self._max = float(pynvml.nvmlDeviceGetMaxClockInfo(self._handle, pynvml.NVML_CLOCK_SM))
            self._nvml = pynvml
            self.source = "nvml"
        except Exception:
            self._nvml = None

    def _run_nvml(self):
        n = self._nvml
        bits = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
        while not self._stop.is_set():
            try:
                sm = float(n.nvmlDeviceGetClockInfo(self._handle, n.NVML_CLOCK_SM))
                r = int(n.nvmlDeviceGetCurrentClocksEventReasons(self._handle))
                self.samples.append([str(sm), str(self._max), ""] +
                                    ["Active" if r & b else "Not Active" for b in bits])
            except Exception:
                pass
            self._stop.wait(0.005)

    def _run(self):
        if self._nvml is not None:
            return self._run_nvml()
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thr.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "", 1).isdigit()]
        smax = [float(s[1]) for s in self.samples if s[1].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and "Active" in s[3 + i]
                          and not s[3 + i].startswith("Not")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.samples), "source": self.source}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def gemm_peak(torch, dtype):
    """Measured FP64 (or FP32, TF32 off) denominator: a cuBLAS GEMM 8192^3 (2 N^3 flops), best of
    3, CUDA events. Run outside the timed region."""
    n = 8192
    tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    c = a @ b
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); torch.matmul(a, b, out=c); e1.record(); torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = tf32
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def ncu_traffic(p: int, viscous: bool, precision: str, ndofs: int):
    """DRAM bytes (read + write) of one stage-kernel launch, from the ncu capture summarised
    in profiles/dram_traffic.json (bytes per DOF of a smaller case of the same order and
    physics, scaled by the DOFs of this workload), or None when no capture matches."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    e = d.get(f"residual_kernel/{'navier_stokes' if viscous else 'euler'}/p{p}/{precision}")
    if not e:
        return None
    return {"bytes_per_launch": e["bytes_per_dof"] * ndofs, "bytes_per_dof": e["bytes_per_dof"],
            "alg_bytes_per_dof_same_stage": e["alg_bytes_per_dof_same_stage"], "captured": e["captured"]}


def cpu_baseline(workload: str, n_threads: int | None = None, boundaries=None):
    """Time the CPU oracle (a port of the reference path) on one RK stage of the workload."""
    from oracle.oracle import Oracle, lib as orc_lib
    from philip_b200.prm import Parameters
    prm = Parameters.from_dict(prm_for(workload))
    if n_threads:
        Oracle.set_threads(n_threads)
    cores = int(orc_lib().orc_max_threads())
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, boundaries=boundaries)
    U = orc.initial_condition("tgv")
    t0 = time.perf_counter()
    R = orc.residual(U)
    k = orc.inverse_mass(R)
    U += 1e-4 * k
    dt = time.perf_counter() - t0
    return {"value": orc.ndofs / dt, "unit": "DOF-updates/s/stage", "cores": cores, "kind": "port",
            "sample": f"one RK stage (assemble_residual + inverse mass + update) of the full {workload} "
                      f"mesh ({orc.ndofs} DOFs) on {cores} OpenMP threads, {dt:.2f} s"}


def reference_sample_workload(workload: str):
    """The reference arm's bounded sample: the same physics and order on the sub-cube
    with half the cells per direction (1/8 of the DOFs; the per-DOF cost of the CPU
    code does not depend on the mesh size)."""
    p, n, pde, diss, desc = WORKLOADS[workload]
    d = prm_for(workload)
    d["flow_solver/grid/number_of_grid_elements_per_dimension"] = max(2, n // 2)
    d["flow_solver/grid/grid_right_bound"] = TWO_PI * max(2, n // 2) / n
    return d, max(2, n // 2)


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle.oracle import Oracle, lib as orc_lib
    from philip_b200.prm import Parameters
    d, nsub = reference_sample_workload(args.workload)
    prm = Parameters.from_dict(d)
    cores = int(orc_lib().orc_max_threads())
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds, boundaries=args.bnd)
    U = orc.initial_condition("tgv")
    # one RK stage (residual + inverse mass + update) per step; one untimed stage warms up
    for _ in range(min(args.warmup, 1)):
        orc.inverse_mass(orc.residual(U))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        k = orc.inverse_mass(orc.residual(U))
        U += 1e-6 * k
    el = time.perf_counter() - t0
    value = orc.ndofs * args.steps / el
    _, n, _, _, desc = WORKLOADS[args.workload]
    sample = (f"{args.steps} RK stages, each on the {nsub}^3-cell sub-cube of the workload ({orc.ndofs} DOFs, "
              f"same order and physics), {cores} OpenMP threads; the reference itself cannot be built here "
              "(deal.II/MPI/Trilinos/p4est absent), so this is the from-source CPU port")
    line = {
        "impl": "reference", "metric": "TGV DOF-updates/s/stage", "value": value, "unit": "DOF-updates/s/stage",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Taylor-Green initial condition interpolated at the GLL nodes)",
        "config": {"workload": args.workload, "description": desc, "sample_ndofs": orc.ndofs,
                   "step": "one RK stage on the host", "boundaries": args.bnd or "periodic"},
        "cpu_baseline": {"value": value, "unit": "DOF-updates/s/stage", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "DOF-updates/s/stage", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# Batched and served forms (many independent Euler solves on one GPU)
# ------------------------------------------------------------------------------------------
MANY = {
    "vortex_batch_256": "256 isentropic-vortex solves on [0,10]^3, n^3 cells with n in {4,6,8,12,16}, p in 2..5, "
                        "beta ~ U[1,5], Mach ~ U[0.1,0.5], random direction, to t=1; all admitted at once",
    "served_stream": "Poisson arrivals (50/s) of Euler solves on sine-warped periodic cubes (x_i += 0.1 sin x sin y "
                     "sin z), TGV or isentropic vortex 50/50, Mach ~ U[0.1,0.4], n in 6..20, p in 2..5, to t=1",
}


def many_requests(kind: str, count: int, seed: int = 20261203):
    from philip_b200.serve import SolveRequest
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        if kind == "vortex_batch_256":
            reqs.append(SolveRequest("isentropic_vortex", n_cells=int(rng.choice([4, 6, 8, 12, 16])),
                                     poly_degree=int(rng.integers(2, 6)), mach=float(rng.uniform(0.1, 0.5)),
                                     beta=float(rng.uniform(1.0, 5.0)), direction=tuple(d), final_time=1.0))
        else:
            tgv = rng.random() < 0.5
            reqs.append(SolveRequest("taylor_green_vortex" if tgv else "isentropic_vortex",
                                     n_cells=int(rng.integers(6, 21)), poly_degree=int(rng.integers(2, 6)),
                                     left=0.0, right=TWO_PI if tgv else 10.0, warp=0.1,
                                     mach=float(rng.uniform(0.1, 0.4)), beta=float(rng.uniform(1.0, 5.0)),
                                     direction=tuple(d), final_time=1.0))
    return reqs


def one_at_a_time(reqs):
    """The same solves one after another through the single-solve context in FP64
    (ph_ctx_create, ph_set_state, ph_rk_step, ph_get_state per solve)."""
    import torch
    from philip_b200 import _lib
    from philip_b200.dg import DGStrong
    prepared = [(r, *r.prepare()) for r in reqs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    work = 0
    for r, U0, dt, nsteps in prepared:
        dg = DGStrong(r.parameters(), precision=_lib.PH_FP64, warp=r.warp)
        dg.solution = U0
        _lib.check(dg.L.ph_rk_step(dg.handle, dt, nsteps))
        dg.solution   # read back (synchronises)
        work += r.ndofs * 4 * nsteps
        del dg
    el = time.perf_counter() - t0
    return {"solves": len(reqs), "seconds": el, "solves_per_s": len(reqs) / el,
            "dof_updates_per_s_stage": work / el, "dtype": "f64", "path": "single-solve context per solve"}


def served_sample(count: int = 24, rate: float = 50.0, budget_gb: float = 32.0, chunk: int = 16):
    """A bounded sample of the served snapshot stream beside the default line: the first `count`
    seeded requests of the served_stream workload arriving at its Poisson rate, served by the
    library's native loop in the precision form, then the same solves one at a time in FP64.
    Returns solves/s, p50 / p99 latency and the ratio to one at a time."""
    from philip_b200 import _lib
    from philip_b200.serve import Server, autotune, poisson_arrivals, serve_native
    prec = _lib.PH_FP32_RESIDUAL
    reqs = many_requests("served_stream", count)
    arrivals = list(poisson_arrivals(rate, count, np.random.default_rng(7)))
    tuned = {}
    for r in reqs:   # tile shapes per (order, mesh kind) and the requests' payloads, before the clock
        key = (r.poly_degree, r.warp != 0.0)
        if key not in tuned:
            tuned[key] = autotune(r.poly_degree, prec, key[1])
        r.prepare()
    warm = Server(1 << 28, prec, chunk=chunk)
    serve_native(warm, [(0.0, many_requests("served_stream", 1, seed=1)[0])])
    warm.close()
    srv = Server(int(budget_gb * (1 << 30)), prec, chunk=chunk)
    stats = serve_native(srv, list(zip(arrivals, reqs)))
    srv.close()
    lat = sorted(c.latency for c in stats.completed)

    def pct(q):
        return lat[min(len(lat) - 1, max(0, int(np.ceil(q / 100.0 * len(lat))) - 1))]
    work = sum(c.request.ndofs * 4 * c.steps for c in stats.completed)
    base = one_at_a_time(reqs)
    served = {"solves_per_s": len(lat) / stats.makespan, "dof_updates_per_s_stage": work / stats.makespan,
              "makespan_s": stats.makespan, "latency_ms": {"p50": 1e3 * pct(50), "p99": 1e3 * pct(99)},
              "dtype": "f32-residual/f64-state", "server": "ph_server (native worker thread)"}
    return {"workload": "served_stream", "requests": count, "arrival_rate_per_s": rate,
            "description": "the first %d requests of the served_stream workload (%s)" % (count, MANY["served_stream"]),
            "served": served, "one_at_a_time": base,
            "speedup_vs_one_at_a_time": served["dof_updates_per_s_stage"] / base["dof_updates_per_s_stage"],
            "status_flags": int(np.bitwise_or.reduce([c.status for c in stats.completed]))}


def run_many(args, rank: int = 0, world: int = 1, local_rank: int = 0):
    """Batched (all admitted at t=0) or served (Poisson arrivals, continuous batching) form.
    With N GPUs every rank serves a cost-balanced share of the same requests (by solve; no
    exchange between ranks), so the total work is fixed (strong scaling)."""
    import torch
    from philip_b200 import _lib
    from philip_b200.serve import Batch, Server, SnapshotServer, autotune, poisson_arrivals, serve_native
    from philip_b200.shard import reduce_max, reduce_sum, request_cost, shard_by_cost
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    prec = _lib.PH_FP32_RESIDUAL if args.precision == "fp32" else _lib.PH_FP64
    count = args.requests or (256 if args.workload == "vortex_batch_256" else 64)
    all_reqs = many_requests(args.workload, count)
    rng0 = np.random.default_rng(7)
    all_arrivals = [0.0] * count if args.workload == "vortex_batch_256" else list(poisson_arrivals(args.rate, count, rng0))
    mine = shard_by_cost([request_cost(r) for r in all_reqs], world)[rank] if world > 1 else list(range(count))
    reqs = [all_reqs[i] for i in mine]
    arrivals = [all_arrivals[i] for i in mine]
    tuned = {}
    for r in reqs:   # tile shapes per (order, mesh kind), before the clock starts
        key = (r.poly_degree, r.warp != 0.0)
        if key not in tuned:
            tuned[key] = autotune(r.poly_degree, prec, key[1])
    for r in reqs:   # the requests' payload (initial state, time step), before the clock starts
        r.prepare()
    budget = int(args.budget_gb * (1 << 30))
    keep = args.workload == "vortex_batch_256"
    native = args.server == "native"
    # warm-up: one small solve through the same batch machinery
    warm_req = many_requests(args.workload, 1, seed=1)[0]
    if native:
        warm = Server(1 << 28, prec, chunk=args.chunk)
        serve_native(warm, [(0.0, warm_req)])
        warm.close()
    else:
        warm = Batch(1 << 28, prec)
        SnapshotServer(warm, chunk=args.chunk, precision=prec).run([(0.0, warm_req)])
        warm.close()
    batch = Server(budget, prec, chunk=args.chunk) if native else Batch(budget, prec)
    if dist is not None:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        if native:   # the loop in the library's worker thread; requests submitted as they arrive
            stats = serve_native(batch, list(zip(arrivals, reqs)), keep_states=keep)
        else:
            srv = SnapshotServer(batch, chunk=args.chunk, keep_states=keep, precision=prec)
            stats = srv.run(list(zip(arrivals, reqs)))
    launches = batch.stats()["launches"] if native else batch.launches
    batch.close()
    work = sum(c.request.ndofs * 4 * c.steps for c in stats.completed)
    if dist is not None:   # whole job: all ranks' solves and work over the slowest rank's makespan
        lat = [None] * world
        dist.all_gather_object(lat, [c.latency for c in stats.completed])
        makespan = reduce_max(stats.makespan, dist, "cuda")
        work = reduce_sum(work, dist, "cuda")
        launches = int(reduce_sum(launches, dist, "cuda"))
        latencies = sorted(x for part in lat for x in part)
        stats.makespan = makespan
        stats.completed_all = latencies
        if rank != 0:
            dist.barrier()
            dist.destroy_process_group()
            return 0
    else:
        latencies = sorted(c.latency for c in stats.completed)

    def pct(q):
        k = min(len(latencies) - 1, max(0, int(np.ceil(q / 100.0 * len(latencies))) - 1))
        return latencies[k]
    line = {
        "metric": "served solves/s" if args.workload == "served_stream" else "batched DOF-updates/s/stage",
        "unit": "solves/s" if args.workload == "served_stream" else "DOF-updates/s/stage",
        "value": len(latencies) / stats.makespan if args.workload == "served_stream" else work / stats.makespan,
        "n_gpus": world, "steps": None, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-residual/f64-state" if prec == _lib.PH_FP32_RESIDUAL else "f64",
        "data": "synthetic (seeded requests; exact initial conditions)",
        "config": {"workload": args.workload, "description": MANY[args.workload], "requests": count,
                   "budget_gb": args.budget_gb, "chunk_steps": args.chunk,
                   "server": "ph_server (native worker thread)" if native else "SnapshotServer (Python loop)",
                   "arrival_rate_per_s": None if args.workload == "vortex_batch_256" else args.rate,
                   "total_dofs": int(sum(r.ndofs for r in reqs)),
                   "tile_variants": {f"p{k[0]}{'c' if k[1] else 'a'}": v for k, v in tuned.items()}},
        "solves_per_s": len(latencies) / stats.makespan, "dof_updates_per_s_stage": work / stats.makespan,
        "makespan_s": stats.makespan,
        "latency_ms": {"p50": 1e3 * pct(50), "p99": 1e3 * pct(99), "max": 1e3 * latencies[-1]},
        "parallelism": f"solves sharded over {world} GPU(s)" if world > 1 else "one GPU",
        "max_resident": stats.max_in_flight, "gpu_launches": launches,
        "status_flags": int(np.bitwise_or.reduce([c.status for c in stats.completed])),
        "clocks": clk.summary(),
    }
    if args.workload == "vortex_batch_256":
        errs = []
        for c in stats.completed:
            ex = c.request.exact_state()
            errs.append(float(np.max(np.abs(c.state - ex)) / np.max(np.abs(ex))))
        line["vortex_rel_max_error"] = {"median": float(np.median(errs)), "max": float(np.max(errs))}
    if not args.no_cpu_baseline and world == 1:
        sample = reqs[: args.baseline_sample] if args.baseline_sample else reqs
        base = one_at_a_time(sample)
        base["sample"] = f"first {len(sample)} of the {count} requests, run back to back (no arrival gaps)"
        line["one_at_a_time"] = base
        line["speedup_vs_one_at_a_time"] = (line["dof_updates_per_s_stage"] / base["dof_updates_per_s_stage"])
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


PRECISION_CHECK = "tgv_precision_check_32_p3"


def run_precision_check(args, rank: int = 0, world: int = 1, local_rank: int = 0):
    """The precision form's error against the FP64 path on the viscous TGV at 32^3 cells, p=3
    over t in [0, t_final] (default 5): both forms take the same constant time step (the
    adaptive formula evaluated once at t=0) and record kinetic energy and enstrophy every 10
    steps on the device (ph_run). Reports the relative max errors of the kinetic-energy
    dissipation rate -dKE/dt (from each recorded state and its time derivative M^-1 R(u), on
    the device; also by central differences of the KE rows, which amplify the rows' rounding),
    of the vorticity-based dissipation rate 2 enstrophy / Re and of the KE itself, and the two
    forms' rates with the rows included. Independent replicas on every rank (no exchange)."""
    import torch
    from philip_b200 import _lib
    from philip_b200.dg import FlowSolver
    from philip_b200.prm import Parameters
    torch.cuda.set_device(local_rank)
    prm = Parameters.from_dict(prm_for("tgv_viscous_32_p3"))
    t_final = args.final_time
    record_every = 10
    out = {}
    dt = None
    for name, prec in (("fp64", _lib.PH_FP64), ("fp32", _lib.PH_FP32_RESIDUAL)):
        stream = torch.cuda.Stream()
        fs = FlowSolver(prm, precision=prec, stream=stream.cuda_stream)
        if dt is None:
            dt = fs.adaptive_time_step()
        nsteps = int(round(t_final / dt)) // record_every * record_every
        q0 = fs.dg.integrals()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        rows = fs.ode_solver.step_in_time_with_records(dt, nsteps, record_every)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        status = fs.dg.status()
        del fs
        # the same steps again, with -dKE/dt from each recorded state's time derivative
        # M^-1 R(u) on the device (ph_kinetic_energy_rate) after every record interval
        fs = FlowSolver(prm, precision=prec, stream=stream.cuda_stream)
        rates = [-fs.dg.kinetic_energy_rate()]
        for _ in range(nsteps // record_every):
            fs.ode_solver.step_in_time_with_records(dt, record_every, record_every)
            rates.append(-fs.dg.kinetic_energy_rate())
        out[name] = dict(t=np.array([0.0] + [r[0] for r in rows]), ke=np.array([q0[0]] + [r[1] for r in rows]),
                         eps_w=np.array([q0[2]] + [r[3] for r in rows]), ms=ms, rate=np.array(rates),
                         nsteps=nsteps, status=status, ndofs=fs.dg.n_dofs)
        del fs
        torch.cuda.empty_cache()
    a, b = out["fp64"], out["fp32"]

    def rel(x, y):
        return float(np.max(np.abs(x - y)) / np.max(np.abs(x)))

    dke_a = -np.gradient(a["ke"], a["t"])
    dke_b = -np.gradient(b["ke"], b["t"])

    def rate(o):
        return o["ndofs"] * 4 * o["nsteps"] / (o["ms"] * 1e-3)

    if rank == 0:
        line = {
            "metric": "KE-dissipation-rate rel error, precision form vs FP64 (viscous TGV 32^3 p3)",
            "value": rel(a["rate"], b["rate"]), "unit": "relative max error", "higher_is_better": False,
            "n_gpus": world, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-residual/f64-state vs f64", "data": "synthetic (Taylor-Green initial condition)",
            "config": {"workload": PRECISION_CHECK, "t_final": t_final, "dt": dt, "steps": a["nsteps"],
                       "record_every": record_every, "rows": len(a["t"]) - 1},
            "errors": {"ke_dissipation_rate_minus_dKE_dt": rel(a["rate"], b["rate"]),
                       "ke_dissipation_rate_by_central_differences_of_rows": rel(dke_a, dke_b),
                       "vorticity_dissipation_rate_2_enstrophy_over_Re": rel(a["eps_w"], b["eps_w"]),
                       "kinetic_energy": rel(a["ke"], b["ke"])},
            "rates_with_rows": {"fp64": rate(a), "fp32": rate(b), "ratio": rate(b) / rate(a),
                                "unit": "DOF-updates/s/stage"},
            "status_flags": [a["status"], b["status"]],
            "ke_final": [float(a["ke"][-1]), float(b["ke"][-1])],
        }
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv_viscous_24_p5",
                    choices=sorted(WORKLOADS) + sorted(MANY) + [PRECISION_CHECK])
    ap.add_argument("--final-time", type=float, default=5.0, help="precision check: end of the compared window")
    ap.add_argument("--requests", type=int, default=0, help="batched / served forms: number of solves")
    ap.add_argument("--rate", type=float, default=50.0, help="served form: Poisson arrival rate per second")
    ap.add_argument("--budget-gb", type=float, default=96.0, help="batched / served forms: HBM budget")
    ap.add_argument("--chunk", type=int, default=16, help="batched / served forms: RK steps per enqueue")
    ap.add_argument("--baseline-sample", type=int, default=0,
                    help="batched / served forms: solves in the one-at-a-time FP64 comparison (0 = all)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served-sample", action="store_true",
                    help="TGV workloads: skip the bounded served-stream sample reported beside the line")
    ap.add_argument("--server", default="native", choices=["native", "python"],
                    help="batched / served forms: the library's serving loop or the Python one")
    ap.add_argument("--shard", default="replicas", choices=["replicas", "slab"],
                    help="N > 1: a copy of the cube per GPU, or one cube in slabs of cell layers")
    ap.add_argument("--boundaries", default=None,
                    help="TGV workloads: six comma-separated boundary conditions for the sides x-,x+,y-,y+,z-,z+ "
                         "(names such as periodic, wall, riemann_farfield, or boundary_id values), e.g. "
                         "periodic,periodic,wall,wall,periodic,periodic (default: the periodic cube)")
    args = ap.parse_args()
    args.bnd = None
    if args.boundaries:
        args.bnd = [t if not t.strip().lstrip("-").isdigit() else int(t) for t in
                    (x.strip() for x in args.boundaries.split(","))]
        if len(args.bnd) != 6:
            ap.error("--boundaries takes six entries")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == PRECISION_CHECK:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the precision check compares this build's two "
                              "forms with each other; the reference has no precision form"}), flush=True)
            return 0
        return run_precision_check(args, rank, world, local_rank)
    if args.workload in MANY:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched and served forms have no reference "
                              "counterpart (the reference runs one FlowSolver per snapshot); their baseline is the "
                              "one-at-a-time line inside this arm's output"}), flush=True)
            return 0
        if args.precision == "fp64" and "--precision" not in sys.argv:
            args.precision = "fp32"   # the batched and served forms run the precision form by default
        return run_many(args, rank, world, local_rank)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from philip_b200 import _lib
    from philip_b200.dg import FlowSolver
    from philip_b200.prm import Parameters
    from philip_b200.shard import reduce_max

    if args.warmup < 3:
        args.warmup = 3
    prm = Parameters.from_dict(prm_for(args.workload))
    prec = _lib.PH_FP32_RESIDUAL if args.precision == "fp32" else _lib.PH_FP64
    # the context runs on its own stream (multi-step calls then replay a captured RK step);
    # every CUDA event below is recorded on that stream
    stream = torch.cuda.Stream()
    slab = args.shard == "slab"
    if slab:   # this rank's layers of the one cube, the partition faces over NCCL (one GPU: to itself)
        from philip_b200.slab import DistributedHalo, LoopbackHalo, slab_bounds
        fs = FlowSolver(prm, precision=prec, stream=stream.cuda_stream,
                        slab=slab_bounds(prm.n_cells, world, rank),
                        halo=DistributedHalo() if world > 1 else LoopbackHalo(), dist=dist)
    else:
        fs = FlowSolver(prm, precision=prec, stream=stream.cuda_stream, boundaries=args.bnd)
    dg = fs.dg
    # DOFs that one timed step updates over the whole job
    job_dofs = prm.n_cells ** 3 * 5 * dg.n_shape if slab else world * dg.n_dofs
    L, h = dg.L, dg.handle
    dt = fs.adaptive_time_step()
    p, n, pde, _, desc = WORKLOADS[args.workload]
    viscous = pde == "navier_stokes"
    stages = 4

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- warm-up. Timing mode 2: the captured RK step that ph_rk_step replays carries an
    # event-record node around each kernel, and every replay records its own events, so the
    # stage and auxiliary kernel durations below come from the timed steps themselves
    # (slab contexts launch directly: mode 2 times nothing there, mode 1 is used after)
    timing_mode = 1 if slab else 2
    if not slab:
        _lib.check(L.ph_set_timing(h, 2))
    _lib.check(L.ph_rk_step(h, dt, args.warmup))
    torch.cuda.synchronize()

    # ---- device-timed region (inputs resident in HBM; the working set is larger than L2)
    _lib.check(L.ph_set_timing(h, 0 if slab else 2))   # resets the sums; the captured step stays
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(); torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ev0.record(stream)
        _lib.check(L.ph_rk_step(h, dt, args.steps))
        ev1.record(stream)
        # wait inside the library (ctypes releases the interpreter lock there, so the clock
        # sampler thread keeps sampling while the GPU runs), then on the device as a whole
        _lib.check(L.ph_sync(h))
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    tm = np.zeros(7)
    _lib.check(L.ph_get_timing(h, tm.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    launches = int(tm[6])
    if not slab:   # mean duration per launch over the timed steps
        # per stage: with boundary faces each stage launches the periodic kernel on the interior
        # tiles and the boundary-face kernel on the others
        per = 2 if args.bnd else 1
        stage_ms = per * tm[0] / max(tm[1], 1)
        aux_ms = per * tm[2] / max(tm[3], 1)
    _lib.check(L.ph_set_timing(h, 0))
    ms = reduce_max(ms, dist, "cuda")
    ms_per_step = ms / args.steps
    value = job_dofs * stages * args.steps / (ms * 1e-3)

    # ---- the same steps through the device time loop with the kinetic energy / enstrophy
    # rows every 10 steps (ph_run: the integrals reduced on the device, one copy at the end)
    record_every = 10
    rows = np.zeros((max(args.steps // record_every, 2), 4))
    if not slab:   # slab contexts step through ph_rk_step (the exchange callback runs on the host)
        # warm-up: captures the graph of one record interval
        _lib.check(L.ph_run(h, dt, 2 * record_every, record_every,
                            rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        barrier(); torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        _lib.check(L.ph_run(h, dt, args.steps, record_every, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        r1.record(stream); torch.cuda.synchronize()
        ms_rec = reduce_max(r0.elapsed_time(r1), dist, "cuda")
        value_rec = job_dofs * stages * args.steps / (ms_rec * 1e-3)

    if slab:   # per-launch events after the timed region (a slab splits each stage into launches)
        _lib.check(L.ph_set_timing(h, 1))
        _lib.check(L.ph_rk_step(h, dt, 2))
        _lib.check(L.ph_get_timing(h, tm.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        _lib.check(L.ph_set_timing(h, 0))
        stage_ms = tm[0] / (2 * stages)
        aux_ms = tm[2] / (2 * stages)

    # ---- end to end through the C-ABI with host buffers (pinned), every step:
    # H2D of the state, one RK4 step, D2H of the state
    U_host = torch.empty(dg.n_dofs, dtype=torch.float64, pin_memory=True)
    _lib.check(L.ph_get_state(h, U_host.data_ptr(), _lib.PH_HOST))
    barrier(); torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        _lib.check(L.ph_set_state(h, U_host.data_ptr(), _lib.PH_HOST))
        _lib.check(L.ph_rk_step(h, dt, 1))
        _lib.check(L.ph_get_state(h, U_host.data_ptr(), _lib.PH_HOST))
    e1.record(stream); torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ms_e2e = reduce_max(ms_e2e, dist, "cuda")
    e2e = job_dofs * stages * args.steps / (ms_e2e * 1e-3)
    status = dg.status()

    if rank == 0:
        peak, peak_src = measured_peaks()
        bpd = bytes_per_dof_stage(viscous, p)
        if args.precision == "fp32":
            pass   # the state stays FP64, so the stage bytes are the same (+8 B/DOF Kahan term at the last stage)
        bytes_launch = bpd["stage"] * dg.n_dofs
        achieved_gbs = bytes_launch / (stage_ms * 1e-3) / 1e9
        traffic = ncu_traffic(p, viscous, args.precision, dg.n_dofs)
        flops = flops_per_dof_stage(p, viscous)
        alg_tflops = flops["per_dof"] * dg.n_dofs / (stage_ms * 1e-3) / 1e12
        fp32 = args.precision == "fp32"
        gemm_tflops = gemm_peak(torch, torch.float32 if fp32 else torch.float64)
        mix = measured_fp64_mix(p, viscous, args.precision)
        if "_gl_" in args.workload:   # the byte and flop models above are the collocated kernel's
            flops = dict(flops, applies_to="collocated (GLL) stage kernel; this workload runs the GL kernels")
        line = {
            "metric": "TGV DOF-updates/s/stage", "value": value, "unit": "DOF-updates/s/stage",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong" if slab else "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-residual/f64-state",
            "data": "synthetic (Taylor-Green initial condition interpolated at the GLL nodes)",
            "config": {"workload": args.workload, "description": desc, "ndofs": n ** 3 * 5 * dg.n_shape,
                       "cells": n ** 3, "poly_degree": p, "stages_per_step": stages, "dt": dt,
                       "l2": "inputs larger than L2 (state 120 MB/vector, working set > 600 MB)"
                       if args.workload != "tgv_inviscid_8_p3" else "L2-resident (6.6 MB/vector)",
                       "parallelism": f"slabs x{world}" if slab else f"replicas x{world}",
                       "boundaries": args.bnd or "periodic",
                       "status_flags": status},
            "e2e": {"value": e2e, "unit": "DOF-updates/s/stage",
                    "h2d_bytes_per_step": 8 * dg.n_dofs, "d2h_bytes_per_step": 8 * dg.n_dofs,
                    "path": "ph_set_state(host pinned) + ph_rk_step + ph_get_state(host pinned) per step"},
            "gpu_launches": launches,
            "with_integrals": {"record_every": record_every, "value": value_rec, "ms_per_step": ms_rec / args.steps,
                               "rows": int(args.steps // record_every),
                               "path": "ph_run: the same steps with kinetic energy, enstrophy, dissipation rate "
                                       "and wave speed reduced on the device every 10 steps"}
            if not slab else {"skipped": "slab contexts step through ph_rk_step"},
            # the binding roof of the stage kernel is its floating-point pipe (arithmetic intensity
            # above the HBM ridge); the HBM figures are kept beside it
            "roofline": {"bound": "fp32" if fp32 else "fp64", "achieved": alg_tflops, "peak": gemm_tflops,
                         "unit": "TFLOP/s", "frac": alg_tflops / gemm_tflops,
                         "traffic": traffic["bytes_per_launch"] if traffic else None,   # DRAM bytes per launch
                         "traffic_detail": traffic,
                         "kernel": "residual_kernel (stage: residual + mass inverse + RK update)",
                         "kernel_ms": stage_ms, "aux_kernel_ms": aux_ms,
                         "kernel_ms_source": "mean over the timed steps: CUDA events recorded by graph nodes "
                                             "around each kernel of every replayed RK step (ph_set_timing mode 2)"
                                             if not slab else "per-launch CUDA events after the timed steps",
                         "alg_flops_per_dof": flops,
                         "peak_source": ("measured here: cuBLAS " + ("SGEMM (TF32 off)" if fp32 else "DGEMM")
                                         + " 8192^3, best of 3; MEASURED_PEAKS.json holds no FP64/FP32 figure"),
                         "executed": mix,
                         "hbm": {"achieved": achieved_gbs, "peak": peak, "unit": "GB/s", "frac": achieved_gbs / peak,
                                 "alg_bytes_per_dof": bpd, "peak_source": peak_src}},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_served_sample and not slab:
            try:   # a bounded sample of the served form beside the headline (not part of `value`)
                line["served_sample"] = served_sample()
            except Exception as e:
                line["served_sample"] = {"error": str(e)}
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(args.workload, boundaries=args.bnd)
            except Exception as e:  # the checker must not hide a failure of the GPU arm
                line["cpu_baseline"] = {"value": None, "error": str(e)}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
