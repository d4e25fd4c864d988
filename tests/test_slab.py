"""One mesh over several ranks: slabs of cell layers with a halo exchange of the partition
faces (the reference's ghost-value refresh before each residual, DGBase::assemble_residual,
src/dg/dg_base.cpp:2742, and of the auxiliary solution, src/dg/strong_dg.cpp:648).

CPU (gloo, 2 and 3 ranks): the slab plan names, for every owned cell's face, either the owned
neighbour or a ghost slot, and the exchange through philip_b200.slab.DistributedHalo fills each
ghost slot with the data of the cell that the periodic cube puts there.
GPU (one device): the slabs of a mesh run as contexts in threads of one process, exchanging
through device copies between host barriers (no kernel waits on another context); their
residuals and RK steps are bitwise those of one context over the whole mesh.
"""
import ctypes
import os
import socket
import threading

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from philip_b200 import _lib
from philip_b200.slab import DistributedHalo, global_integrals, slab_bounds


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plan(n, z0, nz):
    L = _lib.load()
    nown = nz * n * n
    ijk = np.zeros((nown, 3), np.int32)
    nbr = np.zeros((nown, 6), np.int32)
    _lib.check(L.ph_slab_connectivity(n, z0, nz, ijk.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                      nbr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
    return ijk, nbr


def _gid(n, i, j, k):
    return (k * n + j) * n + i


def test_slab_bounds_cover_the_layers():
    for n in (1, 4, 7, 24):
        for world in range(1, n + 1):
            spans = [slab_bounds(n, world, r) for r in range(world)]
            layers = [z for z0, nz in spans for z in range(z0, z0 + nz)]
            assert layers == list(range(n))
            assert max(s[1] for s in spans) - min(s[1] for s in spans) <= 1
    with pytest.raises(ValueError):
        slab_bounds(3, 4, 0)


@pytest.mark.parametrize("n,z0,nz", [(4, 0, 2), (4, 3, 1), (3, 1, 2), (5, 2, 5), (2, 0, 1)])
def test_slab_plan_names_the_periodic_neighbours(n, z0, nz):
    ijk, nbr = _plan(n, z0, nz)
    nown = nz * n * n
    assert sorted(ijk[:, 2].tolist()) == sorted([(z0 + k) % n for k in range(nz) for _ in range(n * n)])
    for c in range(nown):
        for f in range(6):
            t = list(ijk[c]); d = f // 2
            t[d] = (t[d] + (1 if f & 1 else -1)) % n
            g = int(nbr[c, f])
            if g < nown:
                assert list(ijk[g]) == t
            else:                               # ghost slot: only z faces of the first / last layer
                assert d == 2
                side, ii = divmod(g - nown, n * n)
                layer = (z0 - 1) % n if side == 0 else (z0 + nz) % n
                assert (ii % n, ii // n, layer) == tuple(t)


def _exchange_worker(rank, world, port, n, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z0, nz = slab_bounds(n, world, rank)
        ijk, nbr = _plan(n, z0, nz)
        nown, L2, m = nz * n * n, n * n, 3
        halo = DistributedHalo(device="cpu")
        ok = True
        for what in (_lib.PH_HALO_STATE, _lib.PH_HALO_VISCOUS):
            # the packed layout: one record of m values per cell of the layer, (y, x) order
            bufs = [np.zeros((L2, m)) for _ in range(4)]
            for ii in range(L2):
                i, j = ii % n, ii // n
                bufs[0][ii] = _gid(n, i, j, z0) + 0.25 * what
                bufs[1][ii] = _gid(n, i, j, (z0 + nz - 1) % n) + 0.25 * what
            ptr = [b.ctypes.data for b in bufs]
            halo.begin(what, *ptr, bufs[0].nbytes)
            halo.end()
            recv_lo, recv_hi = bufs[2], bufs[3]
            for c in range(nown):
                for f in (4, 5):
                    g = int(nbr[c, f])
                    if g < nown:
                        continue
                    side, ii = divmod(g - nown, L2)
                    t = list(ijk[c]); t[2] = (t[2] + (1 if f & 1 else -1)) % n
                    want = _gid(n, *t) + 0.25 * what
                    ok &= bool(np.all((recv_lo if side == 0 else recv_hi)[ii] == want))
        # the volume averages of the slabs add up, the wave speed is the largest
        tot = global_integrals([1.0 + rank, 2.0, 0.5, 3.0 + rank], dist)
        # the relaxation RK sum through the library's callback type: in place, on every rank
        vals = (ctypes.c_double * 3)(1.0 + rank, -0.5 * rank, 0.25)
        rc = halo.sum_callback(None, vals, 3)
        out[rank] = (ok, tot, rc, list(vals))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 4), (3, 4), (2, 2)])
def test_halo_exchange_fills_the_ghost_layers(world, n):
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_exchange_worker, args=(world, _free_port(), n, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ok, tot, rc, sums = res[r]
        assert ok
        assert tot == [sum(1.0 + q for q in range(world)), 2.0 * world, 0.5 * world, 3.0 + world - 1]
        assert rc == 0 and sums == [sum(1.0 + q for q in range(world)), sum(-0.5 * q for q in range(world)),
                                    0.25 * world]


def test_loopback_halo_feeds_a_slab_its_own_layers():
    from philip_b200.slab import LoopbackHalo
    bufs = [np.arange(6.0) + 10 * k for k in range(4)]
    halo = LoopbackHalo(device="cpu")
    ptr = [b.ctypes.data for b in bufs]
    assert halo.callback(None, _lib.PH_HALO_STATE, _lib.PH_HALO_BEGIN, *ptr, bufs[0].nbytes, None) == 0
    assert halo.callback(None, _lib.PH_HALO_STATE, _lib.PH_HALO_END, *ptr, bufs[0].nbytes, None) == 0
    assert np.array_equal(bufs[2], np.arange(6.0) + 10) and np.array_equal(bufs[3], np.arange(6.0))


def test_slab_refusals_without_a_gpu():
    from helpers import prm_dict
    from philip_b200.prm import Parameters
    L = _lib.load()
    prm = Parameters.from_dict(prm_dict(poly_degree=2, n_cells=4))
    p = prm.to_ph_params()
    h = ctypes.c_void_p()

    def create(z0, nz, warp=0.0, edit=None):
        q = prm.to_ph_params()
        if edit:
            edit(q)
        m = _lib.PhMeshDesc(4, 0, 0.0, 6.283185307179586, warp, 2)
        return L.ph_ctx_create_slab(ctypes.byref(m), ctypes.byref(q), z0, nz, None, ctypes.byref(h))

    assert create(4, 1) == _lib.PH_ERR_INVALID
    assert create(0, 0) == _lib.PH_ERR_INVALID
    assert create(1, 5) == _lib.PH_ERR_INVALID
    assert create(0, 2, edit=lambda q: setattr(q, "overintegration", 3)) == _lib.PH_ERR_UNSUPPORTED
    del p


# ------------------------------------------------------------------------------- GPU

class ThreadHalo:
    """The exchange of `world` slab contexts of one process, each stepped by its own thread:
    every rank synchronises its stream, publishes its send buffers, and after a barrier copies
    its neighbours' into its receive buffers on its stream; a second barrier keeps the send
    buffers until every rank has copied. Host barriers only: no kernel waits on another."""

    def __init__(self, world, state):
        self.world = world
        self.state = state              # shared: barrier and published pointers

    def for_rank(self, rank):
        h = ThreadHalo(self.world, self.state)
        h.rank = rank
        h.callback = _lib.HALO_FN(h._call)
        h.sum_callback = _lib.RANK_SUM_FN(h._sum)
        return h

    @staticmethod
    def shared(world):
        return {"barrier": threading.Barrier(world, timeout=120), "send": {}, "sums": {}}

    def _sum(self, user, values, count):
        """ph_rank_sum_fn: every rank publishes its values and, after a barrier, sums all ranks'
        in rank order (the same result on every rank); a second barrier keeps them published
        until all have read."""
        try:
            st = self.state
            st["sums"][self.rank] = [values[i] for i in range(count)]
            st["barrier"].wait()
            for i in range(count):
                acc = 0.0
                for r in range(self.world):
                    acc += st["sums"][r][i]
                values[i] = acc
            st["barrier"].wait()
            return 0
        except Exception:
            import traceback
            traceback.print_exc()
            try:
                self.state["barrier"].abort()
            except Exception:
                pass
            return 1

    def _call(self, user, what, phase, send_lo, send_hi, recv_lo, recv_hi, nbytes, stream):
        import torch
        from philip_b200.slab import _as_tensor
        try:
            if phase == _lib.PH_HALO_END:
                return 0
            s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
            s.synchronize()
            st = self.state
            st["send"][self.rank] = (send_lo, send_hi)
            st["barrier"].wait()
            lo, hi = (self.rank - 1) % self.world, (self.rank + 1) % self.world
            with torch.cuda.stream(s):
                _as_tensor(recv_lo, nbytes, "cuda").copy_(_as_tensor(st["send"][lo][1], nbytes, "cuda"))
                _as_tensor(recv_hi, nbytes, "cuda").copy_(_as_tensor(st["send"][hi][0], nbytes, "cuda"))
            s.synchronize()
            st["barrier"].wait()
            return 0
        except Exception:
            import traceback
            traceback.print_exc()
            try:
                self.state["barrier"].abort()
            except Exception:
                pass
            return 1


def _slabs(prm, world, precision=_lib.PH_FP64, warp=0.0, boundaries=None):
    import torch
    from philip_b200.dg import DGStrong
    shared = ThreadHalo.shared(world)
    base = ThreadHalo(world, shared)
    out = []
    for r in range(world):
        s = torch.cuda.Stream()
        halo = base.for_rank(r)
        dg = DGStrong(prm, precision=precision, stream=s.cuda_stream,
                      slab=slab_bounds(prm.n_cells, world, r), halo=halo, warp=warp, boundaries=boundaries)
        out.append((dg, s))
    return out


def _in_threads(fns):
    errs = [None] * len(fns)
    res = [None] * len(fns)

    def run(k):
        try:
            res[k] = fns[k]()
        except Exception as e:          # noqa: BLE001
            errs[k] = e

    th = [threading.Thread(target=run, args=(k,)) for k in range(len(fns))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for e in errs:
        if e is not None:
            raise e
    return res


def _slice_map(whole, part):
    """Cell indices of `part`'s owned cells in `whole`'s order."""
    pos = {tuple(r): i for i, r in enumerate(whole.cell_ijk())}
    return np.array([pos[tuple(r)] for r in part.cell_ijk()])


def _gather(whole, parts, vecs):
    nd = 5 * whole.n_shape
    U = np.empty(whole.n_dofs)
    for dg, v in zip(parts, vecs):
        idx = _slice_map(whole, dg)
        U.reshape(-1, nd)[idx] = v.reshape(-1, nd)
    return U


def _scatter(whole, parts, U):
    nd = 5 * whole.n_shape
    return [U.reshape(-1, nd)[_slice_map(whole, dg)].reshape(-1).copy() for dg in parts]


SLAB_CASES = [
    ("ns_br2_p3_two_slabs", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 2),
    ("ns_sipg_p2_three_slabs", dict(poly_degree=2, n_cells=4, pde="navier_stokes"), 3),
    ("euler_ch_p5_two_slabs", dict(poly_degree=5, n_cells=3), 2),
    ("ns_p4_one_layer_each", dict(poly_degree=4, n_cells=3, pde="navier_stokes", diss="bassi_rebay_2"), 3),
    ("euler_p1_interior_overlap", dict(poly_degree=1, n_cells=8), 2),
    ("ns_br2_p2_interior_overlap", dict(poly_degree=2, n_cells=6, pde="navier_stokes", diss="bassi_rebay_2"), 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,world", SLAB_CASES, ids=[c[0] for c in SLAB_CASES])
def test_slab_residual_is_the_whole_mesh_residual(name, kw, world):
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong
    from philip_b200.prm import Parameters
    from helpers import perturbed_tgv, prm_dict
    prm = Parameters.from_dict(prm_dict(**kw))
    whole = DGStrong(prm)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    U = perturbed_tgv(orc, seed=len(name))
    R_whole = whole.residual_of(U)
    parts = _slabs(prm, world)
    Us = _scatter(whole, [p for p, _ in parts], U)
    Rs = _in_threads([lambda k=k: parts[k][0].residual_of(Us[k]) for k in range(world)])
    R = _gather(whole, [p for p, _ in parts], Rs)
    print(f"{name}: max |R_slabs - R_whole| = {np.max(np.abs(R - R_whole)):.3e}")
    assert np.array_equal(R, R_whole)


STEP_CASES = [
    ("ns_br2_rk4_p3", dict(poly_degree=3, n_cells=6, pde="navier_stokes", diss="bassi_rebay_2"), 2, _lib.PH_FP64),
    ("euler_ssprk3_p2", dict(poly_degree=2, n_cells=4, rk="ssprk3_ex"), 3, _lib.PH_FP64),
    ("euler_forward_euler_p2", dict(poly_degree=2, n_cells=3, rk="euler_ex"), 2, _lib.PH_FP64),
    ("ns_lsrk_p3", dict(poly_degree=3, n_cells=4, pde="navier_stokes", rk="RK3_2_5F_3SStarPlus"), 2, _lib.PH_FP64),
    ("ns_br2_precision_form_p5", dict(poly_degree=5, n_cells=6, pde="navier_stokes", diss="bassi_rebay_2"), 2,
     _lib.PH_FP32_RESIDUAL),
    ("euler_precision_form_p3_one_layer_each", dict(poly_degree=3, n_cells=3), 3, _lib.PH_FP32_RESIDUAL),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,world,precision", STEP_CASES, ids=[c[0] for c in STEP_CASES])
def test_slab_steps_are_the_whole_mesh_steps(name, kw, world, precision):
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.prm import Parameters
    from helpers import TWO_PI, prm_dict
    prm = Parameters.from_dict(prm_dict(**kw))
    whole = DGStrong(prm, precision=precision)
    U0 = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds).initial_condition("tgv")
    whole.solution = U0
    dt = 0.1 * TWO_PI / prm.n_cells / (prm.poly_degree + 1) / 11.0
    ode = RungeKuttaODESolver(whole)
    ode.step_in_time(dt, nsteps=3)
    parts = _slabs(prm, world, precision)
    dgs = [p for p, _ in parts]
    for dg, u in zip(dgs, _scatter(whole, dgs, U0)):
        dg.solution = u

    def steps(k):
        o = RungeKuttaODESolver(dgs[k])
        o.step_in_time(dt, nsteps=3)
        parts[k][1].synchronize()
        return dgs[k].solution, dgs[k].integrals(), (o.error_norm() if "lsrk" in name else 0.0)

    res = _in_threads([lambda k=k: steps(k) for k in range(world)])
    U = _gather(whole, dgs, [r[0] for r in res])
    print(f"{name}: max |U_slabs - U_whole| = {np.max(np.abs(U - whole.solution)):.3e}")
    assert np.array_equal(U, whole.solution)
    assert all(dg.status() == 0 for dg in dgs)
    # the slabs' shares of the volume averages add up to the whole mesh's
    q = np.array([r[1] for r in res])
    qw = whole.integrals()
    assert np.allclose(q[:, :3].sum(axis=0), qw[:3], rtol=1e-13, atol=0.0)
    assert q[:, 3].max() == qw[3]
    if "lsrk" in name:   # the error norm: the RMS over the slabs' DOFs
        w = np.sqrt(sum(r[2] ** 2 * dg.n_dofs for r, dg in zip(res, dgs)) / whole.n_dofs)
        assert abs(w - ode.error_norm()) <= 1e-13 * ode.error_norm()


@pytest.mark.gpu
def test_slab_exchange_failures_are_reported():
    from philip_b200.dg import DGStrong
    from philip_b200.prm import Parameters
    from helpers import prm_dict
    prm = Parameters.from_dict(prm_dict(poly_degree=2, n_cells=4))
    lonely = DGStrong(prm, slab=(0, 2))
    U = np.zeros(lonely.n_dofs) + 1.0
    with pytest.raises(_lib.PhError, match="ph_set_halo_exchange"):
        lonely.residual_of(U)

    class Failing:
        def __init__(self):
            self.callback = _lib.HALO_FN(lambda *a: 7)

    dg = DGStrong(prm, slab=(0, 2), halo=Failing())
    with pytest.raises(_lib.PhError, match="returned 7"):
        dg.residual_of(U)



@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"),
                                dict(poly_degree=5, n_cells=3)], ids=["ns_br2_p3", "euler_p5"])
def test_one_slab_with_its_own_ghosts_is_the_whole_mesh(kw):
    """The whole mesh as one slab exchanges with itself (LoopbackHalo, stream-ordered device
    copies): residual and RK4 steps bitwise the whole-mesh context's."""
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.prm import Parameters
    from philip_b200.slab import LoopbackHalo
    from helpers import prm_dict
    prm = Parameters.from_dict(prm_dict(**kw))
    whole = DGStrong(prm)
    one = DGStrong(prm, slab=(0, prm.n_cells), halo=LoopbackHalo())
    U0 = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds).initial_condition("tgv")
    one.solution = _scatter(whole, [one], U0)[0]
    assert np.array_equal(_gather(whole, [one], [one.residual_of(one.solution)]), whole.residual_of(U0))
    whole.solution = U0
    RungeKuttaODESolver(whole).step_in_time(1e-3, nsteps=2)
    RungeKuttaODESolver(one).step_in_time(1e-3, nsteps=2)
    assert np.array_equal(_gather(whole, [one], [one.solution]), whole.solution)


CURV_CASES = [
    ("euler_ch_p3_two_slabs", dict(poly_degree=3, n_cells=4), 2, _lib.PH_FP64),
    ("euler_ir_p2_three_slabs", dict(poly_degree=2, n_cells=4, two_point="IR", conv="two_point_flux"), 3,
     _lib.PH_FP64),
    ("euler_ch_p4_precision_form", dict(poly_degree=4, n_cells=4), 2, _lib.PH_FP32_RESIDUAL),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,world,precision", CURV_CASES, ids=[c[0] for c in CURV_CASES])
def test_curvilinear_slabs_are_the_whole_curvilinear_mesh(name, kw, world, precision):
    """Slabs of the sine-warped cube (warp 0.1): each slab builds the metric terms of its own
    cells, and its faces use the metric of their own side, so the residual, three RK4 steps and
    the integrals are bitwise (the sums to rounding) the whole curvilinear mesh's."""
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.prm import Parameters
    from helpers import TWO_PI, perturbed_tgv, prm_dict
    warp = 0.1
    prm = Parameters.from_dict(prm_dict(**kw))
    whole = DGStrong(prm, precision=precision, warp=warp)
    U0 = perturbed_tgv(Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds), seed=len(name))
    parts = _slabs(prm, world, precision, warp=warp)
    dgs = [p for p, _ in parts]
    Us = _scatter(whole, dgs, U0)
    Rs = _in_threads([lambda k=k: dgs[k].residual_of(Us[k]) for k in range(world)])
    R = _gather(whole, dgs, Rs)
    print(f"{name}: max |R_slabs - R_whole| = {np.max(np.abs(R - whole.residual_of(U0))):.3e}")
    assert np.array_equal(R, whole.residual_of(U0))
    dt = 0.1 * TWO_PI / prm.n_cells / (prm.poly_degree + 1) / 11.0
    whole.solution = U0
    RungeKuttaODESolver(whole).step_in_time(dt, nsteps=3)
    for dg, u in zip(dgs, Us):
        dg.solution = u

    def steps(k):
        RungeKuttaODESolver(dgs[k]).step_in_time(dt, nsteps=3)
        parts[k][1].synchronize()
        return dgs[k].solution, dgs[k].integrals()

    res = _in_threads([lambda k=k: steps(k) for k in range(world)])
    U = _gather(whole, dgs, [r[0] for r in res])
    print(f"{name}: max |U_slabs - U_whole| = {np.max(np.abs(U - whole.solution)):.3e}")
    assert np.array_equal(U, whole.solution)
    q = np.array([r[1] for r in res])
    qw = whole.integrals()
    assert np.allclose(q[:, :3].sum(axis=0), qw[:3], rtol=1e-13, atol=0.0)
    assert q[:, 3].max() == qw[3]


RRK_CASES = [
    ("entropy_conservative_p3_two_slabs", dict(poly_degree=3, n_cells=4, two_point="CH", conv="two_point_flux"), 2),
    ("roe_dissipation_p2_three_slabs", dict(poly_degree=2, n_cells=4), 3),
    ("gl_entropy_conservative_p3_two_slabs", dict(poly_degree=3, n_cells=4, two_point="CH", conv="two_point_flux",
                                                  nodes="GL"), 2),
    ("gl_ns_ra_sipg_p2_two_slabs", dict(poly_degree=2, n_cells=4, pde="navier_stokes", fr="cPlus", two_point="Ra",
                                        conv="two_point_flux", rk="ssprk3_ex", nodes="GL"), 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,world", RRK_CASES, ids=[c[0] for c in RRK_CASES])
def test_relaxation_rk_on_slabs(name, kw, world):
    """Relaxation RK on slabs: the entropy integrals of every root iterate and the stage
    estimates are summed over the ranks (ph_set_rank_sum), so every slab takes the same
    relaxation parameter as the whole mesh up to the summation order of those integrals (the
    bounds of the GPU-vs-oracle relaxation test: 1e-5 on gamma, 5e-9 on the state), on GL flux
    nodes too; with the entropy-conservative Euler scheme the slabs' relaxed steps conserve the
    mesh's numerical entropy to rounding, and dissipative schemes lose entropy. A slab without the
    sum is refused at its first step."""
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.prm import Parameters
    from philip_b200.slab import LoopbackHalo
    from helpers import prm_dict
    kw = dict(kw)
    nodes = kw.pop("nodes", "GLL")
    d = prm_dict(**kw)
    d["flux_nodes_type"] = nodes
    d["ODE solver/rrk root solver/use_relaxation_runge_kutta"] = "true"
    prm = Parameters.from_dict(d)
    orc = Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds)
    U0 = orc.initial_condition("tgv")
    dt = 0.02 if kw.get("pde") != "navier_stokes" else 0.01
    whole = DGStrong(prm)
    whole.solution = U0
    ode = RungeKuttaODESolver(whole)
    parts = _slabs(prm, world)
    dgs = [p for p, _ in parts]
    for dg, u in zip(dgs, _scatter(whole, dgs, U0)):
        dg.solution = u
    odes = [RungeKuttaODESolver(dg) for dg in dgs]
    e0 = orc.numerical_entropy(U0)
    for step in range(4):
        ode.step_in_time(dt)
        _in_threads([lambda k=k: (odes[k].step_in_time(dt), parts[k][1].synchronize()) for k in range(world)])
        gam = [o.relaxation_parameter for o in odes]
        U = _gather(whole, dgs, [dg.solution for dg in dgs])
        err = float(np.max(np.abs(U - whole.solution)) / np.max(np.abs(whole.solution)))
        g_err = max(abs(g - ode.relaxation_parameter) for g in gam) / ode.relaxation_parameter
        print(f"{name} step {step}: gamma {gam[0]:.15f} (whole {ode.relaxation_parameter:.15f}, rel {g_err:.2e}), "
              f"state rel err {err:.2e}")
        assert len(set(gam)) == 1          # every rank took the same root
        assert g_err <= 1e-5 and err <= 5e-9
    assert abs(odes[0].current_time - ode.current_time) <= 1e-5 * ode.current_time
    drift = (orc.numerical_entropy(U) - e0) / abs(e0)
    print(f"{name}: entropy change over 4 relaxed slab steps {drift:.3e}")
    if kw.get("conv") == "two_point_flux" and kw.get("pde", "euler") == "euler":
        assert abs(drift) <= 1e-12
    else:
        assert drift < 0.0

    class NoSum:
        def __init__(self, halo):
            self.callback = halo.callback

    lonely = DGStrong(prm, slab=(0, prm.n_cells), halo=NoSum(LoopbackHalo()))
    lonely.solution = _scatter(whole, [lonely], U0)[0]
    with pytest.raises(_lib.PhError, match="ph_set_rank_sum"):
        RungeKuttaODESolver(lonely).step_in_time(dt)


def _gl_prm(nodes="GL", overintegration=0, **kw):
    from philip_b200.prm import Parameters
    from helpers import prm_dict
    d = prm_dict(**kw)
    d["flux_nodes_type"] = nodes
    d["overintegration"] = overintegration
    return Parameters.from_dict(d)


GL_SLAB_CASES = [
    ("gl_ns_br2_split_p3_two_slabs", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 2, 0.0),
    ("gl_euler_conservative_roe_p2_three_slabs", dict(poly_degree=2, n_cells=4, split=False, conv="roe"), 3, 0.0),
    ("gll_overint1_ns_sipg_p2_two_slabs", dict(nodes="GLL", overintegration=1, poly_degree=2, n_cells=4,
                                               pde="navier_stokes"), 2, 0.0),
    ("gl_curvilinear_euler_p3_two_slabs", dict(poly_degree=3, n_cells=4), 2, 0.1),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,world,warp", GL_SLAB_CASES, ids=[c[0] for c in GL_SLAB_CASES])
def test_gl_slabs_are_the_whole_mesh(name, kw, world, warp):
    """Slabs on uncollocated flux nodes: the partition faces' face values (after the face-value
    kernel) and each side's F_v . n (after the auxiliary kernel) go through the exchange into
    the ghost cells' face blocks, so the residual and three RK4 steps are bitwise the whole
    mesh's."""
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from helpers import TWO_PI, perturbed_tgv
    prm = _gl_prm(**kw)
    whole = DGStrong(prm, warp=warp)
    U0 = perturbed_tgv(Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds), seed=len(name))
    parts = _slabs(prm, world, warp=warp)
    dgs = [p for p, _ in parts]
    Us = _scatter(whole, dgs, U0)
    Rs = _in_threads([lambda k=k: dgs[k].residual_of(Us[k]) for k in range(world)])
    R = _gather(whole, dgs, Rs)
    R_whole = whole.residual_of(U0)
    print(f"{name}: max |R_slabs - R_whole| = {np.max(np.abs(R - R_whole)):.3e}")
    assert np.array_equal(R, R_whole)
    dt = 0.1 * TWO_PI / prm.n_cells / (prm.poly_degree + 1) / 11.0
    whole.solution = U0
    RungeKuttaODESolver(whole).step_in_time(dt, nsteps=3)
    for dg, u in zip(dgs, Us):
        dg.solution = u
    _in_threads([lambda k=k: (RungeKuttaODESolver(dgs[k]).step_in_time(dt, nsteps=3), parts[k][1].synchronize())
                 for k in range(world)])
    U = _gather(whole, dgs, [dg.solution for dg in dgs])
    print(f"{name}: max |U_slabs - U_whole| = {np.max(np.abs(U - whole.solution)):.3e}")
    assert np.array_equal(U, whole.solution)


WALL_SLAB_CASES = [
    ("ns_br2_p3_walls_y_two_slabs", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 2,
     "GLL", ["periodic", "periodic", "wall", "wall", "periodic", "periodic"], 0.0),
    ("euler_roe_p2_riemann_x_three_slabs", dict(poly_degree=2, n_cells=6, split=False, conv="roe"), 3, "GLL",
     ["riemann_farfield", "riemann_farfield", "slip_wall", "slip_wall", "periodic", "periodic"], 0.0),
    ("ns_br2_p2_walls_interior_overlap", dict(poly_degree=2, n_cells=6, pde="navier_stokes", diss="bassi_rebay_2"), 2,
     "GLL", ["wall", "wall", "wall", "wall", "periodic", "periodic"], 0.0),
    ("gl_ns_br2_p3_walls_y_two_slabs", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 2,
     "GL", ["periodic", "periodic", "wall", "wall", "periodic", "periodic"], 0.0),
    ("curvilinear_ns_br2_p3_walls_y_two_slabs", dict(poly_degree=3, n_cells=4, pde="navier_stokes",
                                                     diss="bassi_rebay_2"), 2, "GLL",
     ["periodic", "periodic", "wall", "wall", "periodic", "periodic"], 0.1),
    # walls on the sides the slabs cut: the first and last slab's outer faces are boundary faces
    # (the halo's wrap-around transfer is then unused)
    ("ns_br2_p3_walls_z_two_slabs", dict(poly_degree=3, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 2,
     "GLL", ["periodic", "periodic", "periodic", "periodic", "wall", "wall"], 0.0),
    ("gl_euler_p2_farfield_z_three_slabs", dict(poly_degree=2, n_cells=6, split=False, conv="roe"), 3, "GL",
     ["slip_wall", "slip_wall", "periodic", "periodic", "riemann_farfield", "riemann_farfield"], 0.0),
    ("ns_br2_p2_box_two_slabs", dict(poly_degree=2, n_cells=4, pde="navier_stokes", diss="bassi_rebay_2"), 2,
     "GLL", ["wall"] * 6, 0.0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,world,nodes,bnd,warp", WALL_SLAB_CASES, ids=[c[0] for c in WALL_SLAB_CASES])
def test_slabs_with_walls_are_the_whole_mesh(name, kw, world, nodes, bnd, warp):
    """Slabs of a mesh with boundary conditions on its x / y sides: every slab splits its launches
    into the periodic kernel's tiles and the boundary-face kernel's, also for the interior cells
    that run while a transfer is in flight, so the residual and three RK4 steps are bitwise the
    whole mesh's."""
    from oracle.oracle import Oracle
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from helpers import TWO_PI, perturbed_tgv
    prm = _gl_prm(nodes=nodes, **kw)
    whole = DGStrong(prm, warp=warp, boundaries=bnd)
    U0 = perturbed_tgv(Oracle(prm.oracle_cfg(), prm.n_cells, *prm.grid_bounds), seed=len(name))
    parts = _slabs(prm, world, warp=warp, boundaries=bnd)
    dgs = [p for p, _ in parts]
    Us = _scatter(whole, dgs, U0)
    Rs = _in_threads([lambda k=k: dgs[k].residual_of(Us[k]) for k in range(world)])
    R = _gather(whole, dgs, Rs)
    R_whole = whole.residual_of(U0)
    print(f"{name}: max |R_slabs - R_whole| = {np.max(np.abs(R - R_whole)):.3e}")
    assert np.array_equal(R, R_whole)
    dt = 0.1 * TWO_PI / prm.n_cells / (prm.poly_degree + 1) / 11.0
    whole.solution = U0
    RungeKuttaODESolver(whole).step_in_time(dt, nsteps=3)
    for dg, u in zip(dgs, Us):
        dg.solution = u
    _in_threads([lambda k=k: (RungeKuttaODESolver(dgs[k]).step_in_time(dt, nsteps=3), parts[k][1].synchronize())
                 for k in range(world)])
    U = _gather(whole, dgs, [dg.solution for dg in dgs])
    print(f"{name}: max |U_slabs - U_whole| = {np.max(np.abs(U - whole.solution)):.3e}")
    assert np.array_equal(U, whole.solution)
