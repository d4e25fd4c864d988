"""Snapshot matrix and POD basis (OnlinePOD::addSnapshot / computeBasis,
src/reduced_order/pod_basis_online.cpp:28-89; the time POD of FlowSolver::run,
src/flow_solver/flow_solver.cpp:110-120, :675-688).

CPU: the oracle's restatement against the SVD's defining properties (centring, reconstruction,
orthonormality, ordering). GPU: the device snapshot matrix holds exactly the appended states
(from a host vector, a context's resident state and a batch solve, all by device copies for the
latter two), grows past its capacity, and its POD (method of snapshots: cuBLAS DSYRK Gram,
Jacobi eigenvectors, cuBLAS DGEMM) matches the oracle within the method's accuracy
(sigma_k to 1e-16 (sigma_1 / sigma_k)^2 relative; the basis vectors of well-separated singular
values to 1e-8); FlowSolver's time POD keeps every snapshot-iteration state bitwise and writes
the snapshot file."""
import os

import numpy as np
import pytest

from oracle.pod import compute_basis, sign_rule


def _low_rank(ndofs=20000, m=10, seed=3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((ndofs, m)))
    R, _ = np.linalg.qr(rng.standard_normal((m, m)))
    sig = np.logspace(0, -3, m)
    return 5.0 + Q @ np.diag(sig) @ R.T * 100.0


def test_oracle_pod_properties():
    S = _low_rank(2000, 8)
    ref, s, U = compute_basis(S)
    Sc = S - ref[:, None]
    assert np.allclose(ref, S.mean(axis=1))
    assert np.allclose(U.T @ U, np.eye(U.shape[1]), atol=1e-12)
    assert np.all(np.diff(s) <= 0)
    # reconstruction of the centred snapshots from the basis
    assert np.allclose(U @ (U.T @ Sc), Sc, atol=1e-10 * np.abs(Sc).max())
    Us = sign_rule(U)
    for k in range(Us.shape[1]):
        assert Us[np.argmax(np.abs(Us[:, k])), k] > 0


@pytest.mark.gpu
def test_device_pod_matches_the_oracle():
    from philip_b200.pod import OnlinePOD
    S = _low_rank()
    pod = OnlinePOD(S.shape[0], 4, rel_tol=1e-5)       # capacity 4: grows twice
    for j in range(S.shape[1]):
        pod.addSnapshot(S[:, j])
    assert pod.count == S.shape[1]
    assert np.array_equal(pod.getSnapshotMatrix(), S)
    U = pod.computeBasis()
    ref_o, s_o, U_o = compute_basis(S)
    assert np.max(np.abs(pod.getReferenceState() - ref_o)) <= 1e-14 * np.max(np.abs(ref_o))
    r = U.shape[1]
    assert r == S.shape[1] - 1                          # centring removes one dimension
    s = pod.singular_values
    rel = np.abs(s[:r] - s_o[:r]) / s_o[:r]
    bound = 1e-16 * (s_o[0] / s_o[:r]) ** 2 * 100 + 1e-14
    print("sigma", s[:r], "rel err", rel)
    assert np.all(rel <= bound)
    assert s[r] == 0.0
    U_o = sign_rule(U_o[:, :r])
    for k in range(r):
        err = np.max(np.abs(U[:, k] - U_o[:, k]))
        print(f"mode {k}: sigma {s[k]:.3e}, max |u - u_oracle| {err:.2e}")
        assert err <= 1e-8 * (s_o[0] / s_o[k]) ** 2
    assert np.allclose(U.T @ U, np.eye(r), atol=1e-8)
    pod.close()


@pytest.mark.gpu
def test_snapshots_from_a_context_and_a_batch_solve():
    from philip_b200 import _lib
    from philip_b200.dg import DGStrong, RungeKuttaODESolver
    from philip_b200.pod import OnlinePOD
    from philip_b200.serve import Batch, SolveRequest
    req = SolveRequest("isentropic_vortex", n_cells=3, poly_degree=3, mach=0.3, final_time=0.05)
    U0, dt, nsteps = req.prepare()
    dg = DGStrong(req.parameters())
    dg.solution = U0
    pod = OnlinePOD(req.ndofs, 2)
    pod.addSnapshot(dg)
    RungeKuttaODESolver(dg).step_in_time(dt, nsteps=nsteps)
    pod.addSnapshot(dg)
    b = Batch(1 << 28, _lib.PH_FP64)
    slot = b.admit(req.mesh(), req.parameters().to_ph_params(_lib.PH_FP64), U0, dt, nsteps)
    b.step(nsteps)
    pod.addSnapshot(b, slot=slot)
    S = pod.getSnapshotMatrix()
    assert np.array_equal(S[:, 0], U0)
    assert np.array_equal(S[:, 1], dg.solution)
    assert np.array_equal(S[:, 2], b.state(slot, req.ndofs))
    assert np.array_equal(S[:, 1], S[:, 2])            # a batch solve is the single solve bitwise
    b.close()
    pod.close()


@pytest.mark.gpu
def test_flow_solver_time_pod(tmp_path, monkeypatch):
    from helpers import prm_dict
    from philip_b200.dg import FlowSolver
    from philip_b200.prm import Parameters
    monkeypatch.chdir(tmp_path)
    d = prm_dict(poly_degree=2, n_cells=3, pde="navier_stokes", final_time=0.03, cfl=0.01)
    d["reduced order/output_snapshot_every_x_timesteps"] = "2"
    prm = Parameters.from_dict(d)
    fs = FlowSolver(prm)
    dt = fs.time_step()
    fs.run(record_every=1)
    S = fs.time_pod.getSnapshotMatrix()
    # the same steps on the host, keeping the state at iterations 0, 2, 4, ...
    ref = FlowSolver(Parameters.from_dict({k: v for k, v in d.items() if not k.startswith("reduced order")}))
    ode = ref.ode_solver
    cols = [ref.dg.solution]
    while ode.current_time < 0.03:
        ode.step_in_time(min(dt, 0.03 - ode.current_time))
        if ode.current_iteration % 2 == 0:
            cols.append(ref.dg.solution)
    assert S.shape == (fs.dg.n_dofs, len(cols))
    for j, c in enumerate(cols):
        assert np.array_equal(S[:, j], c), j
    name = f"solution_snapshots_iteration_{fs.ode_solver.current_iteration}.txt"
    assert os.path.exists(name)
    F = np.loadtxt(name, ndmin=2)
    assert F.shape == S.shape and np.allclose(F, S, rtol=1e-15, atol=0.0)
