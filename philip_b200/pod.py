"""Snapshot matrix on the device and its POD basis: the host mirror of the reference's
OnlinePOD (src/reduced_order/pod_basis_online.h / .cpp:28-99) over ph_snapshots_* in
include/philip_b200.h.

  addSnapshot(x) ......... append a column: a DGStrong (its resident state, copied on the
                           device), a batch solve (Batch, slot), or a host vector
  computeBasis() ......... reference state (row mean), centred snapshots, thin SVD's left
                           singular vectors, computed on the device by the method of snapshots
  getPODBasis() / getReferenceState() / getSnapshotMatrix() / singular_values
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class OnlinePOD:
    def __init__(self, ndofs: int, capacity: int, rel_tol: float = 1e-6):
        """rel_tol: singular values below rel_tol x the largest are dropped from the basis (the
        centred matrix has rank at most m - 1; the method of snapshots resolves sigma_k to about
        1e-16 (sigma_1 / sigma_k)^2 relative, and the Gram matrix's rounding leaves the null
        directions at about 1e-7 sigma_1)."""
        self.L = _lib.load()
        self.ndofs = int(ndofs)
        self.rel_tol = float(rel_tol)
        h = ctypes.c_void_p()
        _lib.check(self.L.ph_snapshots_create(self.ndofs, int(capacity), ctypes.byref(h)))
        self._h = h
        self._basis = None
        self._reference = None
        self.singular_values = None

    def close(self):
        if getattr(self, "_h", None) is not None:
            self.L.ph_snapshots_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def count(self) -> int:
        m = ctypes.c_int(0)
        _lib.check(self.L.ph_snapshots_count(self._h, ctypes.byref(m)))
        return int(m.value)

    def addSnapshot(self, snapshot, slot: int | None = None):
        """OnlinePOD::addSnapshot (pod_basis_online.cpp:28-46)."""
        from .dg import DGStrong
        if isinstance(snapshot, DGStrong):
            _lib.check(self.L.ph_snapshots_add_state(self._h, snapshot.handle))
        elif slot is not None:                       # a Batch and the slot of one of its solves
            _lib.check(self.L.ph_snapshots_add_batch(self._h, snapshot._h, int(slot)))
        else:
            U = np.ascontiguousarray(snapshot, dtype=np.float64)
            if U.size != self.ndofs:
                raise ValueError("snapshot size mismatch")
            _lib.check(self.L.ph_snapshots_add(self._h, U.ctypes.data, _lib.PH_HOST))

    def getSnapshotMatrix(self) -> np.ndarray:
        """ndofs x m, as OnlinePOD::getSnapshotMatrix."""
        m = self.count
        S = np.empty((m, self.ndofs))
        if m:
            _lib.check(self.L.ph_snapshots_get(self._h, S.ctypes.data, _lib.PH_HOST))
        return S.T

    def computeBasis(self):
        """OnlinePOD::computeBasis (pod_basis_online.cpp:49-89)."""
        m = self.count
        ref = np.empty(self.ndofs)
        sig = np.empty(max(m, 1))
        basis = np.empty((max(m, 1), self.ndofs))
        r = ctypes.c_int(0)
        _lib.check(self.L.ph_snapshots_pod(self._h, self.rel_tol, ref.ctypes.data, sig.ctypes.data, basis.ctypes.data,
                                           _lib.PH_HOST, ctypes.byref(r)))
        self._reference = ref
        self.singular_values = sig[:m]
        self._basis = basis[: r.value].T.copy()
        return self._basis

    def getPODBasis(self) -> np.ndarray:
        return self._basis

    def getReferenceState(self) -> np.ndarray:
        return self._reference


def write_snapshot_matrix(path: str, S: np.ndarray):
    """The snapshot file FlowSolver::run writes at the end (flow_solver.cpp:683-688): one row per
    DOF, one column per snapshot, 16 significant digits in scientific notation, zeros as "0"."""
    with open(path, "w") as f:
        for row in S:
            f.write(" ".join("0" if v == 0.0 else f"{v:.16e}" for v in row) + "\n")
