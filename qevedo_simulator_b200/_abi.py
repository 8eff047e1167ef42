"""ctypes mirror of include/qvdg.h: the op, options and stats structs and the
marshalling of host ops into them."""

from __future__ import annotations

import ctypes as ct

import numpy as np


class QvdgOp(ct.Structure):
    _fields_ = [
        ("num_targets", ct.c_uint32),
        ("num_controls", ct.c_uint32),
        ("targets", ct.POINTER(ct.c_uint32)),
        ("controls", ct.POINTER(ct.c_uint32)),
        ("control_values", ct.POINTER(ct.c_uint8)),
        ("matrix", ct.POINTER(ct.c_double)),
    ]


class QvdgOptions(ct.Structure):
    _fields_ = [
        ("max_fused_qubits", ct.c_uint32),
        ("staged", ct.c_uint32),
        ("tile_qubits", ct.c_uint32),
        ("planner", ct.c_uint32),
        ("math", ct.c_uint32),
    ]


class QvdgStats(ct.Structure):
    _fields_ = [
        ("gates", ct.c_uint64),
        ("kernels", ct.c_uint64),
        ("passes", ct.c_uint64),
        ("stages", ct.c_uint64),
        ("gate_seconds", ct.c_double),
        ("bytes", ct.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class QvdgLayeredCircuit(ct.Structure):
    _fields_ = [
        ("num_qubits", ct.c_uint32),
        ("num_layers", ct.c_uint32),
        ("entangler", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("gates", ct.POINTER(ct.c_double)),
    ]


class QvdgBatchOptions(ct.Structure):
    _fields_ = [("tile_qubits", ct.c_uint32), ("threads", ct.c_uint32)]


class QvdgBatchSummary(ct.Structure):
    _fields_ = [
        ("tile_qubits", ct.c_uint32),
        ("threads", ct.c_uint32),
        ("ctas", ct.c_uint32),
        ("candidates", ct.c_uint32),
        ("circuits", ct.c_uint64),
        ("outputs", ct.c_uint64),
        ("tune_seconds", ct.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PackedOps:
    """Ops laid out as a contiguous qvdg_op array; owns every buffer the
    structs point into, so it must outlive the call it is passed to."""

    def __init__(self, ops):
        n = len(ops)
        self.array = (QvdgOp * max(n, 1))()
        qubits = sum(len(op.targets) + len(op.controls) for op in ops)
        self._q = np.zeros(max(qubits, 1), dtype=np.uint32)
        self._v = np.zeros(max(qubits, 1), dtype=np.uint8)
        sizes = [4 ** len(op.targets) for op in ops]
        self._m = np.zeros(2 * max(sum(sizes), 1), dtype=np.float64)
        qpos = mpos = 0
        qbase = self._q.ctypes.data
        vbase = self._v.ctypes.data
        mbase = self._m.ctypes.data
        for i, op in enumerate(ops):
            k, c = len(op.targets), len(op.controls)
            self._q[qpos:qpos + k] = op.targets
            for j, (q, v) in enumerate(op.controls):
                self._q[qpos + k + j] = q
                self._v[qpos + k + j] = 1 if v else 0
            m = np.ascontiguousarray(op.matrix, dtype=np.complex128).reshape(-1)
            if m.size != sizes[i]:
                raise ValueError("op matrix does not match its targets")
            self._m[2 * mpos:2 * (mpos + m.size)] = m.view(np.float64)
            s = self.array[i]
            s.num_targets = k
            s.num_controls = c
            s.targets = ct.cast(qbase + 4 * qpos, ct.POINTER(ct.c_uint32))
            s.controls = ct.cast(qbase + 4 * (qpos + k), ct.POINTER(ct.c_uint32))
            s.control_values = ct.cast(vbase + qpos + k, ct.POINTER(ct.c_uint8))
            s.matrix = ct.cast(mbase + 16 * mpos, ct.POINTER(ct.c_double))
            qpos += k + c
            mpos += m.size
        self.count = n


def as_double_ptr(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def as_u64_ptr(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_uint64))
