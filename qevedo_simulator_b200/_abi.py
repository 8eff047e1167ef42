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
        ("settings", QvdgOptions),
    ]

    def as_dict(self) -> dict:
        out = {name: getattr(self, name) for name, _ in self._fields_ if name != "settings"}
        out["settings"] = settings_dict(self.settings)
        return out


MATH_NAMES = {0: "fp32", 1: "tensor", 2: "gates", 3: "tensor_pairs"}


def settings_dict(o: QvdgOptions) -> dict:
    """Plan settings as plain values (math by name)."""
    return {"max_fused_qubits": int(o.max_fused_qubits), "staged": bool(o.staged), "tile_qubits": int(o.tile_qubits),
            "math": MATH_NAMES.get(int(o.math), str(int(o.math)))}


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


# numpy view of a qvdg_op (two uint32 counts, four pointers).
_OP_DTYPE = np.dtype([("num_targets", "<u4"), ("num_controls", "<u4"), ("targets", "<u8"), ("controls", "<u8"),
                      ("control_values", "<u8"), ("matrix", "<u8")])
assert _OP_DTYPE.itemsize == ct.sizeof(QvdgOp)


class PackedOps:
    """Ops laid out as a contiguous qvdg_op array; owns every buffer the
    structs point into, so it must outlive the call it is passed to."""

    def __init__(self, ops=None, *, parts=None):
        """From ops (targets, controls [(qubit, value)], matrix), or from
        `parts` = (target counts, control counts, qubits with targets first,
        their values, matrices) already laid out."""
        if parts is None:
            qubits, values, mats, ks, cs = [], [], [], [], []
            for op in ops:
                t, ctl = op.targets, op.controls
                ks.append(len(t))
                cs.append(len(ctl))
                qubits += t
                values += [0] * len(t)
                for q, v in ctl:
                    qubits.append(q)
                    values.append(1 if v else 0)
                mats.append(op.matrix)
        else:
            ks, cs, qubits, values, mats = parts
        n = len(ks)
        ks = np.array(ks or [0], dtype=np.uint32)
        cs = np.array(cs or [0], dtype=np.uint32)
        if n:
            sizes = np.fromiter((np.size(m) for m in mats), dtype=np.uint64, count=n)
            if np.any(sizes != np.uint64(4) ** ks.astype(np.uint64)):
                raise ValueError("op matrix does not match its targets")
        self._q = np.array(qubits or [0], dtype=np.uint32)
        self._v = np.array(values or [0], dtype=np.uint8)
        self._m = (np.concatenate([np.ravel(m) for m in mats], dtype=np.complex128).view(np.float64)
                   if mats else np.zeros(2))
        self._ops = np.zeros(max(n, 1), dtype=_OP_DTYPE)
        if n:
            ks, cs = ks[:n], cs[:n]
            qpos = np.concatenate(([0], np.cumsum(ks.astype(np.uint64) + cs)[:-1])).astype(np.uint64)
            sizes = np.uint64(4) ** ks.astype(np.uint64)
            mpos = np.concatenate(([0], np.cumsum(sizes)[:-1])).astype(np.uint64)
            qbase, vbase, mbase = (np.uint64(a.ctypes.data) for a in (self._q, self._v, self._m))
            o = self._ops[:n]
            o["num_targets"] = ks
            o["num_controls"] = cs
            o["targets"] = qbase + np.uint64(4) * qpos
            o["controls"] = qbase + np.uint64(4) * (qpos + ks)
            o["control_values"] = vbase + qpos + ks
            o["matrix"] = mbase + np.uint64(16) * mpos
        self.array = (QvdgOp * max(n, 1)).from_buffer(self._ops)
        self.count = n


def as_double_ptr(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def as_u64_ptr(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_uint64))
