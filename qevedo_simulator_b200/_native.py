"""ctypes binding of libqvdgpu.so (include/qvdg.h).

The library is the product: there is no CPU fallback. Loading fails loudly
when it has not been built (python -m qevedo_simulator_b200.build) or when
no CUDA device is present at the first call that needs one.
"""

from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from ._abi import (PackedOps, QvdgBatchOptions, QvdgBatchSummary, QvdgLayeredCircuit, QvdgOp, QvdgOptions,
                   QvdgStats, as_double_ptr, as_u64_ptr)

LIBRARY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libqvdgpu.so")

STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA error", 4: "unsupported", 5: "timeout"}

# Every exported function: name -> (restype, argtypes).
_P = ct.c_void_p
_SIGNATURES = {
    "qvdg_default_options": (None, [ct.POINTER(QvdgOptions)]),
    "qvdg_last_error": (ct.c_char_p, []),
    "qvdg_version": (ct.c_char_p, []),
    "qvdg_state_create": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.POINTER(_P)]),
    "qvdg_state_destroy": (ct.c_int, [_P]),
    "qvdg_state_zero": (ct.c_int, [_P]),
    "qvdg_state_info": (ct.c_int, [_P, ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint32)]),
    "qvdg_state_set_amplitudes": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.c_size_t]),
    "qvdg_state_get_amplitudes": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.c_size_t]),
    "qvdg_apply_ops": (ct.c_int, [_P, ct.POINTER(QvdgOp), ct.c_size_t, ct.POINTER(QvdgOptions),
                                  ct.POINTER(QvdgStats)]),
    "qvdg_apply": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.POINTER(ct.c_uint32), ct.c_uint32,
                              ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint8), ct.c_uint32]),
    "qvdg_norm_sqr": (ct.c_int, [_P, ct.POINTER(ct.c_double)]),
    "qvdg_scale": (ct.c_int, [_P, ct.c_double]),
    "qvdg_probability_one": (ct.c_int, [_P, ct.c_uint32, ct.POINTER(ct.c_double)]),
    "qvdg_expect_z_all": (ct.c_int, [_P, ct.POINTER(ct.c_double)]),
    "qvdg_probabilities": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.c_size_t]),
    "qvdg_measure": (ct.c_int, [_P, ct.c_uint32, ct.c_double, ct.POINTER(ct.c_int32)]),
    "qvdg_reset": (ct.c_int, [_P, ct.c_uint32, ct.c_double]),
    "qvdg_sample_unordered": (ct.c_int, [_P, ct.c_size_t, ct.POINTER(ct.c_double), ct.POINTER(ct.c_uint64),
                                         ct.POINTER(ct.c_size_t)]),
    "qvdg_swap_physical": (ct.c_int, [_P, ct.POINTER(ct.c_uint32), ct.c_uint32]),
    "qvdg_state_layout": (ct.c_int, [_P, ct.POINTER(ct.c_uint32)]),
    "qvdg_state_device_buffer": (ct.c_int, [_P, ct.POINTER(_P), ct.POINTER(ct.c_size_t)]),
    "qvdg_synchronize": (ct.c_int, [_P]),
    "qvdg_plan_create": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.POINTER(QvdgOp), ct.c_size_t,
                                    ct.POINTER(QvdgOptions), ct.POINTER(_P)]),
    "qvdg_plan_destroy": (ct.c_int, [_P]),
    "qvdg_plan_info": (ct.c_int, [_P, ct.POINTER(QvdgStats)]),
    "qvdg_plan_execute": (ct.c_int, [_P, _P, ct.POINTER(QvdgStats)]),
    "qvdg_set_device": (ct.c_int, [ct.c_int32]),
    "qvdg_get_device": (ct.c_int, [ct.POINTER(ct.c_int32)]),
    "qvdg_max_abs_diff": (ct.c_int, [_P, _P, ct.POINTER(ct.c_double)]),
    "qvdg_set_pass_timing": (ct.c_int, [_P, ct.c_int32]),
    "qvdg_pass_times": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double), ct.POINTER(ct.c_int32),
                                   ct.c_size_t, ct.POINTER(ct.c_size_t)]),
    "qvdg_batch_create": (ct.c_int, [ct.POINTER(QvdgLayeredCircuit), ct.c_size_t, ct.POINTER(QvdgBatchOptions),
                                     ct.POINTER(_P)]),
    "qvdg_batch_destroy": (ct.c_int, [_P]),
    "qvdg_batch_set_gates": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.c_size_t]),
    "qvdg_batch_run": (ct.c_int, [_P, ct.POINTER(ct.c_double), ct.c_size_t, ct.POINTER(ct.c_double)]),
    "qvdg_batch_info": (ct.c_int, [_P, ct.POINTER(QvdgBatchSummary)]),
    "qvdg_batch_tuning": (ct.c_int, [_P, ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_double),
                                     ct.c_size_t, ct.POINTER(ct.c_size_t)]),
    "qvdg_sample_counts": (ct.c_int, [_P, ct.c_size_t, ct.POINTER(ct.c_double), ct.POINTER(ct.c_uint32),
                                      ct.POINTER(ct.c_uint32), ct.c_size_t, ct.POINTER(ct.c_uint64),
                                      ct.POINTER(ct.c_uint64), ct.c_size_t, ct.POINTER(ct.c_size_t)]),
    "qvdg_expect_pauli": (ct.c_int, [_P, ct.POINTER(ct.c_uint32), ct.c_char_p, ct.c_size_t, ct.POINTER(ct.c_double)]),
    "qvdg_plan_features": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.POINTER(QvdgOp), ct.c_size_t,
                                      ct.POINTER(QvdgOptions), ct.POINTER(ct.c_float), ct.c_size_t,
                                      ct.POINTER(ct.c_size_t)]),
    "qvdg_plan_features_from": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.POINTER(QvdgOp), ct.c_size_t,
                                           ct.POINTER(QvdgOptions), ct.c_int32, ct.POINTER(ct.c_float), ct.c_size_t,
                                           ct.POINTER(ct.c_size_t)]),
    "qvdg_plan_fused_ops": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.POINTER(QvdgOp), ct.c_size_t,
                                       ct.POINTER(QvdgOptions), ct.c_int32, ct.POINTER(ct.c_uint32),
                                       ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint8),
                                       ct.POINTER(ct.c_double), ct.c_size_t, ct.POINTER(ct.c_size_t),
                                       ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_size_t)]),
    "qvdg_mlp_create": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.c_uint64, ct.POINTER(_P)]),
    "qvdg_mlp_destroy": (ct.c_int, [_P]),
    "qvdg_mlp_num_params": (ct.c_int, [_P, ct.POINTER(ct.c_size_t)]),
    "qvdg_mlp_get_params": (ct.c_int, [_P, ct.POINTER(ct.c_float), ct.c_size_t]),
    "qvdg_mlp_set_params": (ct.c_int, [_P, ct.POINTER(ct.c_float), ct.c_size_t]),
    "qvdg_mlp_forward": (ct.c_int, [_P, ct.POINTER(ct.c_float), ct.c_size_t, ct.POINTER(ct.c_float)]),
    "qvdg_mlp_gradients": (ct.c_int, [_P, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), ct.c_size_t,
                                      ct.POINTER(ct.c_float), ct.POINTER(ct.c_float)]),
    "qvdg_mlp_train": (ct.c_int, [_P, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), ct.c_size_t, ct.c_uint32,
                                  ct.c_uint32, ct.c_float, ct.c_uint64, ct.POINTER(ct.c_float)]),
    "qvdg_bit_probabilities_noalloc": (ct.c_int, [_P, ct.c_uint32, ct.c_uint32, _P, ct.POINTER(ct.c_double),
                                                  ct.POINTER(ct.c_double)]),
    "qvdg_cost_model_set": (ct.c_int, [ct.POINTER(ct.c_float), ct.c_size_t, ct.c_uint32, ct.c_uint32]),
    "qvdg_cost_model_clear": (ct.c_int, []),
    "qvdg_planner_candidates": (ct.c_int, [ct.c_uint32, ct.POINTER(QvdgOptions), ct.c_size_t,
                                           ct.POINTER(ct.c_size_t)]),
    "qvdg_plan_choose": (ct.c_int, [ct.c_uint32, ct.c_uint32, ct.POINTER(QvdgOp), ct.c_size_t, ct.c_int32,
                                    ct.POINTER(QvdgOptions), ct.POINTER(ct.c_double), ct.c_size_t,
                                    ct.POINTER(ct.c_size_t)]),
}

_lib = None


def lib() -> ct.CDLL:
    """The loaded library (raises if it is missing: no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(f"{LIBRARY} is missing: build it with `python -m qevedo_simulator_b200.build`")
        L = ct.CDLL(LIBRARY)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class QvdgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} ({STATUS.get(status, status)})")
        self.status = status


def check(status: int):
    if status != 0:
        msg = lib().qvdg_last_error().decode()
        if status == 1:
            raise ValueError(msg)
        if status == 2:
            raise MemoryError(msg)
        raise QvdgError(status, msg)


def bit_probabilities_noalloc(pointer: int, num_qubits: int, precision_bits: int, stream: int = 0):
    """(p1, total) of a state vector in the caller's own device memory at
    `pointer`, computed with the library's fixed scratch array and no
    allocation (for callers whose device memory is all spoken for). p1[q] is
    the unnormalised weight of bit q = 1; calls that overlap on the GPU race."""
    p1 = np.zeros(max(int(num_qubits), 1), dtype=np.float64)
    total = ct.c_double()
    check(lib().qvdg_bit_probabilities_noalloc(ct.c_void_p(pointer), int(num_qubits), int(precision_bits),
                                               ct.c_void_p(stream), as_double_ptr(p1), ct.byref(total)))
    return p1[:num_qubits], total.value


def set_device(device: int):
    """Select the CUDA device for states and plans created by this thread."""
    check(lib().qvdg_set_device(int(device)))


MATH = {"fp32": 0, "tensor": 1, "gates": 2, "tensor_pairs": 3}
PLANNERS = {"greedy": 0, "learned": 1}
COST_MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "cost_model.npz")
_models_registered = set()


def register_cost_model(params, inputs: int, hidden: int):
    """Register the learned planner's cost model (the MLP parameters) for the
    current device, replacing any earlier one."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    check(lib().qvdg_cost_model_set(p.ctypes.data_as(ct.POINTER(ct.c_float)), p.size, int(inputs), int(hidden)))
    _models_registered.add(_current_device())


def ensure_cost_model() -> bool:
    """Register the committed cost model (data/cost_model.npz) for the current
    device once; False when the file is absent (the learned planner then
    uses its fallback settings)."""
    dev = _current_device()
    if dev in _models_registered:
        return True
    if not os.path.exists(COST_MODEL_PATH):
        return False
    d = np.load(COST_MODEL_PATH)
    register_cost_model(d["params"], int(d["inputs"]), int(d["hidden"]))
    return True


def clear_cost_model():
    check(lib().qvdg_cost_model_clear())
    _models_registered.discard(_current_device())


def _current_device() -> int:
    d = ct.c_int32()
    check(lib().qvdg_get_device(ct.byref(d)))
    return int(d.value)


def planner_candidates(precision_bits: int = 32) -> list:
    """The learned planner's candidate settings, in its reporting order."""
    n = ct.c_size_t()
    check(lib().qvdg_planner_candidates(int(precision_bits), None, 0, ct.byref(n)))
    arr = (QvdgOptions * max(n.value, 1))()
    check(lib().qvdg_planner_candidates(int(precision_bits), arr, n.value, ct.byref(n)))
    return [arr[i] for i in range(n.value)]


def plan_choose(ops, num_qubits: int, from_zero: bool = True):
    """(chosen options, [predicted seconds per candidate]) of the learned
    planner for `ops` on a complex64 state (needs a registered model)."""
    packed = PackedOps(ops)
    chosen = QvdgOptions()
    cands = planner_candidates(32)
    pred = np.zeros(max(len(cands), 1), dtype=np.float64)
    n = ct.c_size_t()
    check(lib().qvdg_plan_choose(int(num_qubits), 32, packed.array, packed.count, 1 if from_zero else 0,
                                 ct.byref(chosen), as_double_ptr(pred), pred.size, ct.byref(n)))
    return chosen, pred[:n.value]


def options(max_fused_qubits: int = 4, staged: bool = True, tile_qubits: int = 0, planner: int | str = 0,
            math: str = "fp32") -> QvdgOptions:
    """Simulator options (the reference's Options, src/simulator.rs:37-66).
    `math="tensor"` runs fused dense gates on the tensor cores (complex64
    states only): 3-6 qubit gates inside staged tiles, 4-6 qubit gates as
    plain passes; `math="gates"` makes plain passes
    apply a fused 4-5 qubit group gate by gate in registers;
    `math="tensor_pairs"` is "tensor" with two fused 6-qubit gates per plain
    pass where they have no controls."""
    o = QvdgOptions()
    o.max_fused_qubits = int(max_fused_qubits)
    o.staged = 1 if staged else 0
    o.tile_qubits = int(tile_qubits)
    o.planner = PLANNERS[planner] if isinstance(planner, str) else int(planner)
    o.math = MATH[math]
    return o


class DeviceState:
    """A state vector on the current CUDA device (a qvdg_state handle).

    Mirrors the reference's StateVector<T> (src/state.rs, src/measure.rs):
    logical qubits and indices everywhere, precision 32 (complex64) or 64
    (complex128)."""

    def __init__(self, num_qubits: int, precision_bits: int = 32):
        self._h = ct.c_void_p()
        check(lib().qvdg_state_create(int(num_qubits), int(precision_bits), ct.byref(self._h)))
        self.num_qubits = int(num_qubits)
        self.precision_bits = int(precision_bits)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().qvdg_state_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state management
    def zero(self):
        check(lib().qvdg_state_zero(self._h))

    def set_amplitudes(self, amplitudes):
        a = np.ascontiguousarray(amplitudes, dtype=np.complex128)
        check(lib().qvdg_state_set_amplitudes(self._h, as_double_ptr(a.view(np.float64)), a.size))

    def amplitudes(self) -> np.ndarray:
        out = np.empty(1 << self.num_qubits, dtype=np.complex128)
        check(lib().qvdg_state_get_amplitudes(self._h, as_double_ptr(out.view(np.float64)), out.size))
        return out

    # -- gates
    def apply_ops(self, ops, opts: QvdgOptions | None = None) -> dict:
        packed = PackedOps(ops)
        stats = QvdgStats()
        check(lib().qvdg_apply_ops(self._h, packed.array, packed.count, ct.byref(opts) if opts else None,
                                   ct.byref(stats)))
        return stats.as_dict()

    def apply_packed(self, packed: PackedOps, opts: QvdgOptions | None = None) -> dict:
        stats = QvdgStats()
        check(lib().qvdg_apply_ops(self._h, packed.array, packed.count, ct.byref(opts) if opts else None,
                                   ct.byref(stats)))
        return stats.as_dict()

    def apply(self, matrix, qubits, controls=()):
        m = np.ascontiguousarray(matrix, dtype=np.complex128)
        q = np.array(list(qubits) or [0], dtype=np.uint32)
        cq = np.array([c for c, _ in controls] or [0], dtype=np.uint32)
        cv = np.array([1 if v else 0 for _, v in controls] or [0], dtype=np.uint8)
        check(lib().qvdg_apply(self._h, as_double_ptr(m.view(np.float64)), q.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                               len(qubits), cq.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                               cv.ctypes.data_as(ct.POINTER(ct.c_uint8)), len(controls)))

    def scale(self, factor: float):
        check(lib().qvdg_scale(self._h, float(factor)))

    def swap_physical(self, pairs):
        flat = np.array([x for p in pairs for x in p] or [0], dtype=np.uint32)
        check(lib().qvdg_swap_physical(self._h, flat.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(pairs)))

    def layout(self) -> list:
        out = (ct.c_uint32 * self.num_qubits)()
        check(lib().qvdg_state_layout(self._h, out))
        return list(out)

    # -- measurement
    def norm_sqr(self) -> float:
        v = ct.c_double()
        check(lib().qvdg_norm_sqr(self._h, ct.byref(v)))
        return v.value

    def probability_one(self, qubit: int) -> float:
        v = ct.c_double()
        check(lib().qvdg_probability_one(self._h, int(qubit), ct.byref(v)))
        return v.value

    def expect_z_all(self) -> np.ndarray:
        out = np.empty(self.num_qubits, dtype=np.float64)
        check(lib().qvdg_expect_z_all(self._h, as_double_ptr(out)))
        return out

    def probabilities(self) -> np.ndarray:
        out = np.empty(1 << self.num_qubits, dtype=np.float64)
        check(lib().qvdg_probabilities(self._h, as_double_ptr(out), out.size))
        return out

    def measure(self, qubit: int, uniform: float) -> int:
        v = ct.c_int32()
        check(lib().qvdg_measure(self._h, int(qubit), float(uniform), ct.byref(v)))
        return v.value

    def reset(self, qubit: int, uniform: float):
        check(lib().qvdg_reset(self._h, int(qubit), float(uniform)))

    def sample_unordered(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.empty(max(u.size, 1), dtype=np.uint64)
        count = ct.c_size_t()
        check(lib().qvdg_sample_unordered(self._h, u.size, as_double_ptr(u), as_u64_ptr(out), ct.byref(count)))
        return out[:count.value]

    def sample_counts(self, uniforms, measures):
        """(keys, counts): distinct classical keys (ascending; bit c = the value
        measured into classical bit c) of the shots sampled with `uniforms`,
        for `measures` = [(qubit, clbit), ...] with clbits 0..63."""
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        q = np.array([m[0] for m in measures] or [0], dtype=np.uint32)
        c = np.array([m[1] for m in measures] or [0], dtype=np.uint32)
        n = ct.c_size_t()
        args = (self._h, u.size, as_double_ptr(u), q.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                c.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(measures))
        # At most one distinct key per shot: one call samples and fills.
        keys = np.zeros(max(u.size, 1), dtype=np.uint64)
        counts = np.zeros(max(u.size, 1), dtype=np.uint64)
        check(lib().qvdg_sample_counts(*args, as_u64_ptr(keys), as_u64_ptr(counts), keys.size, ct.byref(n)))
        return keys[:n.value], counts[:n.value]

    def expect_pauli(self, label) -> float:
        """<psi|P|psi> for a Pauli label in Qiskit order (rightmost letter =
        qubit 0), or for [(qubit, letter), ...]."""
        if isinstance(label, str):
            pairs = [(i, ch) for i, ch in enumerate(reversed(label)) if ch.upper() != "I"]
        else:
            pairs = list(label)
        q = np.array([p[0] for p in pairs] or [0], dtype=np.uint32)
        letters = "".join(p[1] for p in pairs).encode()
        v = ct.c_double()
        check(lib().qvdg_expect_pauli(self._h, q.ctypes.data_as(ct.POINTER(ct.c_uint32)), letters, len(pairs),
                                      ct.byref(v)))
        return v.value

    def execute(self, plan: "Plan") -> dict:
        stats = QvdgStats()
        check(lib().qvdg_plan_execute(self._h, plan._h, ct.byref(stats)))
        return stats.as_dict()

    def set_pass_timing(self, enabled: bool = True):
        check(lib().qvdg_set_pass_timing(self._h, 1 if enabled else 0))

    def pass_times(self):
        """(seconds, bytes, kind) per pass of the last gate run; kind 1 is a
        staged tile pass, 0 a single-gate pass, 2 a single-gate pass on the
        tensor cores, 3 the same through a shared-memory stage (gates on
        index bits 1-3), 4 a zero-start pass (run from |0...0>, it skips the
        still-zero amplitudes of qubits no earlier pass touched)."""
        count = ct.c_size_t()
        check(lib().qvdg_pass_times(self._h, None, None, None, 0, ct.byref(count)))
        n = count.value
        sec = np.zeros(max(n, 1))
        byt = np.zeros(max(n, 1))
        kind = np.zeros(max(n, 1), dtype=np.int32)
        check(lib().qvdg_pass_times(self._h, as_double_ptr(sec), as_double_ptr(byt),
                                    kind.ctypes.data_as(ct.POINTER(ct.c_int32)), n, ct.byref(count)))
        return sec[:n], byt[:n], kind[:n]

    def max_abs_diff(self, other: "DeviceState") -> float:
        v = ct.c_double()
        check(lib().qvdg_max_abs_diff(self._h, other._h, ct.byref(v)))
        return v.value

    def device_buffer(self):
        p, n = ct.c_void_p(), ct.c_size_t()
        check(lib().qvdg_state_device_buffer(self._h, ct.byref(p), ct.byref(n)))
        return p.value, n.value

    def synchronize(self):
        check(lib().qvdg_synchronize(self._h))


class Plan:
    """A circuit fused, cut into stages and uploaded once (qvdg_plan), for
    states of `num_qubits` qubits in `precision_bits` precision."""

    def __init__(self, ops, num_qubits: int, precision_bits: int = 32, opts: QvdgOptions | None = None):
        packed = PackedOps(ops)
        self._h = ct.c_void_p()
        check(lib().qvdg_plan_create(int(num_qubits), int(precision_bits), packed.array, packed.count,
                                     ct.byref(opts) if opts else None, ct.byref(self._h)))
        self.num_qubits = int(num_qubits)
        self.precision_bits = int(precision_bits)

    def info(self) -> dict:
        stats = QvdgStats()
        check(lib().qvdg_plan_info(self._h, ct.byref(stats)))
        return stats.as_dict()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().qvdg_plan_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


ENTANGLERS = {"none": 0, "cx": 1, "cz": 2}


class Batch:
    """Many small layered circuits run to <Z_q> in one persistent,
    graph-captured launch (qvdg_batch). Each circuit is (num_qubits,
    gates, entangler): `gates` an array of shape (layers, num_qubits, 2, 2)
    complex, one 2x2 gate per qubit per layer, each layer followed by the
    entangler ladder ("cx", "cz" or "none") on (q, q+1), q = 0..n-2.
    `tile_qubits`/`threads` of 0 let the autotuner choose the launch shape."""

    def __init__(self, circuits, tile_qubits: int = 0, threads: int = 0):
        self._h = ct.c_void_p()
        arr = (QvdgLayeredCircuit * len(circuits))()
        self._keep = []
        self.widths = []
        for i, (n, gates, ent) in enumerate(circuits):
            g = np.ascontiguousarray(gates, dtype=np.complex128).reshape(-1)
            layers = g.size // (4 * n) if n else 0
            if g.size != layers * 4 * n:
                raise ValueError("gates must have shape (layers, num_qubits, 2, 2)")
            flat = g.view(np.float64)
            self._keep.append(flat)
            arr[i].num_qubits = int(n)
            arr[i].num_layers = int(layers)
            arr[i].entangler = ENTANGLERS[ent] if isinstance(ent, str) else int(ent)
            arr[i].gates = as_double_ptr(flat)
            self.widths.append(int(n))
        opts = QvdgBatchOptions(int(tile_qubits), int(threads))
        check(lib().qvdg_batch_create(arr, len(circuits), ct.byref(opts), ct.byref(self._h)))
        self._keep = None
        self.offsets = np.concatenate([[0], np.cumsum(self.widths)]).astype(np.int64)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().qvdg_batch_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self):
        """(<Z> of every qubit of every circuit as one flat array, device seconds)."""
        out = np.empty(max(int(self.offsets[-1]), 1), dtype=np.float64)
        sec = ct.c_double()
        check(lib().qvdg_batch_run(self._h, as_double_ptr(out), out.size, ct.byref(sec)))
        return out[:int(self.offsets[-1])], sec.value

    def split(self, flat) -> list:
        """Per-circuit arrays from run()'s flat output."""
        return [flat[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.widths))]

    def set_gates(self, gates_list):
        """New matrices for every circuit (same shapes as at creation)."""
        flat = np.concatenate([np.ascontiguousarray(g, dtype=np.complex128).reshape(-1) for g in gates_list])
        f = flat.view(np.float64)
        check(lib().qvdg_batch_set_gates(self._h, as_double_ptr(f), flat.size // 4))

    def info(self) -> dict:
        s = QvdgBatchSummary()
        check(lib().qvdg_batch_info(self._h, ct.byref(s)))
        return s.as_dict()

    def tuning(self):
        """[(tile_qubits, threads, sample seconds)] of every autotuned shape."""
        count = ct.c_size_t()
        check(lib().qvdg_batch_tuning(self._h, None, None, None, 0, ct.byref(count)))
        n = count.value
        t = (ct.c_uint32 * max(n, 1))()
        th = (ct.c_uint32 * max(n, 1))()
        s = (ct.c_double * max(n, 1))()
        check(lib().qvdg_batch_tuning(self._h, t, th, s, n, ct.byref(count)))
        return [(t[i], th[i], s[i]) for i in range(n)]
