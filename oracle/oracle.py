"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE, NOT PRODUCT CODE: a C++ restatement of the reference's
naive simulator (src/reference.rs) and of its fast AVX2 engine (kernels,
fusion, cache blocking, sampling; see oracle/engine.cpp for the file:line map).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs may import it, and only as the checker or the timed CPU
baseline. The product path never calls it.
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

from qevedo_simulator_b200._abi import PackedOps, QvdgOp, as_double_ptr, as_u64_ptr

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build() -> str:
    """Compile the oracle (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ct.CDLL(LIB_PATH)
        L.oracle_last_error.restype = ct.c_char_p
        L.oracle_sv_create.restype = ct.c_void_p
        L.oracle_sv_create.argtypes = [ct.c_uint32, ct.c_int]
        L.oracle_sv_destroy.argtypes = [ct.c_void_p]
        for name in ("oracle_sv_set_amplitudes", "oracle_sv_get_amplitudes"):
            getattr(L, name).argtypes = [ct.c_void_p, ct.POINTER(ct.c_double)]
        L.oracle_sv_apply_ops.argtypes = [ct.c_void_p, ct.POINTER(QvdgOp), ct.c_size_t, ct.c_uint32, ct.c_int,
                                          ct.POINTER(ct.c_uint64)]
        L.oracle_sv_apply.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double), ct.POINTER(ct.c_uint32), ct.c_uint32,
                                      ct.POINTER(ct.c_uint32), ct.POINTER(ct.c_uint8), ct.c_uint32]
        L.oracle_sv_norm_sqr.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double)]
        L.oracle_sv_probability_one.argtypes = [ct.c_void_p, ct.c_uint32, ct.POINTER(ct.c_double)]
        L.oracle_sv_measure.argtypes = [ct.c_void_p, ct.c_uint32, ct.c_double, ct.POINTER(ct.c_int32)]
        L.oracle_sv_sample_unordered.argtypes = [ct.c_void_p, ct.c_size_t, ct.POINTER(ct.c_double),
                                                 ct.POINTER(ct.c_uint64), ct.POINTER(ct.c_size_t)]
        L.oracle_sv_layout.argtypes = [ct.c_void_p, ct.POINTER(ct.c_uint32)]
        L.oracle_naive_apply.argtypes = [ct.POINTER(ct.c_double), ct.c_uint32, ct.POINTER(ct.c_double),
                                         ct.POINTER(ct.c_uint32), ct.c_uint32]
        L.oracle_naive_apply_op.argtypes = [ct.POINTER(ct.c_double), ct.c_uint32, ct.POINTER(QvdgOp)]
        L.oracle_fuse_shapes.argtypes = [ct.POINTER(QvdgOp), ct.c_size_t, ct.c_uint32, ct.POINTER(ct.c_size_t),
                                         ct.POINTER(ct.c_uint32), ct.c_size_t]
        L.oracle_sv_set_layout.argtypes = [ct.c_void_p, ct.POINTER(ct.c_uint32)]
        L.oracle_sv_set_physical.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int]
        L.oracle_sv_max_diff_physical.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int, ct.POINTER(ct.c_uint32),
                                                  ct.POINTER(ct.c_double)]
        L.oracle_set_threads.argtypes = [ct.c_int]
        L.oracle_max_threads.restype = ct.c_int
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise RuntimeError(lib().oracle_last_error().decode())


def set_threads(threads: int):
    lib().oracle_set_threads(int(threads))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# ----------------------------------------------------------- naive oracle
def naive_apply_ops(state: np.ndarray, ops) -> np.ndarray:
    """Apply ops one by one with the naive f64 simulator (reference.rs:8-29);
    controls become a controlled matrix on [controls..., targets...]."""
    state = np.array(state, dtype=np.complex128, copy=True)  # never modify the caller's array
    n = int(state.size).bit_length() - 1
    packed = PackedOps(ops)
    for i in range(packed.count):
        _check(lib().oracle_naive_apply_op(as_double_ptr(state.view(np.float64)), n, ct.byref(packed.array[i])))
    return state


def naive_statevector(ops, num_qubits: int, initial: np.ndarray | None = None) -> np.ndarray:
    """reference::statevector (reference.rs:33-44) on lowered ops."""
    if initial is None:
        state = np.zeros(1 << num_qubits, dtype=np.complex128)
        state[0] = 1.0
    else:
        state = np.array(initial, dtype=np.complex128)
    return naive_apply_ops(state, ops)


def fuse_shapes(ops, max_fused: int):
    """(targets, controls) per fused op from the restated greedy fuser."""
    packed = PackedOps(ops)
    n = ct.c_size_t()
    cap = 2 * max(len(ops), 1)
    widths = (ct.c_uint32 * cap)()
    _check(lib().oracle_fuse_shapes(packed.array, packed.count, max_fused, ct.byref(n), widths, cap))
    return [(widths[2 * i], widths[2 * i + 1]) for i in range(n.value)]


# ----------------------------------------------------------- fast engine
class OracleState:
    """The restated CPU engine's StateVector<f32|f64> (blocked layout)."""

    def __init__(self, num_qubits: int, precision_bits: int = 32):
        self.num_qubits = num_qubits
        self.precision_bits = precision_bits
        self._h = lib().oracle_sv_create(num_qubits, precision_bits)
        if not self._h:
            raise RuntimeError(lib().oracle_last_error().decode())

    def close(self):
        if self._h:
            lib().oracle_sv_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_amplitudes(self, amplitudes: np.ndarray):
        a = np.ascontiguousarray(amplitudes, dtype=np.complex128)
        assert a.size == 1 << self.num_qubits
        _check(lib().oracle_sv_set_amplitudes(self._h, as_double_ptr(a.view(np.float64))))

    def amplitudes(self) -> np.ndarray:
        out = np.empty(1 << self.num_qubits, dtype=np.complex128)
        _check(lib().oracle_sv_get_amplitudes(self._h, as_double_ptr(out.view(np.float64))))
        return out

    def apply_ops(self, ops, max_fused: int = 4, region_bits: int | None = 14) -> dict:
        packed = PackedOps(ops)
        stats = (ct.c_uint64 * 3)()
        rb = -1 if region_bits is None else int(region_bits)
        _check(lib().oracle_sv_apply_ops(self._h, packed.array, packed.count, max_fused, rb, stats))
        return {"gates": stats[0], "kernels": stats[1], "passes": stats[2]}

    def apply(self, matrix, qubits, controls=()):
        m = np.ascontiguousarray(matrix, dtype=np.complex128)
        q = np.array(qubits, dtype=np.uint32)
        cq = np.array([c for c, _ in controls] or [0], dtype=np.uint32)
        cv = np.array([1 if v else 0 for _, v in controls] or [0], dtype=np.uint8)
        _check(lib().oracle_sv_apply(self._h, as_double_ptr(m.view(np.float64)),
                                     q.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(qubits),
                                     cq.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                                     cv.ctypes.data_as(ct.POINTER(ct.c_uint8)), len(controls)))

    def norm_sqr(self) -> float:
        v = ct.c_double()
        _check(lib().oracle_sv_norm_sqr(self._h, ct.byref(v)))
        return v.value

    def probability_one(self, qubit: int) -> float:
        v = ct.c_double()
        _check(lib().oracle_sv_probability_one(self._h, qubit, ct.byref(v)))
        return v.value

    def measure(self, qubit: int, uniform: float) -> int:
        v = ct.c_int32()
        _check(lib().oracle_sv_measure(self._h, qubit, float(uniform), ct.byref(v)))
        return v.value

    def sample_unordered(self, uniforms: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.empty(max(u.size, 1), dtype=np.uint64)
        count = ct.c_size_t()
        _check(lib().oracle_sv_sample_unordered(self._h, u.size, as_double_ptr(u), as_u64_ptr(out), ct.byref(count)))
        return out[:count.value]

    def layout(self):
        out = (ct.c_uint32 * max(self.num_qubits, 1))()
        _check(lib().oracle_sv_layout(self._h, out))
        return list(out)[: self.num_qubits]

    def set_layout(self, layout):
        """layout[logical] = physical, without moving amplitudes."""
        arr = (ct.c_uint32 * max(self.num_qubits, 1))(*[int(q) for q in layout])
        _check(lib().oracle_sv_set_layout(self._h, arr))

    def set_physical(self, physical: np.ndarray):
        """Load interleaved amplitudes in physical order (complex64 or
        complex128), as another engine holds them in memory."""
        a = _physical_array(physical, self.num_qubits)
        _check(lib().oracle_sv_set_physical(self._h, a.ctypes.data_as(ct.c_void_p), _bits_of(a)))

    def max_diff_physical(self, physical: np.ndarray, layout) -> float:
        """max |this amplitude - the other's| over logical indices, the other
        state given in physical order with its layout."""
        a = _physical_array(physical, self.num_qubits)
        arr = (ct.c_uint32 * max(self.num_qubits, 1))(*[int(q) for q in layout])
        v = ct.c_double()
        _check(lib().oracle_sv_max_diff_physical(self._h, a.ctypes.data_as(ct.c_void_p), _bits_of(a), arr,
                                                 ct.byref(v)))
        return v.value


def _bits_of(a: np.ndarray) -> int:
    return 32 if a.dtype == np.complex64 else 64


def _physical_array(physical: np.ndarray, num_qubits: int) -> np.ndarray:
    a = np.ascontiguousarray(physical)
    if a.dtype not in (np.complex64, np.complex128):
        raise TypeError("expected complex64 or complex128 amplitudes")
    if a.size != 1 << num_qubits:
        raise ValueError(f"expected {1 << num_qubits} amplitudes")
    return a


def sample_physical(physical: np.ndarray, layout, uniforms: np.ndarray) -> np.ndarray:
    """The reference sampler on a state given as it lies in another engine's
    memory: physical-order amplitudes (complex64 -> a 32-bit state,
    complex128 -> 64-bit) with layout[logical] = physical, so chunks are
    summed in the same physical order; outcomes are logical indices."""
    n = int(physical.size).bit_length() - 1
    st = OracleState(n, _bits_of(np.asarray(physical)))
    try:
        st.set_layout(layout)
        st.set_physical(physical)
        return st.sample_unordered(uniforms)
    finally:
        st.close()


def sample_from_amplitudes(amplitudes: np.ndarray, uniforms: np.ndarray, precision_bits: int) -> np.ndarray:
    """The reference sampler (measure.rs:104-174) on a given logical amplitude
    array, held in `precision_bits` precision with the identity layout."""
    n = int(amplitudes.size).bit_length() - 1
    st = OracleState(n, precision_bits)
    try:
        st.set_amplitudes(amplitudes)
        return st.sample_unordered(uniforms)
    finally:
        st.close()
