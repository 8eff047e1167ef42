import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def max_distance(a, b) -> float:
    """tests/common/mod.rs:65-71: the largest |a_i - b_i|."""
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    return float(np.max(np.abs(a - b))) if a.size else 0.0


# ---- random inputs in the manner of tests/common/mod.rs:12-63 (own seeds)
def random_unitary(rng: np.random.Generator, qubits: int) -> np.ndarray:
    """Gram-Schmidt on a random complex matrix (tests/common/mod.rs:12-37)."""
    dim = 1 << qubits
    columns = []
    while len(columns) < dim:
        v = (rng.random(dim) - 0.5) + 1j * (rng.random(dim) - 0.5)
        for u in columns:
            v = v - np.vdot(u, v) * u
        norm = np.sqrt(np.sum(np.abs(v) ** 2))
        if norm > 1e-6:
            columns.append(v / norm)
    return np.array(columns).T.copy()


def random_diagonal(rng: np.random.Generator, qubits: int) -> np.ndarray:
    phases = rng.random(1 << qubits) * 2 * np.pi
    return np.diag(np.cos(phases) + 1j * np.sin(phases))


def random_state(rng: np.random.Generator, qubits: int) -> np.ndarray:
    v = (rng.random(1 << qubits) - 0.5) + 1j * (rng.random(1 << qubits) - 0.5)
    return v / np.sqrt(np.sum(np.abs(v) ** 2))


def random_qubits(rng: np.random.Generator, n: int, k: int) -> list:
    allq = list(range(n))
    for i in range(k):
        j = int(rng.integers(i, n))
        allq[i], allq[j] = allq[j], allq[i]
    return allq[:k]


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.lib()
    return o


def device_physical(st) -> np.ndarray:
    """A device state's amplitudes as they lie in HBM: physical index order,
    in the state's own precision (complex64 or complex128), copied with the
    CUDA runtime after the library's stream has drained."""
    from cuda.bindings import runtime as rt

    st.synchronize()
    ptr, nbytes = st.device_buffer()
    dtype = np.complex64 if st.precision_bits == 32 else np.complex128
    out = np.empty(1 << st.num_qubits, dtype=dtype)
    assert nbytes >= out.nbytes
    (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess, err
    return out
