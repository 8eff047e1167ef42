"""The allocation-free entry point, qvdg_bit_probabilities_noalloc.

It serves callers that cannot let the library allocate device memory (the
state vector already fills the GPU, or another allocator owns the memory):
it computes the per-qubit probabilities of a state held in the caller's
device buffer with a fixed scratch array built into the library. These
tests call it through the C ABI on the device buffer of a state made by the
regular API and compare it with the regular entry points that allocate
their workspace (qvdg_expect_z_all, qvdg_probability_one, qvdg_norm_sqr),
twice in a row, since every call reuses the same scratch array.

The file name makes pytest collect it last.
"""

import numpy as np
import pytest

from qevedo_simulator_b200 import DeviceState, _native, library, options

pytestmark = pytest.mark.gpu

# Both paths reduce in double precision; the per-bit sums run the same
# kernel, the norm a different summation order.
REL_TOL = 1e-12


def _prepared_state(n, bits, seed):
    st = DeviceState(n, bits)
    st.apply_ops(library.random_grid_circuit(*library.grid_shape(n), 8, seed=seed).ops(), options(4, True))
    st.synchronize()
    assert st.layout() == list(range(n))  # the buffer is in logical order
    return st


def _check_against_regular_entry_points(st):
    ptr, nbytes = st.device_buffer()
    assert nbytes == (1 << st.num_qubits) * (8 if st.precision_bits == 32 else 16)
    p1, total = _native.bit_probabilities_noalloc(ptr, st.num_qubits, st.precision_bits)
    assert total == pytest.approx(st.norm_sqr(), rel=REL_TOL)
    z = st.expect_z_all()
    np.testing.assert_allclose(total - 2.0 * p1, z, rtol=0, atol=REL_TOL * total)
    for q in (0, st.num_qubits // 2, st.num_qubits - 1):
        assert p1[q] == pytest.approx(st.probability_one(q), rel=REL_TOL, abs=REL_TOL * total)
    return p1, total


@pytest.mark.parametrize("n,bits", [(20, 32), (16, 64), (7, 32)])
def test_matches_the_allocating_entry_points_twice_in_a_row(n, bits):
    with _prepared_state(n, bits, seed=n) as a, _prepared_state(n, bits, seed=n + 100) as b:
        pa, ta = _check_against_regular_entry_points(a)
        pb, tb = _check_against_regular_entry_points(b)
        assert not np.array_equal(pa, pb)  # the second call saw the second state
        # A third call on the first state reproduces the first exactly.
        ptr, _ = a.device_buffer()
        again, t_again = _native.bit_probabilities_noalloc(ptr, n, bits)
        assert np.array_equal(again, pa) and t_again == ta


def test_states_beyond_the_limit_are_refused():
    with DeviceState(8, 32) as st:
        ptr, _ = st.device_buffer()
        # Rejected on the host before any device work (the buffer is small).
        with pytest.raises(_native.QvdgError, match="35 qubits"):
            _native.bit_probabilities_noalloc(ptr, 36, 32)
        with pytest.raises(ValueError, match="precision"):
            _native.bit_probabilities_noalloc(ptr, 8, 16)
