"""The C-ABI library loads and exports every entry point include/*.h
declares (no device calls: these run without a GPU)."""

import ctypes as ct
import glob
import os
import re

from qevedo_simulator_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(qvdg_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    lib = ct.CDLL(_native.LIBRARY)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert declared_functions() <= set(_native._SIGNATURES)


def test_host_only_calls_need_no_device():
    lib = _native.lib()
    assert lib.qvdg_version().decode().startswith("qvdgpu")
    o = _native.options()
    lib.qvdg_default_options(ct.byref(o))
    assert o.max_fused_qubits == 4 and o.staged == 1
    # Invalid arguments are rejected before any device work, with a message.
    h = ct.c_void_p()
    assert lib.qvdg_state_create(10, 16, ct.byref(h)) == 1
    assert "precision" in lib.qvdg_last_error().decode()
    assert lib.qvdg_state_destroy(None) == 0
    assert lib.qvdg_norm_sqr(None, None) == 1
    n = ct.c_size_t(99)
    assert lib.qvdg_plan_features_from(50, 32, None, 0, None, 1, None, 0, ct.byref(n)) == 1
    assert "qubits" in lib.qvdg_last_error().decode()
    assert lib.qvdg_plan_features_from(4, 32, None, 0, None, 1, None, 0, ct.byref(n)) == 0 and n.value == 0


def test_batch_validation_needs_no_device():
    """Invalid batches are refused before any device work."""
    import numpy as np

    from qevedo_simulator_b200._abi import QvdgLayeredCircuit, as_double_ptr

    lib = _native.lib()
    g = np.zeros(8 * 25, dtype=np.float64)
    arr = (QvdgLayeredCircuit * 1)()
    arr[0].num_qubits, arr[0].num_layers, arr[0].entangler = 25, 1, 1
    arr[0].gates = as_double_ptr(g)
    h = ct.c_void_p()
    assert lib.qvdg_batch_create(arr, 1, None, ct.byref(h)) == 1
    assert "num_qubits" in lib.qvdg_last_error().decode()
    arr[0].num_qubits, arr[0].entangler = 3, 9
    assert lib.qvdg_batch_create(arr, 1, None, ct.byref(h)) == 1
    assert "entangler" in lib.qvdg_last_error().decode()
    assert lib.qvdg_batch_create(arr, 0, None, ct.byref(h)) == 1
    assert lib.qvdg_batch_destroy(None) == 0


def test_one_pass_gate_packing_equals_packing_the_ops():
    """run() packs a circuit's gate instructions for the C ABI in one pass;
    the arrays equal those of packing gate_op's ops (same counts, qubits,
    control values, matrices and layout)."""
    import numpy as np

    from qevedo_simulator_b200 import library
    from qevedo_simulator_b200._abi import PackedOps
    from qevedo_simulator_b200.circuit import gate_op, packed_gate_ops

    from qevedo_simulator_b200 import Circuit, Gate
    from qevedo_simulator_b200.circuit import _CONTROLLED

    rng = np.random.Generator(np.random.PCG64(8))
    every = Circuit(5)
    for name, (controls, _) in sorted(_CONTROLLED.items()):
        arity = controls + (2 if name == "cswap" else 1)
        params = (0.37,) if name in ("cp", "crx", "cry", "crz") else ()
        every._instructions.append(("gate", Gate(name, params),
                                    [int(q) for q in rng.permutation(5)[:arity]]))
    q = np.linalg.qr(rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8)))[0]
    u2 = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))[0]
    every.unitary(q, [4, 0, 2]).unitary(u2, [3])
    for c in (library.random_grid_circuit(3, 4, 6, 3), library.qft(9), library.random_gate_circuit(8, 200, 5),
              library.ghz(5), every):
        ins = c._instructions
        a = PackedOps([gate_op(i[1], i[2]) for i in ins if i[0] == "gate"])
        b = packed_gate_ops(ins)
        assert a.count == b.count
        for x, y in ((a._q, b._q), (a._v, b._v), (a._m, b._m)):
            assert np.array_equal(x, y)
        for f, base in (("targets", "_q"), ("controls", "_q"), ("control_values", "_v"), ("matrix", "_m")):
            assert np.array_equal(a._ops[f] - np.uint64(getattr(a, base).ctypes.data),
                                  b._ops[f] - np.uint64(getattr(b, base).ctypes.data)), f
        for f in ("num_targets", "num_controls"):
            assert np.array_equal(a._ops[f], b._ops[f]), f


def test_rust_bindings_mirror_the_header():
    """rust/src/gpu/ffi.rs (the seam a qvd maintainer adds; not compiled in
    this image, which has no Rust toolchain) declares every function of the
    header and the same struct fields in the same order."""
    text = open(os.path.join(ROOT, "rust", "src", "gpu", "ffi.rs")).read()
    assert set(re.findall(r"pub fn (qvdg_[a-z0-9_]+)\(", text)) == declared_functions()
    header = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "qvdg.h")).read(), flags=re.S)
    for body, name in re.findall(r"typedef struct \{(.*?)\} (\w+);", header, flags=re.S):
        c_fields = re.findall(r"(\w+);", body)
        m = re.search(r"pub struct " + name + r" \{(.*?)\n\}", text, flags=re.S)
        assert m, name
        assert re.findall(r"pub (\w+):", m.group(1)) == c_fields, name
