"""The learned planner's host side (no device work): its candidate settings
are the cost model's, `run` and `statevector` default to it and plan
greedily as soon as a caller gives settings, and the reference's argument
checks (threads, circuit type) hold."""

import pytest

from qevedo_simulator_b200 import _native, costmodel, simulator
from qevedo_simulator_b200._abi import settings_dict


def test_candidates_match_the_cost_model_list():
    names = [name for name, _ in costmodel.candidates()]
    c32 = [settings_dict(o) for o in _native.planner_candidates(32)]
    assert c32 == [settings_dict(o) for _, o in costmodel.candidates()], names
    c64 = [settings_dict(o) for o in _native.planner_candidates(64)]
    assert c64 == [c for c in c32 if c["math"] not in ("tensor", "tensor_pairs")]
    assert all(o.planner == _native.PLANNERS["greedy"] for o in _native.planner_candidates(32))


def test_default_settings_use_the_learned_planner():
    o = simulator.plan_options()
    assert o.planner == _native.PLANNERS["learned"]
    # the fallback for complex128 / no model: the reference defaults
    assert (o.max_fused_qubits, o.staged, o.math) == (4, 1, 0)
    for given in ({"max_fused_qubits": 6}, {"staged": False}, {"math": "tensor"}):
        assert simulator.plan_options(**given).planner == _native.PLANNERS["greedy"], given
    assert simulator.plan_options(planner="learned", math="tensor").planner == _native.PLANNERS["learned"]
    with pytest.raises(ValueError, match="planner"):
        simulator.plan_options(planner="fastest")


def test_reference_argument_checks():
    for ok in (None, 0, 1, 8, "pcores", "pthreads", "cores", "allcores", "all"):
        simulator._check_threads(ok)
    with pytest.raises(ValueError, match="unknown thread placement `core`"):
        simulator._check_threads("core")
    for bad in (-1, 2.5, [1]):
        with pytest.raises(ValueError, match="number or a placement name"):
            simulator._check_threads(bad)
    with pytest.raises(TypeError, match="Circuit or OpenQASM"):
        simulator._as_circuit(42)
    with pytest.raises(ValueError, match="precision"):
        simulator._precision_bits("half")
    simulator._check_backend("state_vector")
    with pytest.raises(ValueError, match="not part of"):
        simulator._check_backend("mps")
