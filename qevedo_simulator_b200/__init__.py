"""B200-native state-vector engine for the qvd quantum circuit simulator.

A drop-in for the reference's state-vector backend: the same circuit model
and gate conventions (Qiskit's), `run` and `statevector` with the same
meaning, and a device-resident `DeviceState` with the reference
StateVector's methods. The hot path is hand-written sm_100a CUDA in
libqvdgpu.so behind the C ABI of include/qvdg.h; there is no CPU fallback.

    >>> from qevedo_simulator_b200 import Circuit, run
    >>> bell = Circuit(2).h(0).cx(0, 1).measure_all()
    >>> sorted(run(bell, shots=1000, seed=1).counts)
    ['00', '11']
"""

from . import library, qasm
from ._native import Batch, DeviceState, Plan, QvdgError, options, set_device
from .sharded import ShardedStateVector
from .circuit import Circuit, Gate, Op, gate_op
from .simulator import RunResult, count_outcomes, estimate, run, statevector

__all__ = ["Batch", "Circuit", "Gate", "Op", "gate_op", "DeviceState", "Plan", "QvdgError", "options", "set_device", "RunResult", "run",
           "statevector", "count_outcomes", "estimate", "library", "qasm", "ShardedStateVector"]
__version__ = "0.1.0"
