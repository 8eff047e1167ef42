"""The sharded state vector's host logic on CPU: 2 and 4 gloo ranks on
127.0.0.1, each with a local engine built on the oracle's naive f64 apply
(reference.rs:8-29) in place of its GPU, run circuits whose ops touch the
global qubits (exchanges of half states between ranks, controls and
diagonals on global qubits resolved per rank). The gathered state must
equal the oracle's single-process run of the same ops."""

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleEngine:
    """A rank's local state as a numpy array in physical = logical order,
    ops applied by the oracle's naive simulator."""

    def __init__(self, n):
        self.n = n
        self.a = np.zeros(1 << n, dtype=np.complex128)

    def zero(self, one):
        self.a[:] = 0
        if one:
            self.a[0] = 1

    def apply_ops(self, ops, opts=None):
        from oracle import oracle

        self.a = oracle.naive_apply_ops(self.a, ops)

    def layout(self):
        return list(range(self.n))

    def read_half(self, p, v):
        return self.a.reshape(-1, 2, 1 << p)[:, v, :].copy()

    def write_half(self, p, v, data):
        self.a.reshape(-1, 2, 1 << p)[:, v, :] = data.numpy().view(np.complex128).reshape(-1, 1 << p)

    def norm_sqr(self):
        return float(np.sum(np.abs(self.a) ** 2))

    def probability_one(self, i):
        sel = (np.arange(self.a.size) >> i) & 1
        return float(np.sum(np.abs(self.a[sel == 1]) ** 2))

    def amplitudes(self):
        return self.a.copy()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _circuit(n, seed):
    """Mixed layers (Haar SU(2) per qubit, CZ/CX/iSWAP pairs, a phase gate,
    an X with 1-3 controls) plus ops aimed at the top qubits: a dense 3-qubit
    unitary on them, a diagonal on two of them and one low qubit, a phase
    on the top qubit controlled by a low one."""
    from qevedo_simulator_b200 import Op, library

    ops = library.mixed_ops(n, 4, seed=seed)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    u = np.linalg.qr(rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8)))[0]
    ops.append(Op([n - 1, 0, n - 2], [], u))
    ops.append(Op([n - 1, n - 2, 1], [], np.diag(np.exp(1j * rng.uniform(0, 6.3, 8)))))
    ops.append(Op([n - 1], [(2, True)], np.diag([1.0, np.exp(0.7j)])))
    ops.append(Op([0], [(n - 1, True), (n - 2, False)], np.array([[0, 1], [1, 0]], dtype=np.complex128)))
    # diagonals whose targets may all be global: a phase per rank, with and
    # without a local control
    ops.append(Op([n - 1], [], np.diag([np.exp(-0.3j), np.exp(0.3j)])))
    ops.append(Op([n - 2, n - 1], [(0, False)], np.diag(np.exp(1j * np.array([0.1, 0.5, 0.9, 1.3])))))
    ops.append(Op([n - 1, n - 2], [(0, True), (1, True)], np.diag(np.exp(1j * np.array([0.2, 0.4, 0.6, 0.8])))))
    ops.extend(library.mixed_ops(n, 1, seed=seed + 2))
    return ops


def _global_diagonals(global_q, local_q):
    from qevedo_simulator_b200 import Op

    g, l0, l1 = global_q[-1], local_q[0], local_q[1]
    ops = [Op([g], [], np.diag([np.exp(-0.3j), np.exp(0.3j)])),
           Op([g], [(l0, True)], np.diag([np.exp(0.2j), np.exp(-0.5j)])),
           Op([l1, g], [(l0, False)], np.diag(np.exp(1j * np.array([0.1, 0.5, 0.9, 1.3]))))]
    if len(global_q) > 1:
        ops.append(Op([global_q[0], g], [(l1, True)], np.diag(np.exp(1j * np.array([0.2, 0.4, 0.6, 0.8])))))
        ops.append(Op([l0], [(global_q[0], True)], np.array([[0, 1], [1, 0]], dtype=np.complex128)))
    return ops


def _rank(rank, world, port, n, seed, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from qevedo_simulator_b200.sharded import ShardedStateVector
    from test_sharded import OracleEngine, _circuit, _global_diagonals

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        k = world.bit_length() - 1
        sv = ShardedStateVector(n, engine=OracleEngine(n - k))
        ops = _circuit(n, seed)
        info = sv.apply_ops(ops)
        # Diagonals on the qubits that are global now (every rank knows the
        # same placement): phases per rank, with and without local controls.
        more = _global_diagonals(sv.global_q, sv.local_q)
        after = sv.apply_ops(more)
        assert after["exchanges"] == 0
        amps = sv.amplitudes()
        out.put((rank, amps, info, sv.norm_sqr(), sv.probability_one(n - 1), sv.probability_one(0), more))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 8), (4, 9)])
def test_sharded_state_matches_the_oracle(world, n):
    from oracle import oracle

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, 11 + world, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted((out.get(timeout=180) for _ in range(world)), key=lambda g: g[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    more = got[0][6]
    ref = oracle.naive_statevector(_circuit(n, 11 + world) + more, n)
    for rank, amps, info, norm, p_top, p_low, _ in got:
        assert np.abs(amps - ref).max() < 1e-12, rank
        assert info["exchanges"] >= 1  # the ops on the top qubits moved them
        assert abs(norm - 1.0) < 1e-12
        prob = np.abs(ref) ** 2
        idx = np.arange(ref.size)
        assert abs(p_top - prob[(idx >> (n - 1)) & 1 == 1].sum()) < 1e-12
        assert abs(p_low - prob[idx & 1 == 1].sum()) < 1e-12
    # every rank tracks the same placement, so all gathered the same state
    assert all(np.array_equal(g[1], got[0][1]) for g in got)
