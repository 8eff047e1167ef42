"""The sharded state vector with its GPU engine on one B200: two or four
ranks as host threads of one process, each with its own device state
(n - k qubits) on the same GPU, trading half states through in-process
queues instead of NCCL. No kernel waits for another rank: the ranks meet
only on the host, between launches. Checks the device engine's strided
half copies, and the gathered state against the oracle's naive f64 run."""

import queue
import threading

import numpy as np
import pytest

from test_sharded import _circuit

pytestmark = pytest.mark.gpu


class ThreadTransport:
    """Ranks as threads: pairwise exchange through queues, sums and gathers
    through a barrier."""

    def __init__(self, rank, world, boxes, barrier, slots):
        self.rank, self.world = rank, world
        self.boxes, self.barrier, self.slots = boxes, barrier, slots

    def sendrecv(self, send, partner):
        self.boxes[(self.rank, partner)].put(send.clone())
        return self.boxes[(partner, self.rank)].get(timeout=120)

    def _all(self, value):
        self.barrier.wait(timeout=120)
        self.slots[self.rank] = value
        self.barrier.wait(timeout=120)
        out = list(self.slots)
        self.barrier.wait(timeout=120)
        return out

    def sum(self, x):
        return float(sum(self._all(float(x))))

    def gather(self, a):
        return [t.cpu() for t in self._all(a.clone())]


def test_device_engine_half_copies():
    """read_half / write_half move exactly the amplitudes whose physical bit
    p is v (strided 2D device copies), for low, middle and top bits."""
    import torch

    from qevedo_simulator_b200.sharded import DeviceEngine

    n = 12
    rng = np.random.Generator(np.random.PCG64(5))
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    for bits in (32, 64):
        eng = DeviceEngine(n, bits)
        try:
            eng.state.set_amplitudes(a)
            ctype = np.complex64 if bits == 32 else np.complex128
            ref = a.astype(ctype)
            for p in (0, 3, n - 1):
                for v in (0, 1):
                    half = eng.read_half(p, v).cpu().numpy().view(ctype)
                    assert np.array_equal(half, ref.reshape(-1, 2, 1 << p)[:, v, :].reshape(-1)), (bits, p, v)
            new = (rng.standard_normal(1 << (n - 1)) + 1j * rng.standard_normal(1 << (n - 1))).astype(ctype)
            real = torch.from_numpy(new.view(np.float32 if bits == 32 else np.float64).copy()).cuda()
            eng.write_half(5, 1, real)
            ref.reshape(-1, 2, 32)[:, 1, :] = new.reshape(-1, 32)
            got = eng.amplitudes()
            assert np.abs(got - ref).max() < (1e-6 if bits == 32 else 1e-15)
        finally:
            eng.close()


@pytest.mark.parametrize("world,n,bits", [(2, 14, 64), (4, 15, 64), (2, 14, 32)])
def test_threaded_ranks_match_the_oracle(world, n, bits):
    from oracle import oracle
    from qevedo_simulator_b200.sharded import DeviceEngine, ShardedStateVector

    k = world.bit_length() - 1
    boxes = {(a, b): queue.Queue() for a in range(world) for b in range(world)}
    barrier = threading.Barrier(world)
    slots = [None] * world
    results, errors = [None] * world, []
    ops = _circuit(n, 3 + world)

    def rank(r):
        try:
            tr = ThreadTransport(r, world, boxes, barrier, slots)
            sv = ShardedStateVector(n, bits, engine=DeviceEngine(n - k, bits), transport=tr)
            try:
                info = sv.apply_ops(ops)
                results[r] = (sv.amplitudes(), info, sv.norm_sqr())
            finally:
                sv.close()
        except Exception as e:  # reported below
            errors.append(repr(e))
            barrier.abort()

    threads = [threading.Thread(target=rank, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(300)
    assert not errors, errors
    ref = oracle.naive_statevector(ops, n)
    tol = 1e-12 if bits == 64 else 2e-5
    for amps, info, norm in results:
        assert info["exchanges"] >= 1
        assert np.abs(amps - ref).max() < tol
        assert abs(norm - 1.0) < (1e-12 if bits == 64 else 1e-5)
