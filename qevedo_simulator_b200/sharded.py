"""A state vector spread over several GPUs (one process per GPU).

The reference runs on one machine's memory; its research notes sketch the
published way past it (research_notes/Fastest quantum circuit simulator
design/fusion_and_cache_blocking.md:98-105: swap global qubits with local
ones, resolve controlled and diagonal gates on global qubits per rank).
Here a 2^n-amplitude state lives on
N = 2^k ranks: the k highest index bits ("global" qubits) pick the rank, the
other n - k ("local" qubits) index the rank's own device state, a
`DeviceState` of n - k qubits. A rank holds the amplitudes whose global bits
equal its rank.

Applying ops:

- an op whose targets are all local runs on every rank's local state, with
  its controls on global qubits resolved per rank (a rank whose global bits
  do not match skips it) and a diagonal op's global targets fixed to the
  rank's bits (the diagonal restricted to them);
- an op with a global target first swaps that qubit with a local qubit it
  does not touch (chosen among the qubits the next ops need least, on a
  high physical bit where possible): for global bit j and local physical
  bit p, rank r keeps the half of its amplitudes whose bit p equals bit j
  of r and exchanges the other half with rank r ^ 2^j (one send and one
  receive of half the local state: NCCL between GPUs, gloo on CPUs, or any
  transport with the same three calls);
- local ops between two exchanges go to the local engine as one batch, so
  it plans and fuses them as usual.

The local engine is the device state by default. It can be any object with
the engine methods below (`zero`, `apply_ops`, `layout`, `read_half`,
`write_half`, `norm_sqr`, `probability_one`, `amplitudes`), which is how the
CPU tests run the exchange logic between gloo ranks.
"""

from __future__ import annotations

import numpy as np

from . import _native
from .circuit import Op


class DeviceEngine:
    """A rank's local state on its GPU (the product engine). Halves move
    between the state's device buffer and torch tensors (the transport's
    buffers) with 2D device copies."""

    def __init__(self, num_qubits: int, precision_bits: int = 32):
        self.n = num_qubits
        self.bits = precision_bits
        self.state = _native.DeviceState(num_qubits, precision_bits)

    def close(self):
        self.state.close()

    def zero(self, one: bool):
        self.state.zero()
        if not one:
            from cuda.bindings import runtime as rt

            ptr, nbytes = self.state.device_buffer()
            (err,) = rt.cudaMemset(ptr, 0, nbytes)
            _check_cuda(err, "cudaMemset")

    def apply_ops(self, ops, opts=None):
        return self.state.apply_ops(ops, opts)

    def layout(self) -> list:
        return list(self.state.layout())

    def _half_geometry(self, p: int, v: int):
        esize = 8 if self.bits == 32 else 16
        width = (1 << p) * esize
        rows = 1 << (self.n - p - 1)
        ptr, _ = self.state.device_buffer()
        return int(ptr) + v * width, width, rows

    def read_half(self, p: int, v: int):
        """The amplitudes whose physical bit p is v, in index order, as a
        real torch tensor on the device (interleaved re/im)."""
        import torch
        from cuda.bindings import runtime as rt

        self.state.synchronize()
        src, width, rows = self._half_geometry(p, v)
        dtype = torch.float32 if self.bits == 32 else torch.float64
        out = torch.empty(rows * width // (4 if self.bits == 32 else 8), dtype=dtype, device="cuda")
        (err,) = rt.cudaMemcpy2D(out.data_ptr(), width, src, 2 * width, width, rows,
                                 rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
        _check_cuda(err, "cudaMemcpy2D")
        return out

    def write_half(self, p: int, v: int, data):
        import torch
        from cuda.bindings import runtime as rt

        torch.cuda.current_stream().synchronize()
        dst, width, rows = self._half_geometry(p, v)
        (err,) = rt.cudaMemcpy2D(dst, 2 * width, data.data_ptr(), width, width, rows,
                                 rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
        _check_cuda(err, "cudaMemcpy2D")

    def norm_sqr(self) -> float:
        return float(self.state.norm_sqr())

    def probability_one(self, i: int) -> float:
        """The squared norm of the amplitudes with local qubit i = 1 (not
        normalised, as the reference's probability_one)."""
        return float(self.state.probability_one(i))

    def amplitudes(self) -> np.ndarray:
        return self.state.amplitudes()


def _check_cuda(err, what: str):
    from cuda.bindings import runtime as rt

    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"{what} failed: {err}")


def _is_diagonal(m: np.ndarray) -> bool:
    return bool(np.count_nonzero(m - np.diag(np.diag(m))) == 0)


class DistTransport:
    """The ranks of a torch.distributed group (NCCL between GPUs, gloo on
    CPUs): pairwise exchange, sum and gather."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def _device(self):
        return "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"

    def sendrecv(self, send, partner: int):
        """Send `send` to `partner` and return what it sent back."""
        import torch

        recv = torch.empty_like(send)
        peer = partner if self.group is None else self.dist.get_global_rank(self.group, partner)
        ops = [self.dist.P2POp(self.dist.isend, send, peer, self.group),
               self.dist.P2POp(self.dist.irecv, recv, peer, self.group)]
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        if recv.is_cuda:
            torch.cuda.current_stream().synchronize()
        return recv

    def sum(self, x: float) -> float:
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def gather(self, a):
        """Every rank's float64 tensor `a` (same size), in rank order."""
        import torch

        a = a.to(self._device())
        parts = [torch.empty_like(a) for _ in range(self.world)]
        self.dist.all_gather(parts, a, group=self.group)
        return [t.cpu() for t in parts]


class ShardedStateVector:
    """An n-qubit state over the ranks of a transport (by default the
    torch.distributed group: a power of two of ranks, each with its own
    GPU), starting in |0...0>. Under NCCL each rank first selects its GPU
    for torch and for the library (`torch.cuda.set_device(local_rank)`,
    `qevedo_simulator_b200.set_device(local_rank)`).

        >>> sv = ShardedStateVector(36)          # 4 ranks: 2^34 amplitudes each
        >>> sv.apply_ops(circuit.ops())          # {'exchanges': ..., 'batches': ...}
        >>> sv.probability_one(35), sv.norm_sqr()
    """

    def __init__(self, num_qubits: int, precision_bits: int = 32, group=None, engine=None, lookahead: int = 32,
                 transport=None):
        self.transport = transport if transport is not None else DistTransport(group)
        self.world = self.transport.world
        self.rank = self.transport.rank
        k = self.world.bit_length() - 1
        if self.world != 1 << k:
            raise ValueError("the number of ranks must be a power of two")
        if num_qubits - k < 1:
            raise ValueError("each rank needs at least one local qubit")
        self.n, self.k, self.local_n = num_qubits, k, num_qubits - k
        self.lookahead = lookahead
        self.engine = engine if engine is not None else DeviceEngine(self.local_n, precision_bits)
        self.exchanges = 0
        self.zero()

    def close(self):
        if hasattr(self.engine, "close"):
            self.engine.close()

    # --- placement -------------------------------------------------------
    def zero(self):
        """|0...0>: amplitude 1 on rank 0, local index 0; logical qubit q on
        local index q (q < n - k) or global bit q - (n - k)."""
        self.local_q = list(range(self.local_n))  # local index -> logical qubit
        self.global_q = list(range(self.local_n, self.n))  # global bit -> logical qubit
        self.engine.zero(self.rank == 0)

    def _where(self, q: int):
        if q in self.local_q:
            return "l", self.local_q.index(q)
        return "g", self.global_q.index(q)

    def _global_bit(self, j: int) -> int:
        return (self.rank >> j) & 1

    # --- exchange --------------------------------------------------------
    def _exchange(self, j: int, i: int):
        """Swap global bit j with local index i (physical bit p of the local
        state): keep the half whose bit p equals this rank's bit j, trade the
        other half with the rank that differs in bit j."""
        import torch

        p = self.engine.layout()[i]
        b = self._global_bit(j)
        partner = self.rank ^ (1 << j)
        send = self.engine.read_half(p, 1 - b)
        if not isinstance(send, torch.Tensor):
            send = np.ascontiguousarray(send)
            send = torch.from_numpy(send.view(np.float64) if np.iscomplexobj(send) else send)
        self.engine.write_half(p, 1 - b, self.transport.sendrecv(send, partner))
        self.local_q[i], self.global_q[j] = self.global_q[j], self.local_q[i]
        self.exchanges += 1

    def _victim(self, op_qubits: set, upcoming) -> int:
        """The local index to trade for a global qubit: one the op does not
        touch, used latest by the next ops, on the highest physical bit among
        equals (its halves are long contiguous runs)."""
        layout = self.engine.layout()
        best, key = None, None
        for i, q in enumerate(self.local_q):
            if q in op_qubits:
                continue
            nxt = next((d for d, o in enumerate(upcoming) if q in o.qubits()), len(upcoming))
            k = (nxt, layout[i])
            if key is None or k > key:
                best, key = i, k
        if best is None:
            raise ValueError("an op touches more qubits than a rank holds locally")
        return best

    # --- ops -------------------------------------------------------------
    def _localize(self, op: Op):
        """The op on local indices for this rank, or None where it is the
        identity here (a global control that does not match). Its global
        targets must be fixed by now (diagonal ops only)."""
        controls = []
        for q, v in op.controls:
            kind, idx = self._where(q)
            if kind == "g":
                if self._global_bit(idx) != int(v):
                    return None
            else:
                controls.append((idx, v))
        targets, fixed = [], []
        for pos, q in enumerate(op.targets):
            kind, idx = self._where(q)
            if kind == "g":
                fixed.append((pos, self._global_bit(idx)))
            else:
                targets.append((pos, idx))
        matrix = np.asarray(op.matrix, dtype=np.complex128)
        if fixed:
            # A diagonal op: keep the entries whose global target bits are
            # this rank's.
            diag = np.diag(matrix)
            keep = []
            for e in range(1 << len(targets)):
                full = 0
                for t, (pos, _) in enumerate(targets):
                    full |= ((e >> t) & 1) << pos
                for pos, bit in fixed:
                    full |= bit << pos
                keep.append(diag[full])
            if not targets:
                # A phase on this rank's amplitudes (where the local controls
                # hold): as a diagonal on one control qubit, or on a free
                # local qubit.
                phase = keep[0]
                if controls:
                    (c, v), rest = controls[0], controls[1:]
                    d = np.ones(2, dtype=np.complex128)
                    d[int(v)] = phase
                    return Op([c], rest, np.diag(d))
                return Op([0], [], np.diag([phase, phase]))
            matrix = np.diag(np.array(keep))
        return Op([idx for _, idx in targets], controls, matrix)

    def apply_ops(self, ops, opts=None) -> dict:
        """Apply `ops` (on logical qubits 0..n-1). Returns the number of
        exchanges and local batches it took."""
        ops = list(ops)
        pending, batches, before = [], 0, self.exchanges
        for idx, op in enumerate(ops):
            glob = [q for q in op.targets if self._where(q)[0] == "g"]
            if glob and not _is_diagonal(np.asarray(op.matrix)):
                if pending:
                    self.engine.apply_ops(pending, opts)
                    pending, batches = [], batches + 1
                touched = set(op.qubits())
                upcoming = ops[idx + 1: idx + 1 + self.lookahead]
                for q in glob:
                    j = self.global_q.index(q)
                    self._exchange(j, self._victim(touched, upcoming))
            local = self._localize(op)
            if local is not None:
                pending.append(local)
        if pending:
            self.engine.apply_ops(pending, opts)
            batches += 1
        return {"exchanges": self.exchanges - before, "batches": batches}

    # --- reductions and read-out ----------------------------------------
    def norm_sqr(self) -> float:
        """<psi|psi> summed in FP64 over the ranks."""
        return self.transport.sum(self.engine.norm_sqr())

    def probability_one(self, qubit: int) -> float:
        """P(qubit = 1) over the whole (normalised) state."""
        kind, idx = self._where(qubit)
        if kind == "g":
            local = self.engine.norm_sqr() if self._global_bit(idx) else 0.0
        else:
            local = self.engine.probability_one(idx)
        return self.transport.sum(local) / self.norm_sqr()

    def amplitudes(self) -> np.ndarray:
        """The whole state in logical index order, on every rank (complex128;
        for states that fit one host)."""
        import torch

        a = np.asarray(self.engine.amplitudes(), dtype=np.complex128)
        parts = self.transport.gather(torch.from_numpy(a.view(np.float64).copy()))
        # every rank's placement is the same: local index i -> logical
        # local_q[i], global bit j -> logical global_q[j]
        out = np.zeros(1 << self.n, dtype=np.complex128)
        local_idx = np.arange(a.size)
        full_local = np.zeros(a.size, dtype=np.int64)
        for i, q in enumerate(self.local_q):
            full_local |= ((local_idx >> i) & 1).astype(np.int64) << q
        for r, t in enumerate(parts):
            base = 0
            for j, q in enumerate(self.global_q):
                base |= ((r >> j) & 1) << q
            out[full_local | base] = t.numpy().view(np.complex128)
        return out
