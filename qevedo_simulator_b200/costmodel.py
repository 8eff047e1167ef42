"""Learned cost model: an MLP that predicts each planned pass's device time,
used to choose among candidate plans (plain one-pass-per-gate, staged on the
CUDA cores, staged on the tensor cores; fusion widths 2-6) before running
any of them.

There is no learned planner in the reference: it plans with fixed greedy
rules (fusion in src/fusion.rs:63-170, stages in src/blocking.rs:151-302,
defaults in src/simulator.rs:37-66). Here those rules build every candidate
plan; the model only ranks them, and the greedy default stays both the
fallback and the judge: `choose_measured` times the model's pick against
the default on the device and keeps the faster.

Features come from the planner itself (qvdg_plan_features, one row of
QVDG_PASS_FEATURES per pass, no device work). Targets are the engine's own
recorded pass times (DeviceState.set_pass_timing), as log(seconds per 2^24
amplitudes). The network runs on this library's CUDA kernels
(qvdg_mlp_*: forward, backward and Adam written for it).
"""

from __future__ import annotations

import ctypes as ct
import math
import os

import numpy as np

from . import _native
from ._abi import PackedOps
from ._native import DeviceState, Plan, check, lib, options

FEATURES = 32
HIDDEN = 128
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "cost_model.npz")


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_float))


def candidates() -> list:
    """Candidate planner settings: (name, options)."""
    out = []
    for f in (2, 3, 4, 5):
        out.append((f"plain-f{f}", options(f, staged=False)))
    out.append(("staged-cuda", options(4, staged=True)))
    for f in (4, 5):
        out.append((f"staged-tensor-f{f}", options(f, staged=True, math="tensor")))
    return out


def default_options():
    """The greedy planner's default (the reference's defaults: fusion 4,
    staged)."""
    return options(4, staged=True)


def plan_features(ops, num_qubits: int, opts, precision_bits: int = 32) -> np.ndarray:
    """Per-pass feature rows of the plan `opts` builds for `ops` (host only)."""
    packed = PackedOps(ops)
    count = ct.c_size_t()
    check(lib().qvdg_plan_features(num_qubits, precision_bits, packed.array, packed.count, ct.byref(opts), None, 0,
                                   ct.byref(count)))
    rows = np.zeros((max(count.value, 1), FEATURES), dtype=np.float32)
    check(lib().qvdg_plan_features(num_qubits, precision_bits, packed.array, packed.count, ct.byref(opts),
                                   _fptr(rows), rows.shape[0], ct.byref(count)))
    return rows[:count.value]


def time_target(seconds: np.ndarray, num_qubits: int) -> np.ndarray:
    """log(seconds per 2^24 amplitudes)."""
    return np.log(np.maximum(seconds, 1e-9) / 2.0 ** (num_qubits - 24)).astype(np.float32)


def seconds_from_target(y: np.ndarray, num_qubits: int) -> np.ndarray:
    return np.exp(y.astype(np.float64)) * 2.0 ** (num_qubits - 24)


class MLP:
    """The cost model's network on the device (qvdg_mlp)."""

    def __init__(self, inputs: int = FEATURES, hidden: int = HIDDEN, seed: int = 0):
        self._h = ct.c_void_p()
        check(lib().qvdg_mlp_create(int(inputs), int(hidden), int(seed), ct.byref(self._h)))
        self.inputs, self.hidden = int(inputs), int(hidden)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().qvdg_mlp_destroy(self._h)
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

    @property
    def num_params(self) -> int:
        n = ct.c_size_t()
        check(lib().qvdg_mlp_num_params(self._h, ct.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params, dtype=np.float32)
        check(lib().qvdg_mlp_get_params(self._h, _fptr(p), p.size))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().qvdg_mlp_set_params(self._h, _fptr(p), p.size))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros(x.shape[0], dtype=np.float32)
        check(lib().qvdg_mlp_forward(self._h, _fptr(x), x.shape[0], _fptr(y)))
        return y

    def gradients(self, x, t):
        """(mean squared error, gradient of every parameter)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.num_params, dtype=np.float32)
        loss = ct.c_float()
        check(lib().qvdg_mlp_gradients(self._h, _fptr(x), _fptr(t), x.shape[0], ct.byref(loss), _fptr(g)))
        return loss.value, g

    def train(self, x, t, epochs: int = 200, batch: int = 256, lr: float = 1e-3, seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ct.c_float()
        check(lib().qvdg_mlp_train(self._h, _fptr(x), _fptr(t), x.shape[0], int(epochs), int(batch), float(lr),
                                   int(seed), ct.byref(loss)))
        return loss.value


class CostModel:
    """Predicts a plan's device time as the sum of its passes' predicted times."""

    def __init__(self, mlp: MLP | None = None):
        self.mlp = mlp or MLP()

    @classmethod
    def load(cls, path: str = MODEL_PATH) -> "CostModel":
        d = np.load(path)
        m = cls(MLP(int(d["inputs"]), int(d["hidden"])))
        m.mlp.set_params(d["params"])
        return m

    def save(self, path: str = MODEL_PATH, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.mlp.get_params(), inputs=self.mlp.inputs, hidden=self.mlp.hidden, **meta)

    def fit(self, x, t, **kw) -> float:
        return self.mlp.train(x, t, **kw)

    def predict_passes(self, feats: np.ndarray, num_qubits: int) -> np.ndarray:
        if feats.shape[0] == 0:
            return np.zeros(0)
        return seconds_from_target(self.mlp.forward(feats), num_qubits)

    def predict_plan(self, ops, num_qubits: int, opts) -> float:
        return float(self.predict_passes(plan_features(ops, num_qubits, opts), num_qubits).sum())

    def choose(self, ops, num_qubits: int, cands=None):
        """(name, options, predicted seconds) of the candidate with the least
        predicted time."""
        best = None
        for name, opts in cands or candidates():
            sec = self.predict_plan(ops, num_qubits, opts)
            if best is None or sec < best[2]:
                best = (name, opts, sec)
        return best


def measure_plan(ops, num_qubits: int, opts, state: DeviceState, repeats: int = 2):
    """(best device seconds, per-pass seconds) of one plan on `state`."""
    best, passes = math.inf, None
    with Plan(ops, num_qubits, state.precision_bits, opts) as plan:
        state.set_pass_timing(True)
        for _ in range(repeats):
            state.zero()
            s = state.execute(plan)
            if s["gate_seconds"] < best:
                best = s["gate_seconds"]
                passes = state.pass_times()[0].copy()
        state.set_pass_timing(False)
    return best, passes


def collect(op_lists, num_qubits: int, cands=None, repeats: int = 2):
    """Training rows (features, log pass times) from running every candidate
    plan of every op list on one device state."""
    xs, ts = [], []
    with DeviceState(num_qubits, 32) as st:
        for ops in op_lists:
            for _, opts in cands or candidates():
                feats = plan_features(ops, num_qubits, opts)
                _, passes = measure_plan(ops, num_qubits, opts, st, repeats)
                if passes is None or len(passes) != feats.shape[0]:
                    continue
                xs.append(feats)
                ts.append(time_target(passes, num_qubits))
    return np.concatenate(xs), np.concatenate(ts)


def choose_measured(model: CostModel, ops, num_qubits: int, state: DeviceState, cands=None):
    """The model's pick, judged against the greedy default by measurement:
    (chosen name, options, seconds, default seconds)."""
    name, opts, _ = model.choose(ops, num_qubits, cands)
    t_pick, _ = measure_plan(ops, num_qubits, opts, state)
    t_default, _ = measure_plan(ops, num_qubits, default_options(), state)
    if t_default <= t_pick:
        return "default", default_options(), t_default, t_default
    return name, opts, t_pick, t_default
