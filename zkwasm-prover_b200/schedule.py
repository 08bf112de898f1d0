"""MSM schedule selection: exhaustive autotuner, learned cost model, regret.

The reference picks the MSM window width with a fixed formula
(src/cuda/msm.rs:105).  Here three pickers exist:

* ``default``  - the library's cost formula (``zkp_msm_default_window``);
* ``autotune`` - ``zkp_msm_autotune``: time every candidate window on the
  actual bases and scalars and keep the fastest (the yardstick for the others);
* ``learned``  - an MLP cost model (``zkp_mlp_*`` kernels) trained on the
  autotuner's own measurements, predicting log(ms) relative to the shape's
  mean over windows from the shape features [log2 n / 24, log2 batch / 8,
  scalar bit-length histogram (7 bins), (c - 12) / 8], where batch is the
  number of MSMs sharing one zkp_msm_batch pipeline; the window with the
  smallest prediction wins.

A schedule only chooses the window width, so every picker gives the same
MSM result; regret (ms) is measured against the autotuner's best.
"""
from __future__ import annotations

import ctypes
import json
import math
import os

import numpy as np
import torch

from . import abi
from . import host as H

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_PATH = os.path.join(HERE, "msm_schedule_model.npz")
C_MIN, C_MAX = 8, 20
MIXES = ("uniform", "small", "sparse", "mixed")


def lib():
    return abi.load_library()


# ------------------------------------------------------------------ inputs


def bases_with_known_logs(n: int, seed: int, device="cuda"):
    """[k_i] G for seeded 62-bit k_i, generated on the device."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    k = torch.randint(0, 2 ** 62, (n,), dtype=torch.int64, device=device, generator=g)
    out = torch.empty((n, 8), dtype=torch.int64, device=device)
    abi.check(lib().zkp_g1_multiples(out.data_ptr(), k.data_ptr(), n, H.stream_handle()), "zkp_g1_multiples")
    return out, k


def scalars(n: int, mix: str, seed: int, device="cuda") -> torch.Tensor:
    """Montgomery-form scalars with the given distribution of canonical values:
    uniform below 2^253, small (< 2^20, witness-like), sparse (90% zero, the
    rest uniform), or mixed (50% uniform, 35% small, 15% sparse-uniform)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    t = torch.randint(-(2 ** 63), 2 ** 63 - 1, (n, 4), dtype=torch.int64, device=device, generator=g)
    t[:, 3] &= (1 << 61) - 1
    u = torch.rand(n, device=device, generator=g)
    if mix == "small":
        t[:, 1:] = 0
        t[:, 0] &= (1 << 20) - 1
    elif mix == "sparse":
        t[u < 0.9] = 0
    elif mix == "mixed":
        small = (u >= 0.5) & (u < 0.85)
        t[small, 1:] = 0
        t[small, 0] &= (1 << 20) - 1
        zero = (u >= 0.85) & (torch.rand(n, device=device, generator=g) < 0.9)
        t[zero] = 0
    abi.check(lib().zkp_fr_to_mont(t.data_ptr(), t.data_ptr(), n, H.stream_handle()), "zkp_fr_to_mont")
    return t


def histogram(s: torch.Tensor) -> list:
    return histograms([s])[0]


def histograms(cols) -> list:
    """The scalar-distribution features of each column: every histogram is
    launched first and all are read back with one synchronisation."""
    h = torch.zeros((len(cols), 8), dtype=torch.int32, device="cuda")
    for i, s in enumerate(cols):
        abi.check(lib().zkp_scalar_histogram(s.data_ptr(), s.shape[0], h[i].data_ptr(), H.stream_handle()),
                  "zkp_scalar_histogram")
    v = h.cpu().numpy()[:, :7].astype(np.float64)
    return [list(r / max(1.0, r.sum())) for r in v]


# largest batch the model is trained on; larger batches are presented as this
# one instead of being extrapolated (a 256-MSM pipeline otherwise drew windows
# of 13 bits for 2^22-point MSMs, against 16 at batch 32)
BATCH_TRAINED_MAX = 32


def shape_features(n: int, batch: int, hist) -> list:
    b = min(max(batch, 1), BATCH_TRAINED_MAX)
    return [math.log2(max(n, 1)) / 24.0, math.log2(b) / 8.0] + [float(x) for x in hist]


def model_input(feats, c: int) -> list:
    return list(feats) + [(c - 12) / 8.0]


# ------------------------------------------------------------------ pickers


def default_window(n: int) -> int:
    return lib().zkp_msm_default_window(n)


def reference_window(n: int, batch: int = 1) -> int:
    """src/cuda/msm.rs:105"""
    lg = lambda x: max(0, (x - 1).bit_length())
    return min(lg(batch), 3) + 10 + max(lg(n), 22) - 22


def autotune(bases, s, n: int, c_min=C_MIN, c_max=C_MAX, reps=2):
    """Exhaustive search on the device; returns (best c, {c: ms})."""
    L = lib()
    need = max(L.zkp_msm_scratch_bytes(n, c) for c in range(c_min, c_max + 1))
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    out = torch.empty(12, dtype=torch.int64, device="cuda")
    times = (ctypes.c_float * (c_max - c_min + 1))()
    best = L.zkp_msm_autotune(bases.data_ptr(), s.data_ptr(), n, c_min, c_max, reps, scratch.data_ptr(), need,
                              ctypes.addressof(times), out.data_ptr(), H.stream_handle())
    if best < 0:
        raise abi.CudaError("zkp_msm_autotune failed")
    return best, {c: float(times[c - c_min]) for c in range(c_min, c_max + 1) if times[c - c_min] >= 0}


class Model:
    """The MLP parameters on the device plus its training / prediction calls."""

    def __init__(self, params: torch.Tensor):
        self.params = params

    @classmethod
    def fresh(cls, seed=1):
        L = lib()
        p = torch.empty(L.zkp_mlp_param_count(), dtype=torch.float32, device="cuda")
        abi.check(L.zkp_mlp_init(p.data_ptr(), seed, H.stream_handle()), "zkp_mlp_init")
        return cls(p)

    @classmethod
    def load(cls, path=MODEL_PATH):
        d = np.load(path)
        return cls(torch.from_numpy(d["params"].astype(np.float32)).cuda())

    def save(self, path=MODEL_PATH, meta=None):
        np.savez(path, params=self.params.cpu().numpy(), meta=json.dumps(meta or {}))

    def predict(self, X: np.ndarray) -> np.ndarray:
        x = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
        y = torch.empty(x.shape[0], dtype=torch.float32, device="cuda")
        abi.check(lib().zkp_mlp_forward(self.params.data_ptr(), x.data_ptr(), x.shape[0], y.data_ptr(),
                                        H.stream_handle()), "zkp_mlp_forward")
        return y.cpu().numpy()

    def train(self, X: np.ndarray, y: np.ndarray, steps=4000, lr=3e-3, weights=None):
        """Full-batch Adam on the (weighted) mean squared error; returns the
        loss history [(step, loss)]."""
        L = lib()
        x = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
        t = torch.from_numpy(np.ascontiguousarray(y, np.float32)).cuda()
        w = None if weights is None else torch.from_numpy(np.ascontiguousarray(weights, np.float32)).cuda()
        B = x.shape[0]
        g = torch.zeros_like(self.params)
        m = torch.zeros_like(self.params)
        v = torch.zeros_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        scratch = torch.empty(L.zkp_mlp_scratch_floats(B), dtype=torch.float32, device="cuda")
        st = H.stream_handle()
        hist = []
        for step in range(1, steps + 1):
            abi.check(L.zkp_mlp_train_step(self.params.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(),
                                           x.data_ptr(), t.data_ptr(), None if w is None else w.data_ptr(),
                                           B, lr, step, loss.data_ptr(),
                                           scratch.data_ptr(), st), "zkp_mlp_train_step")
            if step == 1 or step % 500 == 0:
                hist.append((step, float(loss.item())))
        return hist

    def pick(self, feats, c_min=C_MIN, c_max=C_MAX) -> int:
        f = (ctypes.c_float * 9)(*[float(x) for x in feats])
        scratch = torch.empty(256, dtype=torch.float32, device="cuda")
        c = lib().zkp_msm_schedule_predict(self.params.data_ptr(), ctypes.addressof(f), c_min, c_max,
                                           scratch.data_ptr(), H.stream_handle())
        if c < 0:
            raise abi.CudaError("zkp_msm_schedule_predict failed")
        return c


# ------------------------------------------------------------------ NTT radices


_R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def _root_of_unity_mont(log_n: int):
    """A primitive 2^log_n-th root of unity of Fr (from the generator 7) in
    Montgomery form, as 4 u64 limbs."""
    w = pow(7, (_R_MOD - 1) >> log_n, _R_MOD)
    v = w * (1 << 256) % _R_MOD
    return np.array([(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)], np.uint64)


def ntt_splits(log_n: int, lo: int = 6, hi: int = 12, max_passes: int = 3) -> list:
    """Every ordered split of log_n into 2..max_passes pass radices in [lo, hi]."""
    out = []

    def rec(left, parts):
        if left == 0 and len(parts) >= 2:
            out.append(list(parts))
            return
        if len(parts) == max_passes:
            return
        for r in range(lo, min(hi, left) + 1):
            rec(left - r, parts + [r])

    rec(log_n, [])
    return out


def autotune_ntt(log_n: int, ncols: int = 1, reps: int = 3, omegas=None):
    """Exhaustive search over the pass splits of a batched NTT of ncols columns
    of 2^log_n points (zkp_ntt_batch_plan on seeded device data); returns
    (best split, {split: ms}).  Results do not depend on the split (the tests
    check that), only the time does."""
    n = 1 << log_n
    g = torch.Generator(device="cuda")
    g.manual_seed(log_n)
    buf = torch.randint(-(2 ** 63), 2 ** 63 - 1, (ncols * n, 4), dtype=torch.int64, device="cuda", generator=g)
    buf[:, 3] &= (1 << 61) - 1
    tmp = torch.empty_like(buf)
    if omegas is None:
        omegas = H.generate_omega_buffers(_root_of_unity_mont(log_n), log_n, False)
    times = {}
    for split in ntt_splits(log_n):
        H.ntt_batch_plan(buf, tmp, omegas, log_n, ncols, split)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            H.ntt_batch_plan(buf, tmp, omegas, log_n, ncols, split)
        b.record()
        b.synchronize()
        times[tuple(split)] = a.elapsed_time(b) / reps
    best = min(times, key=times.get)
    return list(best), times


def autotune_extend(log_n: int, ext_bits: int, ncols: int, chunks=(2, 4, 8, 16), shift: int = 7, reps: int = 2):
    """Exhaustive search over the run-time choices of the extended-domain phase
    for ncols columns of 2^log_n points: the multiplier-table layout
    (zkp_extend_batch over Montgomery tables, or zkp_extend_batch_tables over
    (w, w') pairs) and the columns per launch.  Returns (best (layout, chunk),
    {(layout, chunk): ms for the whole phase}).  The outputs do not depend on
    either choice (the parity tests run both layouts)."""
    n, E = 1 << log_n, 1 << ext_bits
    w = pow(7, (_R_MOD - 1) >> log_n, _R_MOD)
    mont = lambda v: np.array([((v * (1 << 256) % _R_MOD) >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)],
                              np.uint64)
    tw = H.generate_omega_buffers(mont(w), log_n, False)
    tw_inv = H.generate_omega_buffers(mont(pow(w, -1, _R_MOD)), log_n, False)
    n_inv = H.to_device(mont(pow(n, -1, _R_MOD)).reshape(1, 4))
    w_ext = pow(7, (_R_MOD - 1) >> (log_n + ext_bits), _R_MOD)
    twist = H.twist_tables(mont(shift), mont(w_ext), log_n, ext_bits, tw)
    tables = H.extend_tables(tw, tw_inv, n_inv, mont(shift), mont(w_ext), log_n, ext_bits)
    g = torch.Generator(device="cuda")
    g.manual_seed(log_n)
    lag = torch.randint(-(2 ** 63), 2 ** 63 - 1, (ncols * n, 4), dtype=torch.int64, device="cuda", generator=g)
    lag[:, 3] &= (1 << 61) - 1
    coeff = torch.empty_like(lag)
    ext = torch.empty((ncols * E * n, 4), dtype=torch.int64, device="cuda")
    times = {}
    for chunk in chunks:
        if chunk > ncols or ncols % chunk:
            continue
        scratch = torch.empty((chunk * E * n, 4), dtype=torch.int64, device="cuda")
        for layout in ("montgomery", "pairs"):
            def phase():
                for c0 in range(0, ncols, chunk):
                    if layout == "pairs":
                        H.extend_batch_tables(ext[c0 * E * n:], coeff[c0 * n:], lag[c0 * n:], chunk, log_n, ext_bits,
                                              tables, scratch)
                    else:
                        H.extend_batch(ext[c0 * E * n:], coeff[c0 * n:], lag[c0 * n:], chunk, log_n, ext_bits,
                                       tw_inv, n_inv, tw, twist, scratch)
            phase()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                phase()
            b.record()
            b.synchronize()
            times[(layout, chunk)] = a.elapsed_time(b) / reps
        del scratch
    best = min(times, key=times.get)
    return best, times


# ------------------------------------------------------------------ dataset / evaluation


def autotune_batch(bases, cols, n: int, c_min=C_MIN, c_max=C_MAX, reps=2):
    """Exhaustive search for len(cols) same-shape MSMs run as one zkp_msm_batch
    pipeline with one window for all; returns (best c, {c: ms per batch}).
    Windows whose pipeline does not fit (2^32 or more sorted entries) are left
    out."""
    L = lib()
    count = len(cols)
    ns = [n] * count
    n_arr = (ctypes.c_uint32 * count)(*ns)
    need, ok = 0, []
    for c in range(c_min, c_max + 1):
        c_arr = (ctypes.c_int * count)(*([c] * count))
        b = L.zkp_msm_batch_scratch_bytes(ctypes.addressof(n_arr), ctypes.addressof(c_arr), count)
        if b:
            ok.append(c)
            need = max(need, b)
    scratch = torch.empty(max(1, need), dtype=torch.uint8, device="cuda")
    out = torch.empty((count, 12), dtype=torch.int64, device="cuda")
    times = {}
    for c in ok:
        ws = [c] * count
        H.msm_batch(bases, cols, ns, ws, scratch=scratch, out=out)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            H.msm_batch(bases, cols, ns, ws, scratch=scratch, out=out)
        b.record()
        b.synchronize()
        times[c] = a.elapsed_time(b) / reps
    del scratch
    return min(times, key=times.get), times


def collect(sizes, mixes=MIXES, batches=(1,), reps=2, seed=100, c_min=C_MIN, c_max=C_MAX, max_points=1 << 26):
    """Autotune every (size, batch, mix) shape; one record per shape.  A batch
    of b is b same-shape MSMs (independent scalars) through one zkp_msm_batch
    pipeline; batch 1 uses zkp_msm.  "times_ms" is the time of the whole
    batch.  Shapes above max_points scalars in total are skipped."""
    records = []
    nmax = max(sizes)
    bases, _ = bases_with_known_logs(nmax, seed)
    for n in sizes:
        for batch in batches:
            if n * batch > max_points:
                continue
            for mi, mix in enumerate(mixes):
                cols = [scalars(n, mix, seed + 17 * n.bit_length() + 1000 * j + mi) for j in range(batch)]
                hist = histogram(cols[0])
                if batch == 1:
                    best, times = autotune(bases, cols[0], n, c_min, c_max, reps)
                else:
                    best, times = autotune_batch(bases, cols, n, c_min, c_max, reps)
                records.append({"n": n, "batch": batch, "mix": mix, "hist": hist, "best": best,
                                "times_ms": times})
                del cols
    return records


def training_set(records):
    """Model inputs, targets and sample weights.  The target of window c is
    log(ms) minus its mean over the shape's measured windows: the pick is an
    argmin over the windows of one shape, so a per-shape offset carries no
    information and the model's capacity goes to how time depends on c.  The
    weight sqrt(fastest ms of the shape), normalised to mean 1, makes the
    shapes where a wrong pick costs the most milliseconds count the most."""
    X, y, w = [], [], []
    for r in records:
        f = shape_features(r["n"], r["batch"], r["hist"])
        logs = {int(c): math.log(ms) for c, ms in r["times_ms"].items()}
        mean = sum(logs.values()) / len(logs)
        wt = math.sqrt(min(r["times_ms"].values()))
        for c, lt in logs.items():
            X.append(model_input(f, c))
            y.append(lt - mean)
            w.append(wt)
    w = np.array(w, np.float32)
    return np.array(X, np.float32), np.array(y, np.float32), w / w.mean()


def regret(records, picker):
    """Total and per-shape regret (ms) of a picker against the fastest window."""
    total, rows = 0.0, []
    for r in records:
        times = {int(c): v for c, v in r["times_ms"].items()}
        best = min(times.values())
        c = picker(r)
        if c not in times:  # outside the measured range: charge the nearest measured window
            c = min(times, key=lambda k: abs(k - c))
        rows.append({"n": r["n"], "batch": r["batch"], "mix": r["mix"], "picked": c,
                     "regret_ms": times[c] - best})
        total += times[c] - best
    return total, rows


def mlp_forward_numpy(params: np.ndarray, X: np.ndarray) -> np.ndarray:
    """CPU restatement of mlp_forward_kernel (same parameter layout)."""
    D, H1, H2 = X.shape[1], 64, 64
    o = 0
    W1 = params[o:o + D * H1].reshape(D, H1)
    o += D * H1
    b1 = params[o:o + H1]
    o += H1
    W2 = params[o:o + H1 * H2].reshape(H1, H2)
    o += H1 * H2
    b2 = params[o:o + H2]
    o += H2
    W3 = params[o:o + H2]
    o += H2
    b3 = params[o]
    h1 = np.maximum(X @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h2 @ W3 + b3
