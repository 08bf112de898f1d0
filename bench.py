"""Benchmark of the batched extended-domain NTT phase on B200.

Workload (the batched NTT configuration of the KZG prover): 64 Fr columns of
2^20 Lagrange values -> iNTT to coefficients -> coset NTT on the 8x extended
domain (2^23 points, shift = the field's multiplicative generator 7), all
columns through zkp_extend_batch (one launch per stage over a chunk of
columns).  Synthetic seeded inputs, uniform in [0, 2^253), generated on the
device.  One step = the whole 64-column phase.

Metric: algorithmic HBM bytes of the phase per second (GB/s, 1e9 bytes):
per column 32 MiB Lagrange read + 32 MiB coefficients written + 32 MiB
coefficients read + 256 MiB extended evaluations written = 352 MiB.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU under torch.distributed.run; every rank runs
its own 64-column phase (columns are independent: weak scaling, no
collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import gc
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import time

# the proof's buffers come and go in sizes of 0.1-30 GiB: growable segments
# keep the caching allocator from fragmenting HBM between the schedules
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")

import torch  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
GENERATOR = 7
MIB = 1 << 20


def omega(log_n: int) -> int:
    w = pow(GENERATOR, (R_MOD - 1) >> 28, R_MOD)
    for _ in range(log_n, 28):
        w = w * w % R_MOD
    return w


def mont(x: int):
    v = (x % R_MOD) * (1 << 256) % R_MOD
    return [(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)]


def fr_tensor(vals, device):
    import numpy as np

    a = np.array([mont(v) for v in vals], dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64)).to(device)


def random_fr(n: int, seed: int, device) -> torch.Tensor:
    """Seeded uniform values in [0, 2^253) (all below r): 4 int64 limbs each."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    t = torch.randint(-(2 ** 63), 2 ** 63 - 1, (n, 4), dtype=torch.int64, device=device, generator=g)
    t[:, 3] &= (1 << 61) - 1
    return t


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"zk_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ workload


class ExtendPhase:
    """64 columns: iNTT 2^log_n -> coset NTT on 2^(log_n + ext_bits)."""

    def __init__(self, zkp, device, columns=64, log_n=20, ext_bits=3, chunk=8, seed=1, pair_tables=True):
        self.zkp, self.H = zkp, zkp.host
        self.device = device
        self.C, self.log_n, self.e, self.chunk = columns, log_n, ext_bits, chunk
        n = self.n = 1 << log_n
        E = self.E = 1 << ext_bits
        H = self.H
        w = omega(log_n)
        self.tw = H.generate_omega_buffers(mont(w), log_n)
        self.tw_inv = H.generate_omega_buffers(mont(pow(w, -1, R_MOD)), log_n)
        self.n_inv = fr_tensor([pow(n, -1, R_MOD)], device)
        self.twist = H.twist_tables(mont(GENERATOR), mont(omega(log_n + ext_bits)), log_n, ext_bits, self.tw)
        # the same tables as (w, w') pairs: products by known factors
        self.pairs = pair_tables
        self.tables = (H.extend_tables(self.tw, self.tw_inv, self.n_inv, mont(GENERATOR),
                                       mont(omega(log_n + ext_bits)), log_n, ext_bits) if pair_tables else None)
        self.lag = random_fr(columns * n, seed, device)
        self.coeff = torch.empty((columns * n, 4), dtype=torch.int64, device=device)
        self.ext = torch.empty((columns * E * n, 4), dtype=torch.int64, device=device)
        self.scratch = torch.empty((chunk * E * n, 4), dtype=torch.int64, device=device)
        torch.cuda.synchronize()

    # algorithmic bytes / field multiplications
    def bytes_per_column(self):
        return (3 + self.E) * self.n * 32

    def mults_per_column(self):
        n, lg, E = self.n, self.log_n, self.E
        ntt = (n // 2) * lg
        return ntt + n + E * (ntt + n)  # iNTT + n^-1 scale, E sub-transforms + twist

    def fused(self):
        """zkp_extend_batch fuses the last inverse pass with the first coset
        passes when its coset table carries the per-radix factors."""
        return self.zkp.load_library().zkp_coset_table_elems(self.log_n, self.e) > self.E * self.n

    def stage_names(self):
        if self.fused():
            return ["intt_pass1", "none", "fused_intt_pass2_coset_pass1", "coset_pass2"]
        return ["intt_pass1", "intt_pass2", "coset_pass1", "coset_pass2"]

    def stage_bytes(self):
        """algorithmic bytes each stage launch must read + write (one chunk):
        its input and output columns, no twiddle or twist tables."""
        c, n, E = self.chunk, self.n, self.E
        if self.fused():
            return [2 * c * n * 32, 0, (2 + E) * c * n * 32, 2 * E * c * n * 32]
        return [2 * c * n * 32, 2 * c * n * 32, (2 + E) * c * n * 32, 2 * E * c * n * 32]

    def stage_mults(self):
        """algorithmic Fr products per stage launch: (n/2) log2 n per
        transform split evenly over its two passes, n for the n^-1 scale and n
        for each coset twist."""
        c, n, E, lg = self.chunk, self.n, self.E, self.log_n
        half = (n // 2) * lg // 2
        if self.fused():
            return [c * half, 0, c * (half + n + E * (half + n)), c * E * half]
        return [c * half, c * (half + n), c * E * (half + n), c * E * half]

    def launches_per_step(self):
        return (self.C // self.chunk) * (3 if self.fused() else 4)

    def run_chunk(self, c0, events=None, stream=None, lag=None, coeff=None):
        n, E = self.n, self.E
        lag = self.lag if lag is None else lag
        coeff = self.coeff if coeff is None else coeff
        if self.pairs:
            self.H.extend_batch_tables(self.ext[c0 * E * n:], coeff[c0 * n:], lag[c0 * n:], self.chunk, self.log_n,
                                       self.e, self.tables, self.scratch, stage_events=events, stream=stream)
        else:
            self.H.extend_batch(self.ext[c0 * E * n:], coeff[c0 * n:], lag[c0 * n:], self.chunk, self.log_n,
                                self.e, self.tw_inv, self.n_inv, self.tw, self.twist, self.scratch,
                                stage_events=events, stream=stream)

    def step(self, events=None):
        for i, c0 in enumerate(range(0, self.C, self.chunk)):
            self.run_chunk(c0, None if events is None else events[i])


def make_event_array(k):
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
    for e in evs:
        e.record()
    arr = (ctypes.c_void_p * k)(*[e.cuda_event for e in evs])
    return evs, arr


def calib_mont_rate(zkp, device):
    """Sustained Fr Montgomery multiplications per second on this GPU."""
    lib = zkp.load_library()
    out = torch.zeros(4, dtype=torch.int64, device=device)
    props = torch.cuda.get_device_properties(device)
    blocks, iters = props.multi_processor_count * 8, 4096
    st = torch.cuda.current_stream().cuda_stream
    zkp.abi.check(lib.zkp_calib_mont_rate(out.data_ptr(), blocks, 64, st), "calib")
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    zkp.abi.check(lib.zkp_calib_mont_rate(out.data_ptr(), blocks, iters, st), "calib")
    b.record()
    b.synchronize()
    sec = a.elapsed_time(b) / 1e3
    return blocks * 256 * 4 * iters / sec


def calib_shoup_rate(zkp, device):
    """Sustained Fr products by a known factor per second on this GPU."""
    lib = zkp.load_library()
    out = torch.zeros(4, dtype=torch.int64, device=device)
    w = 2 * R_MOD // 3
    pair = torch.tensor([[(v >> (64 * j)) & (2 ** 64 - 1) for j in range(4)] for v in (w, (w << 256) // R_MOD)],
                        dtype=torch.uint64).view(torch.int64).to(device)
    props = torch.cuda.get_device_properties(device)
    blocks, iters = props.multi_processor_count * 8, 4096
    st = torch.cuda.current_stream().cuda_stream
    zkp.abi.check(lib.zkp_calib_shoup_rate(out.data_ptr(), pair.data_ptr(), blocks, 64, st), "calib")
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    zkp.abi.check(lib.zkp_calib_shoup_rate(out.data_ptr(), pair.data_ptr(), blocks, iters, st), "calib")
    b.record()
    b.synchronize()
    return blocks * 256 * 4 * iters / (a.elapsed_time(b) / 1e3)


def cpu_baseline_port(log_n=20, ext_bits=3, reps=1):
    """The oracle (C restatement, OpenMP on all host cores) on one column."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n = 1 << log_n
    a = O.rand_fr(n, 12345)
    t0 = time.perf_counter()
    for _ in range(reps):
        c = O.intt(a, log_n)
        O.coset_ntt(c, log_n, log_n + ext_bits, GENERATOR)
    sec = (time.perf_counter() - t0) / reps
    col_bytes = (3 + (1 << ext_bits)) * n * 32
    cores = os.cpu_count()
    return {"value": col_bytes / sec / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
            "sample": f"1 column (iNTT 2^{log_n} + coset NTT 2^{log_n + ext_bits}) per rep, {reps} rep(s), "
                      f"{sec:.2f} s each"}


def msm_inputs(zkp, n, seed, device):
    """n bases [k_i]G with seeded 64-bit k_i (generated on the device) and n
    seeded scalars below 2^253."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    k = torch.randint(0, 2 ** 62, (n,), dtype=torch.int64, device=device, generator=g)
    bases = torch.empty((n, 8), dtype=torch.int64, device=device)
    zkp.abi.check(zkp.load_library().zkp_g1_multiples(bases.data_ptr(), k.data_ptr(), n,
                                                        torch.cuda.current_stream().cuda_stream), "g1_multiples")
    return bases, random_fr(n, seed + 1, device)


def run_msm(zkp, device, sizes=(1 << 18, 1 << 22), reps=5):
    """Single MSMs through zkp_msm on device-resident bases and scalars."""
    H = zkp.host
    res = []
    for n in sizes:
        bases, scalars = msm_inputs(zkp, n, 77 + n.bit_length(), device)
        scratch = H.msm_scratch(n)
        out = torch.empty(12, dtype=torch.int64, device=device)
        for _ in range(2):
            H.msm(bases, scalars, n=n, scratch=scratch, out=out)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            H.msm(bases, scalars, n=n, scratch=scratch, out=out)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b) / reps
        c = zkp.load_library().zkp_msm_default_window(n)
        line = {"n": n, "ms": round(ms, 4), "mpts_per_s": round(n / ms / 1e3, 2), "window_bits": c}
        # the same MSM over a table of pre-multiplied bases (the bases stay
        # resident across MSMs, as an SRS does); the one-time build is timed
        # apart, into a buffer allocated before the timed region
        lib = zkp.load_library()
        tc = lib.zkp_msm_table_default_window(n)
        table = torch.empty(lib.zkp_msm_table_bytes(n, tc) // 8, dtype=torch.int64, device=device)
        H.msm_table_build(bases, n, tc, table=table)  # untimed: the first launch loads the kernel
        torch.cuda.synchronize()
        a.record()
        H.msm_table_build(bases, n, tc, table=table)
        b.record()
        b.synchronize()
        build_ms = a.elapsed_time(b)
        tscratch = torch.empty(max(1, zkp.load_library().zkp_msm_table_scratch_bytes(n, tc)), dtype=torch.uint8,
                               device=device)
        tout = torch.empty(12, dtype=torch.int64, device=device)
        for _ in range(2):
            H.msm_table(table, n, tc, scalars, n=n, scratch=tscratch, out=tout)
        torch.cuda.synchronize()
        a.record()
        for _ in range(reps):
            H.msm_table(table, n, tc, scalars, n=n, scratch=tscratch, out=tout)
        b.record()
        b.synchronize()
        tms = a.elapsed_time(b) / reps
        line.update({"table_ms": round(tms, 4), "table_mpts_per_s": round(n / tms / 1e3, 2),
                     "table_window_bits": tc, "table_build_ms": round(build_ms, 2)})
        res.append(line)
        del bases, scalars, scratch, table, tscratch
    return res


def run_rows(lib, device, mont_rate, peak_hbm, ours=True, log_n=22, log_ext=24, reps=3):
    """One timed kernel for each remaining hot-path row at the k = 22 column
    size (scans, inversions, grand products: n = 2^22) and its extended domain
    (quotient kernels: N = 2^24), device-resident inputs, CUDA events.  Each
    line gives the algorithmic bytes (the kernel's input and output columns)
    and Fr products (its formula, per row; where this library's formula
    takes fewer products than the reference's, each side is counted by its
    own), the two resulting time bounds (bytes / measured HBM copy rate,
    products / measured Montgomery-product rate; products by a known factor,
    which cost less, are counted as Montgomery products), which one binds,
    and the fraction of that bound reached.

    The rows named by a reference C symbol run through that symbol, so the
    same call times this library (ours=True, lib = its ctypes handle) or the
    reference's kernels rebuilt for sm_100a (ours=False, lib = the oracle/_ref
    handle, only the reference-symbol rows); the zkp_* rows are this library's
    batched entry points."""
    import ctypes

    st = torch.cuda.current_stream().cuda_stream
    n, N = 1 << log_n, 1 << log_ext
    E = 32

    def fr(k, seed):
        return random_fr(k, seed, device)

    cols = [fr(N, 700 + i) for i in range(8)]
    small = [fr(n, 800 + i) for i in range(8)]
    one, y, beta, gamma = fr(1, 901), fr(1, 902), fr(1, 903), fr(1, 904)
    res = fr(N, 905)
    out_n, tmp_n, z_n = torch.empty_like(small[0]), torch.empty_like(small[0]), torch.empty_like(small[0])
    last = fr(1, 912)
    omega_n = torch.zeros((n, 4), dtype=torch.int64, device=device)
    omega_n[:2] = fr(2, 906)
    omega_N = torch.zeros((N, 4), dtype=torch.int64, device=device)
    omega_N[:2] = fr(2, 907)
    coset = fr(3, 908)
    ext = torch.empty((N, 4), dtype=torch.int64, device=device)
    ptrs = lambda ts: torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device=device)
    # field_op_batch_mul_sum: c0 a b + c1 d + c2 e f g (src/eval_h.rs term
    # lists; the coefficients carry powers of y, so they are random here)
    gate_c = fr(3, 913)
    cptr = [gate_c.data_ptr() + 32 * k for k in range(3)]
    vd = torch.tensor([cptr[0], cols[0].data_ptr(), cols[1].data_ptr(), 0, cptr[1],
                       cols[2].data_ptr(), 0, cptr[2], cols[3].data_ptr(), cols[4].data_ptr(),
                       cols[5].data_ptr(), 0], dtype=torch.int64, device=device)
    rd = torch.tensor([0, 1, -1, 2, 0, -2], dtype=torch.int32, device=device)
    # field_sum: sum_j v_j[i] omega^((n + rot_j) i) c_j, one column without
    # its constant
    sum_v = ptrs(small[:3])
    sum_c = torch.tensor([gate_c.data_ptr(), 0, beta.data_ptr()], dtype=torch.int64, device=device)
    sum_rot = torch.tensor([0, 1, -1], dtype=torch.int32, device=device)
    sets4, ins2, tabs2 = ptrs(cols[:4]), ptrs(small[:2]), ptrs(small[2:4])
    pc, ps = ptrs(small[:4]), ptrs(small[4:8])
    betas2, betas4, xt = fr(2, 909), fr(4, 910), fr(log_n, 911)
    P, I, S = "p", "i", "s"
    # (label, algorithmic bytes, Fr products, symbol, args, reference symbol?)
    cases = [
        ("a7 expand_omega_buffer (w^i, 2^24)", N * E, N, "expand_omega_buffer",
         [(P, omega_N), (I, log_ext), (I, 0)], True),
        ("a8 extended_prepare (zeta coset + zero pad, 2^22 -> 2^24)", (n + N) * E, n, "extended_prepare",
         [(P, ext), (P, coset), (I, 3), (I, n), (I, N), (I, 0), (S, st)], True),
        ("a9 logup_sum_input_inv (sum of 1/(input + beta), 2^22)", 3 * n * E, 4 * n, "logup_sum_input_inv",
         [(P, out_n), (P, small[0]), (P, tmp_n), (P, beta), (I, 1), (I, n), (S, st)], True),
        ("a10 eval_logup_z_compose (2^22)", 5 * n * E, 5 * n, "eval_logup_z_compose",
         [(P, z_n), (P, small[1]), (P, small[2]), (P, small[3]), (P, beta), (P, last), (I, n - 9), (I, n),
          (S, st)], True),
        ("a13 field_op_batch_mul_sum (3 terms, 6 columns, 2^24)", 8 * N * E, 6 * N, "field_op_batch_mul_sum",
         [(P, res), (P, vd), (P, rd), (I, 12), (I, N), (S, st)], True),
        # the reference's chain takes 2 (k - 1) products per row for k sets;
        # this library's Horner form k (k - 1 of them by known factors)
        ("a13 permutation_eval_h_p2 (4 sets, rotation, 2^24)", (4 + 1 + 2) * N * E, (4 * N, 6 * N),
         "permutation_eval_h_p2", [(P, res), (P, sets4), (P, cols[4]), (P, cols[5]), (P, y), (I, 4), (I, -8),
                                   (I, N)], True),
        ("a13 logup_eval_h (2^24)", (9 + 2) * N * E, 9 * N, "logup_eval_h",
         [(P, res)] + [(P, c) for c in cols[:8]] + [(P, cols[0]), (P, y), (I, 4), (I, N), (S, st)], True),
        ("a13 shuffle_eval_h (2^24)", (6 + 2) * N * E, 9 * N, "shuffle_eval_h",
         [(P, res)] + [(P, c) for c in cols[:6]] + [(P, y), (I, 4), (I, N)], True),
        ("a13 lookup_eval_h (2^24)", (9 + 1) * N * E, 16 * N, "lookup_eval_h",
         [(P, res)] + [(P, c) for c in cols[:8]] + [(P, y), (P, beta), (P, gamma), (I, 1), (I, N), (S, st)],
         True),
        ("a13 field_op (l[i+1] c_l * r[i-1] c_r, 2^24)", 3 * N * E, 3 * N, "field_op",
         [(P, res), (P, cols[0]), (I, 1), (P, gate_c), (P, cols[1]), (I, -1), (P, beta), (I, N), (I, 1), (S, st)],
         True),
        ("a13 field_mul_zip (3 coset powers, 2^24)", 2 * N * E, N, "field_mul_zip",
         [(P, res), (P, coset), (I, 3), (I, N)], True),
        ("f2 shplonk_h_x_merge (3 points, 2^22)", 4 * n * E, 4 * n, "shplonk_h_x_merge",
         [(P, out_n), (P, y), (P, small[6]), (P, small[7]), (P, coset), (I, 3), (I, n)], True),
        # values / prod_j (w_i - p_j): 4 products, then one batch inversion
        # (3 products per element) and the quotient (1); the reference
        # inverts twice per element instead
        ("f2 shplonk_h_x_div_points (4 points, 2^22)", 3 * n * E, 8 * n, "shplonk_h_x_div_points",
         [(P, small[4]), (P, small[7]), (P, betas4), (I, 4), (I, n)], True),
        ("f2 field_sum (3 columns, omega^(rot i), 2^22)", 4 * n * E, 5 * n, "field_sum",
         [(P, out_n), (P, sum_v), (P, sum_c), (P, sum_rot), (P, small[7]), (I, 3), (I, n)], True),
        ("f1 poly_eval (Horner levels in place, 2^22)", 2 * n * E, n, "poly_eval",
         [(P, small[5]), (P, out_n), (P, xt), (I, n), (S, st)], True),
        ("a9 zkp_batch_inverse (2^22)", 2 * n * E, 3 * n, "zkp_batch_inverse",
         [(P, out_n), (P, small[0]), (P, None), (I, n), (I, 0), (P, tmp_n), (S, st)], False),
        ("a10 zkp_grand_sum (prefix sum, 2^22)", 2 * n * E, 0, "zkp_grand_sum",
         [(P, out_n), (P, small[1]), (I, n), (P, None), (P, tmp_n), (S, st)], False),
        ("a11 zkp_permutation_z (4 columns, 2^22)", (2 * 4 + 2) * n * E, (4 * 4 + 6) * n, "zkp_permutation_z",
         [(P, out_n), (P, pc), (P, ps), (I, 4), (P, beta), (P, gamma), (P, betas4), (P, omega_n), (P, one), (I, n),
          (P, tmp_n), (S, st)], False),
        ("a12 zkp_shuffle_z (2 groups, 2^22)", (2 * 2 + 1) * n * E, (2 * 2 + 6) * n, "zkp_shuffle_z",
         [(P, out_n), (P, ins2), (P, tabs2), (P, betas2), (I, 2), (I, n), (P, ext), (S, st)], False),
    ]

    def conv(spec):
        k, v = spec
        if k == P:
            addr = 0 if v is None else v.data_ptr()
            return addr if ours else ctypes.c_void_p(addr)
        if k == S:
            return v if ours else ctypes.c_void_p(v)
        if k == "hostptr":
            return ctypes.byref(v)
        return v if ours else ctypes.c_int(v)

    # a6: the drop-in ntt on one column, with each library's own twiddle
    # table (expand_omega_buffer, as the reference host builds it,
    # src/cuda/ntt.rs:15-59) and the reference's radix table pq
    def ntt_case(log_nt):
        nt = 1 << log_nt
        w = omega(log_nt)
        om = torch.zeros((nt, 4), dtype=torch.int64, device=device)
        om[:2] = fr_tensor([1, w], device)
        torch.cuda.synchronize()
        assert lib.expand_omega_buffer(conv((P, om)), conv((I, log_nt)), conv((I, 1))) == 0
        md = min(8, log_nt)
        tw8 = pow(w, nt >> md, R_MOD)
        pq = fr_tensor([pow(tw8, i, R_MOD) for i in range((1 << md) >> 1)], device)
        buf = random_fr(nt, 1300 + log_nt, device)
        tmp = torch.empty_like(buf)
        swap = ctypes.c_bool(False)
        return (f"a6 ntt (one column, 2^{log_nt})", 2 * nt * E, (nt // 2) * log_nt, "ntt",
                [(P, buf), (P, tmp), (P, pq), (P, om), (P, None), (I, log_nt), (I, 8), ("hostptr", swap), (S, st)],
                True), (om, pq, buf, tmp, swap)

    keep = []
    for lg in (22, 25):
        case, held = ntt_case(lg)
        cases.append(case)
        keep.append(held)

    out = []
    for name, nbytes, mults, sym, args, is_ref in cases:
        if not ours and not is_ref:
            continue
        if isinstance(mults, tuple):  # (this library's formula, the reference's)
            mults = mults[0] if ours else mults[1]
        fn_c = getattr(lib, sym)
        a = [conv(x) for x in args]

        def fn():
            err = fn_c(*a)
            if err != 0:
                raise RuntimeError(f"{sym} returned {err}")

        fn()
        torch.cuda.synchronize()
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record()
        for _ in range(reps):
            fn()
        eb.record()
        eb.synchronize()
        ms = ea.elapsed_time(eb) / reps
        row = {"row": name, "ms": round(ms, 4), "GB_s": round(nbytes / (ms / 1e3) / 1e9, 1),
               "Gmul_s": round(mults / (ms / 1e3) / 1e9, 2)}
        if mont_rate:
            t_hbm = nbytes / (peak_hbm * 1e9) * 1e3
            t_int = mults / mont_rate * 1e3
            row.update(bound="int" if t_int > t_hbm else "hbm", frac=round(max(t_hbm, t_int) / ms, 3))
        out.append(row)
    del cols, small, res, ext, omega_N, omega_n, keep
    return out


def run_staging(zkp, device, cols=8, log_n=22, reps=2):
    """Column copies between HBM and host memory, 2^22-element columns: the
    library's staging (page-locked huge-page pool + bounded copy queue, two
    copies in flight, the reference's src/hugetlb.rs + src/async_copy_queue.rs
    arrangement) against plain copies to and from pageable host memory."""
    import numpy as np

    H = zkp.host
    nbytes = (1 << log_n) * 32
    dev = [random_fr(1 << log_n, 1200 + i, device) for i in range(cols)]
    pool = H.HostPool(nbytes, chunks_per_block=2, flags=H.HostPool.PIN | H.HostPool.HUGE)
    q = H.CopyQueue(max_in_flight=2)
    host = [pool.alloc(nbytes) for _ in range(cols)]
    pageable = [np.empty(nbytes, np.uint8) for _ in range(cols)]
    cur = torch.cuda.current_stream()
    res = {"columns": cols, "column_bytes": nbytes}

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    def q_d2h():
        for d, p in zip(dev, host):
            q.push(p, d.data_ptr(), nbytes, q.D2H, after=cur)
        q.sync()

    def q_h2d():
        for d, p in zip(dev, host):
            q.push(d.data_ptr(), p, nbytes, q.H2D, after=cur)
        q.sync()

    def plain_d2h():
        for d, h in zip(dev, pageable):
            h[:] = d.view(torch.uint8).reshape(-1).cpu().numpy()

    def plain_h2d():
        for d, h in zip(dev, pageable):
            d.view(torch.uint8).reshape(-1).copy_(torch.from_numpy(h))

    for name, fn in (("pinned_queue_d2h", q_d2h), ("pinned_queue_h2d", q_h2d), ("pageable_d2h", plain_d2h),
                     ("pageable_h2d", plain_h2d)):
        sec = timed(fn)
        res[name + "_GB_s"] = round(cols * nbytes / sec / 1e9, 2)
    q.close()
    pool.close()
    del dev
    return res


def run_msm_columns(zkp, device, count=16, log_n=18, reps=3):
    """count MSMs of 2^log_n points over one base array (columns committed
    together): the drop-in reference ABI (msm per column, then one
    batch_msm_collect, with the reference host's window and scratch sizing,
    src/cuda/msm.rs:239-455) against a loop of zkp_msm calls."""
    H = zkp.host
    n = 1 << log_n
    bases, _ = msm_inputs(zkp, n, 91, device)
    cols = [random_fr(n, 300 + i, device) for i in range(count)]
    ref = H.ReferenceMsmBatch(bases, cols, n)
    scratch = H.msm_scratch(n)
    out = torch.empty((count, 12), dtype=torch.int64, device=device)

    def loop():
        for i, c in enumerate(cols):
            H.msm(bases, c, n=n, scratch=scratch, out=out[i])

    res = {"count": count, "n": n}
    for name, fn in (("reference_abi", ref.enqueue), ("zkp_msm_loop", loop)):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        res[f"{name}_ms"] = round(a.elapsed_time(b) / reps, 3)
    res["reference_abi_window_bits"] = ref.c
    return res


def run_msm_batch(zkp, device, count=32, lo=14, hi=20, seed=2024, reps=3, reference_windows=False,
                  one_window_sweep=True):
    """Batched uneven MSMs over one SRS (sizes 2^U, U uniform in [lo, hi];
    per MSM the scalars are uniform (50%), small < 2^20 (35%) or 90%-sparse
    (15%)): plain per-MSM zkp_msm launches against one zkp_msm_batch pipeline,
    each with the library's default windows and with the learned schedule."""
    import numpy as np

    S, H = zkp.schedule, zkp.host
    rng = np.random.default_rng(seed)
    ns = [1 << int(u) for u in rng.integers(lo, hi + 1, count)]
    mixes = ["uniform" if x < 0.5 else "small" if x < 0.85 else "sparse" for x in rng.random(count)]
    bases, _ = S.bases_with_known_logs(max(ns), seed)
    cols = [S.scalars(n, m, seed + 1 + i) for i, (n, m) in enumerate(zip(ns, mixes))]
    model = S.Model.load()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    learned = [model.pick(S.shape_features(n, count, S.histogram(c))) for n, c in zip(ns, cols)]
    pick_ms = (time.perf_counter() - t0) * 1e3
    default = [S.default_window(n) for n in ns]
    res = {"count": count, "sizes_log2": [n.bit_length() - 1 for n in ns], "mixes": mixes,
           "total_points": int(sum(ns)), "learned_windows": learned, "default_windows": default,
           "schedule_pick_ms": round(pick_ms, 2)}

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / reps

    pickers = [("default", default), ("learned", learned)]
    if reference_windows:
        ref = [H.msm_window_bits(count, n) for n in ns]
        res["reference_windows"] = ref
        pickers.append(("reference_formula", ref))
    for name, ws in pickers:
        scratch = torch.empty(max(zkp.load_library().zkp_msm_scratch_bytes(n, c) for n, c in zip(ns, ws)),
                              dtype=torch.uint8, device=device)
        out = torch.empty((count, 12), dtype=torch.int64, device=device)

        def plain():
            for i, (n, c) in enumerate(zip(ns, ws)):
                H.msm(bases, cols[i], n=n, window_bits=c, scratch=scratch, out=out[i])

        res[f"plain_{name}_ms"] = round(timed(plain), 3)
        del scratch
        n_arr = (ctypes.c_uint32 * count)(*ns)
        c_arr = (ctypes.c_int * count)(*ws)
        need = zkp.load_library().zkp_msm_batch_scratch_bytes(ctypes.addressof(n_arr), ctypes.addressof(c_arr), count)
        if need == 0:  # more than 2^32 sorted entries: not one pipeline
            res[f"batched_{name}_ms"] = None
            continue
        bscr = torch.empty(need, dtype=torch.uint8, device=device)
        bout = torch.empty((count, 12), dtype=torch.int64, device=device)
        res[f"batched_{name}_ms"] = round(timed(lambda: H.msm_batch(bases, cols, ns, ws, scratch=bscr, out=bout)), 3)
        # the result keeps its scratch alive (tens of GB for a 256-MSM pipeline)
        del bscr, bout
    if reference_windows and one_window_sweep:
        # the exhaustive autotuner over one window for the whole pipeline
        tuned = {}
        n_arr = (ctypes.c_uint32 * count)(*ns)
        for c in range(10, 20):
            c_arr = (ctypes.c_int * count)(*([c] * count))
            need = zkp.load_library().zkp_msm_batch_scratch_bytes(ctypes.addressof(n_arr), ctypes.addressof(c_arr),
                                                                   count)
            if need == 0:
                continue
            bscr = torch.empty(need, dtype=torch.uint8, device=device)
            bout = torch.empty((count, 12), dtype=torch.int64, device=device)
            tuned[c] = timed(lambda: H.msm_batch(bases, cols, ns, [c] * count, scratch=bscr, out=bout))
            del bscr, bout
        if tuned:
            best = min(tuned, key=tuned.get)
            res["batched_autotuned_one_window"] = {"window_bits": best, "ms": round(tuned[best], 3),
                                                   "all_ms": {k: round(v, 3) for k, v in sorted(tuned.items())}}
    # one table of the SRS (built once per proving key; the build is timed
    # apart) and one pipeline for the whole batch over it
    nmax = max(ns)
    n_arr = (ctypes.c_uint32 * count)(*ns)
    tc = zkp.load_library().zkp_msm_batch_table_default_window(ctypes.addressof(n_arr), count)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    table = torch.empty(zkp.load_library().zkp_msm_table_bytes(nmax, tc) // 8, dtype=torch.int64, device=device)
    torch.cuda.synchronize()
    a.record()
    H.msm_table_build(bases, nmax, tc, table=table)
    b.record()
    b.synchronize()
    res["table_window_bits"], res["table_build_ms"] = tc, round(a.elapsed_time(b), 2)
    need = zkp.load_library().zkp_msm_batch_table_scratch_bytes(ctypes.addressof(n_arr), count, nmax, tc)
    if need:
        tscr = torch.empty(need, dtype=torch.uint8, device=device)
        tout = torch.empty((count, 12), dtype=torch.int64, device=device)
        res["batched_table_ms"] = round(timed(lambda: H.msm_batch_table(table, nmax, tc, cols, ns, scratch=tscr,
                                                                         out=tout)), 3)
        del tscr, tout
    del table
    if res.get("batched_learned_ms"):
        res["speedup_batched_learned_vs_plain_default"] = round(res["plain_default_ms"] / res["batched_learned_ms"],
                                                                3)
        res["mpts_per_s_batched_learned"] = round(res["total_points"] / res["batched_learned_ms"] / 1e3, 2)
    if res.get("batched_table_ms"):
        res["speedup_batched_table_vs_plain_default"] = round(res["plain_default_ms"] / res["batched_table_ms"], 3)
        res["mpts_per_s_batched_table"] = round(res["total_points"] / res["batched_table_ms"] / 1e3, 2)
    # against the reference host's own plain schedule: one MSM launch per
    # column with its window formula (src/cuda/msm.rs:105)
    if res.get("plain_reference_formula_ms"):
        for k in ("batched_learned_ms", "batched_table_ms"):
            if res.get(k):
                res[f"speedup_{k[:-3]}_vs_plain_reference_formula"] = round(
                    res["plain_reference_formula_ms"] / res[k], 3)
    return res


def msm_uneven(zkp, device, one_window_sweep=True):
    """256 uneven MSMs over one SRS, sizes 2^U with U uniform in [14, 22], the
    mixed scalar distribution of run_msm_batch: plain per-MSM launches and
    one batched pipeline, with the library's windows, the learned schedule
    and the reference host's window formula (src/cuda/msm.rs:105), and one
    pipeline over an SRS table."""
    r = run_msm_batch(zkp, device, count=256, lo=14, hi=22, reps=1, reference_windows=True,
                      one_window_sweep=one_window_sweep)
    r.pop("mixes", None)
    r.pop("sizes_log2", None)
    for k in ("learned_windows", "default_windows", "reference_windows"):
        r.pop(k, None)
    torch.cuda.empty_cache()
    return r


def run_coset_ntt(args):
    """The quotient's coset transform alone: NTT_n of --cols coefficient
    columns of 2^k twisted by (zeta w_N)^i (coset 1 of the 8n domain), one
    zkp_ntt_batch_twisted launch group, Montgomery tables as the proof uses at
    k >= 22.  Prints the device time per launch group and the algorithmic
    GB/s (one read and one write of every column); a bounded case for a
    profiler (8 columns of 2^22: 3 GiB on the device)."""
    torch.cuda.set_device(0)
    P = _prover()
    n = 1 << args.k
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    src = P.rand_fr(args.cols * n, gen).reshape(args.cols, n, 4)
    out = torch.empty_like(src)
    tmp = torch.empty((args.cols * n, 4), dtype=torch.int64, device="cuda")
    tab = P.Tables(args.k)
    sj = P.ZETA * P.omega(args.k + 3) % P.R_MOD
    twist = P.powers(1, sj, n)
    for _ in range(max(3, args.warmup)):
        P.ntt_into(out, src, tab, args.cols, False, in_mul=twist, tmp=tmp)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        P.ntt_into(out, src, tab, args.cols, False, in_mul=twist, tmp=tmp)
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b) / args.steps
    peak, kind = load_peaks()
    gbs = 2 * args.cols * n * 32 / (ms / 1e3) / 1e9
    print(json.dumps({"metric": f"coset NTT of {args.cols} columns of 2^{args.k}", "ms_per_launch_group": round(ms, 3),
                      "algorithmic_gb_per_s": round(gbs, 1), "frac_of_hbm": round(gbs / peak, 4),
                      "peak_kind": kind, "steps": args.steps}))


def run_timeline(args):
    """One proof of the headline workload under CUPTI activity tracing
    (torch.profiler): the device's busy and idle time over the proof, the
    longest idle gaps and every kernel's launches and device time, warm and
    unserialised (ncu's launch list replays each kernel cold)."""
    from torch.profiler import ProfilerActivity, profile

    torch.cuda.set_device(0)
    zkp = importlib.import_module("zkwasm-prover_b200")
    zkp.load_library()
    P = _prover()
    hp = P.HotPath(P.Circuit(_shape(P, args), seed=PIPE_SEED), "batched")
    hp.prove()
    torch.cuda.synchronize()
    # the host's garbage-collection pauses during the traced proof
    gc_pauses, gc_t0 = [], [0.0]

    def on_gc(phase, info):
        if phase == "start":
            gc_t0[0] = time.perf_counter()
        else:
            gc_pauses.append((time.perf_counter() - gc_t0[0], info.get("generation")))

    gc.callbacks.append(on_gc)
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        t0 = time.perf_counter()
        hp.prove()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    gc.callbacks.remove(on_gc)
    iv = sorted((e.time_range.start, e.time_range.end, e.name) for e in prof.events()
                if e.device_type == torch.autograd.DeviceType.CUDA)
    busy, gaps, cur = 0.0, [], None
    for s_, e_, name in iv:
        if cur is None:
            cur = [s_, e_]
        elif s_ > cur[1]:
            busy += cur[1] - cur[0]
            gaps.append((s_ - cur[1], name))
            cur = [s_, e_]
        else:
            cur[1] = max(cur[1], e_)
    busy += cur[1] - cur[0]
    tot = {}
    for s_, e_, name in iv:
        a = tot.setdefault(name.split("(")[0], [0, 0.0])
        a[0] += 1
        a[1] += e_ - s_
    gaps.sort(reverse=True)
    print(json.dumps({"metric": f"k={args.k} proof device timeline (CUPTI)", "wall_s": round(wall, 4),
                      "span_ms": round((iv[-1][1] - iv[0][0]) / 1e3, 2), "busy_ms": round(busy / 1e3, 2),
                      "phases_s": {k_: round(v, 4) for k_, v in hp.phase_s.items()},
                      "longest_gaps_us": [(round(g), nm.split("(")[0]) for g, nm in gaps[:10]],
                      "host_gc_pauses": {"count": len(gc_pauses),
                                         "total_ms": round(1e3 * sum(p for p, _ in gc_pauses), 2),
                                         "longest_ms": round(1e3 * max([p for p, _ in gc_pauses] or [0]), 2)},
                      "kernels": [(k_, n_, round(t_ / 1e3, 2), round(100 * t_ / busy, 1))
                                  for k_, (n_, t_) in sorted(tot.items(), key=lambda x: -x[1][1])]}))


def run_msm_uneven(args):
    torch.cuda.set_device(0)
    zkp = importlib.import_module("zkwasm-prover_b200")
    zkp.load_library()
    r = msm_uneven(zkp, torch.device("cuda", 0))
    print(json.dumps({"metric": "256 uneven MSMs 2^14..2^22 (ms)", "msm_256_uneven": r}))


def run_graph(ph, steps):
    """ms per step of the phase captured once in a CUDA graph and replayed."""
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        ph.step()
    g.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        g.replay()
    b.record()
    b.synchronize()
    del g
    return a.elapsed_time(b) / steps


def run_e2e(ph, steps):
    """Same phase through the C ABI with host buffers: pinned Lagrange columns
    copied in and coefficients copied out every step, overlapped by chunk on
    separate copy streams."""
    n, C, ch = ph.n, ph.C, ph.chunk
    host_in = torch.empty((C * n, 4), dtype=torch.int64, pin_memory=True)
    host_in.copy_(ph.lag)
    host_out = torch.empty((C * n, 4), dtype=torch.int64, pin_memory=True)
    dev_in = torch.empty_like(ph.lag)
    s_h2d, s_cmp, s_d2h = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    nchunks = C // ch

    def one_step():
        ev_in = [torch.cuda.Event() for _ in range(nchunks)]
        ev_cmp = [torch.cuda.Event() for _ in range(nchunks)]
        for i in range(nchunks):
            sl = slice(i * ch * n, (i + 1) * ch * n)
            with torch.cuda.stream(s_h2d):
                dev_in[sl].copy_(host_in[sl], non_blocking=True)
                ev_in[i].record(s_h2d)
        for i in range(nchunks):
            s_cmp.wait_event(ev_in[i])
            ph.run_chunk(i * ch, stream=s_cmp, lag=dev_in)
            ev_cmp[i].record(s_cmp)
            sl = slice(i * ch * n, (i + 1) * ch * n)
            s_d2h.wait_event(ev_cmp[i])
            with torch.cuda.stream(s_d2h):
                host_out[sl].copy_(ph.coeff[sl], non_blocking=True)

    one_step()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(s_h2d)
    s_cmp.wait_stream(s_h2d)
    s_d2h.wait_stream(s_h2d)
    for _ in range(steps):
        one_step()
    s_d2h.wait_stream(s_cmp)
    s_d2h.wait_stream(s_h2d)
    end.record(s_d2h)
    end.synchronize()
    sec = start.elapsed_time(end) / 1e3 / steps
    ok = bool((host_out[: n] == ph.coeff[: n].cpu()).all())
    return {"value": C * ph.bytes_per_column() / sec / 1e9, "unit": "GB/s",
            "h2d_bytes_per_step": C * n * 32, "d2h_bytes_per_step": C * n * 32,
            "ms_per_step": sec * 1e3, "coeff_roundtrip_ok": ok}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_msm_only(args):
    """Single MSMs through zkp_msm (device-resident inputs) at the given sizes;
    one JSON line.  Used for profiling the MSM kernels on their own."""
    torch.cuda.set_device(0)
    zkp = importlib.import_module("zkwasm-prover_b200")
    zkp.load_library()
    sizes = tuple(1 << int(x) for x in args.msm_log_sizes.split(","))
    print(json.dumps({"metric": "MSM Mpts/s", "msm": run_msm(zkp, torch.device("cuda", 0), sizes=sizes,
                                                            reps=max(1, args.steps))}))


def run_rows_only(args):
    """The per-row kernel timings alone (one JSON line), of this library or,
    with --impl reference, of the reference's kernels rebuilt for sm_100a;
    used for profiling those kernels on their own."""
    torch.cuda.set_device(0)
    device = torch.device("cuda", 0)
    zkp = importlib.import_module("zkwasm-prover_b200")
    lib = zkp.load_library()
    peak_hbm, _ = load_peaks()
    mont_rate = calib_mont_rate(zkp, device)
    reps = max(1, args.steps)
    if args.impl == "reference":
        path = os.path.join(ROOT, "oracle", "_ref", "libzkwasm_prover_kernel_ref.so")
        if not os.path.exists(path):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
            return
        rows = run_rows(ctypes.CDLL(path), device, mont_rate, peak_hbm, ours=False, reps=reps)
    else:
        rows = run_rows(lib, device, mont_rate, peak_hbm, reps=reps)
    print(json.dumps({"impl": args.impl, "rows": rows}))


def run_ours(args):
    ws, rank, local = dist_setup()
    device = torch.device("cuda", local)
    zkp = importlib.import_module("zkwasm-prover_b200")
    zkp.load_library()
    ph = ExtendPhase(zkp, device, columns=args.columns, log_n=args.log_n, ext_bits=args.ext_bits,
                     chunk=args.chunk, seed=1 + rank, pair_tables=not args.montgomery_tables)
    nchunks = ph.C // ph.chunk
    for _ in range(args.warmup):
        ph.step()
    torch.cuda.synchronize()
    ev_sets = [[make_event_array(5) for _ in range(nchunks)] for _ in range(args.steps)]
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.4)
    barrier(ws)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for k in range(args.steps):
        ph.step(events=[ev_sets[k][i][1] for i in range(nchunks)])
    end.record()
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop() if clocks else None
    ms = start.elapsed_time(end) / args.steps
    ms = max_over_ranks(ms, ws)
    # the same step captured once as a CUDA graph and replayed (the launches
    # of all chunks as one graph launch); timed the same way, after the eager
    # timed region
    graph_ms = max_over_ranks(run_graph(ph, args.steps), ws)
    # per-stage device time from the events recorded inside the timed region
    stage_ms = [0.0] * 4
    for k in range(args.steps):
        for i in range(nchunks):
            evs = ev_sets[k][i][0]
            for s in range(4):
                stage_ms[s] += evs[s].elapsed_time(evs[s + 1])
    launches = args.steps * nchunks
    stage_ms = [x / launches for x in stage_ms]
    dom = max(range(4), key=lambda s: stage_ms[s])
    peak_hbm, peak_kind = load_peaks()
    total_bytes = ws * ph.C * ph.bytes_per_column()
    value = total_bytes / (ms / 1e3) / 1e9
    # end to end through the C ABI with host buffers, on every rank at once:
    # the whole-job figure is all ranks' bytes over the slowest rank's time
    barrier(ws)
    e2e = run_e2e(ph, max(1, min(args.steps, 3)))
    e2e_ms = max_over_ranks(e2e["ms_per_step"], ws)
    e2e.update({"ms_per_step": e2e_ms, "value": ws * ph.C * ph.bytes_per_column() / (e2e_ms / 1e3) / 1e9})
    # every collective is behind this point: rank 0's remaining work (rates,
    # the CPU baseline, MSMs, rows) waits on no other rank, and with more than
    # one rank it is skipped so that the N-GPU run holds its GPUs only for the
    # phase itself
    extras = ws == 1
    out = None
    if rank == 0:
        mont_rate = calib_mont_rate(zkp, device)
        shoup_rate = calib_shoup_rate(zkp, device)
        # the phase multiplies by table factors: its product form is the one
        # of its tables
        prod_rate = mont_rate if args.montgomery_tables else shoup_rate
        sb, sm = ph.stage_bytes()[dom], ph.stage_mults()[dom]
        achieved = sb / (stage_ms[dom] / 1e3) / 1e9
        # no capture of the extend kernels' DRAM bytes matches their current
        # block order (column-fastest), so none is reported
        traffic = None
        cpu = cpu_baseline_port(args.log_n, args.ext_bits) if extras and not args.no_cpu_baseline else None
        do_msm = extras and not args.no_msm
        do_rows = extras and not args.no_rows
        msm = run_msm(zkp, device) if do_msm else None
        msm_batch = run_msm_batch(zkp, device) if do_msm else None
        msm_columns = ([run_msm_columns(zkp, device), run_msm_columns(zkp, device, count=8, log_n=22, reps=2)]
                       if do_msm else None)
        rows = run_rows(zkp.load_library(), device, mont_rate, peak_hbm) if do_rows else None
        staging = run_staging(zkp, device) if do_rows else None
        out = {
            "metric": f"NTT HBM GB/s: batched iNTT 2^{args.log_n} -> coset NTT 2^{args.log_n + args.ext_bits}, "
                      f"{args.columns} columns",
            "value": round(value, 3),
            "unit": "GB/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "bn254-fr (8x u32 Montgomery)",
            "data": "synthetic, seeded, uniform in [0, 2^253), generated on device",
            "config": {"workload": f"{args.columns} columns x 2^{args.log_n} Lagrange -> iNTT -> coset NTT on "
                                   f"2^{args.log_n + args.ext_bits} (shift 7)",
                       "columns": args.columns, "log_n": args.log_n, "ext_bits": args.ext_bits,
                       "chunk_columns": args.chunk, "parallelism": f"replicas x{ws}",
                       "multiplier_tables": "montgomery" if args.montgomery_tables else "shoup_pairs",
                       "l2": "inputs and outputs (2 GiB in, 18 GiB out per step) exceed L2; no flush needed"},
            "e2e": e2e,
            "graph": {"ms_per_step": round(graph_ms, 3),
                      "value": round(total_bytes / (graph_ms / 1e3) / 1e9, 3), "unit": "GB/s",
                      "launches_per_step": 1},
            # kernels per chunk: inverse pass 1, the fused stage and coset
            # pass 2 (four separate passes without the fused stage)
            "gpu_launches": launches * (3 if ph.fused() else 4),
            "roofline": {
                "bound": "hbm", "achieved": round(achieved, 2), "peak": peak_hbm, "unit": "GB/s",
                "frac": round(achieved / peak_hbm, 4), "traffic": traffic,
                "kernel": ph.stage_names()[dom],
                "peak_kind": peak_kind,
                "note": "integer-pipe bound: see roofline_int",
            },
            "roofline_int": {
                "bound": "int", "unit": "Gmul/s",
                "achieved": round(sm / (stage_ms[dom] / 1e3) / 1e9, 2),
                "peak": round(prod_rate / 1e9, 2),
                "frac": round(sm / (stage_ms[dom] / 1e3) / prod_rate, 4),
                "phase_frac": round(ph.C * ph.mults_per_column() / (ms / 1e3) / prod_rate, 4),
                "peak_kind": ("measured Fr Montgomery products/s (zkp_calib_mont_rate)" if args.montgomery_tables
                              else "measured Fr products by a known factor/s (zkp_calib_shoup_rate)"),
                "montgomery_rate": round(mont_rate / 1e9, 2),
                "known_factor_rate": round(shoup_rate / 1e9, 2),
            },
            "stage_ms": [round(x, 4) for x in stage_ms],
            "cpu_baseline": cpu,
            "msm": msm,
            "msm_batch": msm_batch,
            "msm_columns": msm_columns,
            "rows": rows,
            "staging": staging,
        }
        if clk:
            out["clocks"] = clk
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


def reference_gpu_timings(args):
    """The reference's own CUDA kernels (cuda/bn254.cu + cuda/msm.cu, rebuilt
    unmodified for sm_100a into oracle/_ref/) on the same phase, called the
    way its Rust host calls them: per column ntt (iNTT, src/cuda/ntt.rs:61-93),
    extended_prepare + ntt at the extended size (src/eval_h.rs:255-265), and
    msm + batch_msm_collect (src/cuda/msm.rs:239-455) for single MSMs."""
    path = os.path.join(ROOT, "oracle", "_ref", "libzkwasm_prover_kernel_ref.so")
    if not os.path.exists(path) or not torch.cuda.is_available():
        return {"unavailable": "oracle/_ref not built or no GPU"}
    import numpy as np

    L = ctypes.CDLL(path)
    VP = ctypes.c_void_p
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None

    def tables(log_n, inverse):
        n = 1 << log_n
        w = omega(log_n)
        if inverse:
            w = pow(w, -1, R_MOD)
        om = torch.zeros((n, 4), dtype=torch.int64, device=dev)
        om[:2] = fr_tensor([1, w], dev)
        torch.cuda.synchronize()
        assert L.expand_omega_buffer(p(om), log_n, 1) == 0
        md = min(8, log_n)
        tw = pow(w, n >> md, R_MOD)
        pq = fr_tensor([pow(tw, i, R_MOD) for i in range((1 << md) >> 1)], dev)
        torch.cuda.synchronize()
        return om, pq

    out = {}
    # NTT phase: C columns, iNTT 2^k then zeta-coset extension to 2^(k+e)
    k, e, C = args.log_n, args.ext_bits, args.columns
    n, N = 1 << k, 1 << (k + e)
    om_i, pq_i = tables(k, True)
    om_f, pq_f = tables(k + e, False)
    ninv = fr_tensor([pow(n, -1, R_MOD)], dev)
    zeta = pow(GENERATOR, (R_MOD - 1) // 3, R_MOD)
    cp = fr_tensor([zeta, zeta * zeta % R_MOD], dev)
    lag = random_fr(C * n, 5, dev)
    tmp = torch.empty((n, 4), dtype=torch.int64, device=dev)
    ext = torch.empty((N, 4), dtype=torch.int64, device=dev)
    text = torch.empty((N, 4), dtype=torch.int64, device=dev)
    swap = ctypes.c_bool(False)

    def phase():
        for c in range(C):
            col = lag[c * n:(c + 1) * n]
            assert L.ntt(p(col), p(tmp), p(pq_i), p(om_i), p(ninv), k, 8, ctypes.byref(swap), VP(st)) == 0
            coeff = tmp if swap.value else col
            ext[:n].copy_(coeff)
            assert L.extended_prepare(p(ext), p(cp), 3, n, N, 0, VP(st)) == 0
            assert L.ntt(p(ext), p(text), p(pq_f), p(om_f), None, k + e, 8, ctypes.byref(swap), VP(st)) == 0

    phase()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    phase()
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b)
    out["ntt_phase"] = {"ms_per_step": round(ms, 3),
                        "value": round(C * (3 + (1 << e)) * n * 32 / (ms / 1e3) / 1e9, 3), "unit": "GB/s",
                        "flow": "per column: ntt(iNTT 2^k) -> copy -> extended_prepare(zeta) -> ntt(2^(k+e))"}
    del lag, tmp, ext, text
    # single MSMs
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    res = []
    for nn in (1 << 18, 1 << 22):
        d = O.rand_fr(nn, 901)
        bases = torch.from_numpy(O.g1_gen_bases(d).view(np.int64)).to(dev)
        sc = torch.from_numpy(O.rand_fr(nn, 902).view(np.int64)).to(dev)
        c = 10 + max((nn - 1).bit_length(), 22) - 22
        windows = (254 + c - 1) // c
        bucket = windows << c
        worker = (nn + 63) // 64 * 64 if nn < 128 * 512 else 128 * 512
        curve = torch.empty((bucket + 2 * worker, 12), dtype=torch.int64, device=dev)
        single = nn * windows
        idx = [torch.empty(single, dtype=torch.int32, device=dev) for _ in range(4)]
        sort = torch.empty(3 * single, dtype=torch.int32, device=dev)
        acc = torch.empty(2 * worker, dtype=torch.int32, device=dev)
        ptrs = lambda xs: torch.tensor(xs, dtype=torch.int64, device=dev)
        base = curve.data_ptr()
        ri, nri = ptrs([acc.data_ptr()]), ptrs([acc.data_ptr() + worker * 4])
        ra, nra = ptrs([base + bucket * 96]), ptrs([base + (bucket + worker) * 96])
        bk = ptrs([base])

        def one():
            assert L.msm(p(curve), p(bases), p(sc), p(idx[0]), p(idx[1]), p(idx[2]), p(idx[3]), p(sort), p(acc),
                         nn, windows, c, 64, worker, 3 * single * 4, 1, VP(st)) == 0
            assert L.batch_msm_collect(p(ri), p(ra), p(nri), p(nra), p(bk), worker, windows, c, 1, VP(st)) == 0

        one()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        reps = 3
        for _ in range(reps):
            one()
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) / reps * 1e3
        ok = bool((O.g1_jac_to_aff(curve[0:1].cpu().numpy().view(np.uint64)) == O.msm_known_dlog(d, O.rand_fr(nn, 902))).all())
        res.append({"n": nn, "ms": round(ms, 3), "mpts_per_s": round(nn / ms / 1e3, 2), "window_bits": c,
                    "matches_oracle": ok})
        if True:
            # columns committed together (16 of 2^18, 8 of 2^22), as
            # src/cuda/msm.rs:239-455 issues them: msm per column into its own
            # region, then one batch_msm_collect
            B = 16 if nn == 1 << 18 else 8
            lgB = (B - 1).bit_length()
            c16 = min(lgB, 3) + 10 + max((nn - 1).bit_length(), 22) - 22  # msm.rs:105 for B MSMs
            w16 = (254 + c16 - 1) // c16
            bucket16 = w16 << c16
            region = bucket16 + 2 * worker
            curves = torch.empty((B * region, 12), dtype=torch.int64, device=dev)
            single16 = nn * w16
            idx16 = [torch.empty(single16, dtype=torch.int32, device=dev) for _ in range(4)]
            sort16 = torch.empty(3 * single16, dtype=torch.int32, device=dev)
            accs = [torch.empty(2 * worker, dtype=torch.int32, device=dev) for _ in range(B)]
            cols = [torch.from_numpy(O.rand_fr(nn, 1000 + i).view(np.int64)).to(dev) for i in range(B)]
            cb = curves.data_ptr()
            ri16 = ptrs([a.data_ptr() for a in accs])
            nri16 = ptrs([a.data_ptr() + worker * 4 for a in accs])
            bk16 = ptrs([cb + i * region * 96 for i in range(B)])
            ra16 = ptrs([cb + (i * region + bucket16) * 96 for i in range(B)])
            nra16 = ptrs([cb + (i * region + bucket16 + worker) * 96 for i in range(B)])

            def columns():
                for i in range(B):
                    assert L.msm(VP(cb + i * region * 96), p(bases), p(cols[i]), p(idx16[0]), p(idx16[1]),
                                 p(idx16[2]), p(idx16[3]), p(sort16), p(accs[i]), nn, w16, c16, 64, worker,
                                 3 * single16 * 4, 1, VP(st)) == 0
                assert L.batch_msm_collect(p(ri16), p(ra16), p(nri16), p(nra16), p(bk16), worker, w16, c16, B,
                                           VP(st)) == 0

            columns()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                columns()
            torch.cuda.synchronize()
            out.setdefault("msm_columns", []).append(
                {"count": B, "n": nn, "window_bits": c16,
                 "reference_abi_ms": round((time.perf_counter() - t0) / reps * 1e3, 3)})
            del curves, idx16, sort16, accs, cols
        del bases, sc, curve, idx, sort, acc
    out["msm"] = res
    peak, _ = load_peaks()
    out["rows"] = run_rows(L, dev, None, peak, ours=False)
    return out


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # The reference's CPU path (halo2 best_fft) is Rust and absent here; its
    # algorithm is timed as the oracle's C restatement on all host cores.
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_baseline_port(args.log_n, args.ext_bits)
    vals = [cpu_baseline_port(args.log_n, args.ext_bits) for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[0])
    cb["value"] = v
    out = {
        "impl": "reference",
        "metric": f"NTT HBM GB/s: batched iNTT 2^{args.log_n} -> coset NTT 2^{args.log_n + args.ext_bits}, "
                  f"{args.columns} columns",
        "value": round(v, 4), "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round((3 + (1 << args.ext_bits)) * (1 << args.log_n) * 32 / (v * 1e9) * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bn254-fr",
        "data": "synthetic, seeded",
        "config": {"workload": f"{args.columns} columns x 2^{args.log_n} Lagrange -> iNTT -> coset NTT on "
                               f"2^{args.log_n + args.ext_bits} (shift 7)", "sample": "one column per step"},
        "cpu_baseline": cb,
        "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_gpu:
        out["reference_gpu_sm100a"] = reference_gpu_timings(args)
    print(json.dumps(out))


# ------------------------------------------------------------------ proof hot path (headline)

PIPE_SEED = 1


def _prover():
    return importlib.import_module("zkwasm-prover_b200.prover")


def _shape(P, args):
    return P.shplonk_shape(args.k) if args.config == "e" else P.gwc_shape(args.k)


def proof_digest(proof) -> str:
    """SHA-256 of every commitment (affine) and evaluation of a proof, in
    transcript order: equal digests mean bit-identical proofs."""
    import hashlib

    h = hashlib.sha256()
    for name, pts in proof["commitments"]:
        h.update(name.encode())
        for x, y in pts:
            h.update(x.to_bytes(32, "little") + y.to_bytes(32, "little"))
    for e in proof["evals"]:
        h.update(int(e).to_bytes(32, "little"))
    return h.hexdigest()


def _time_proofs(hp, steps, warmup, ws, clocks=None, profile=False):
    """W untimed proofs, then exactly K timed ones bracketed by a barrier and
    a device synchronisation; CUDA events on the proving stream; seconds per
    proof, max over ranks."""
    for _ in range(warmup):
        proof = hp.prove()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.4)
    barrier(ws)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if profile:
        torch.cuda.profiler.start()
    a.record()
    for _ in range(steps):
        proof = hp.prove()
    b.record()
    torch.cuda.synchronize()
    if profile:
        torch.cuda.profiler.stop()
    barrier(ws)
    clk = clocks.stop() if clocks else None
    sec = max_over_ranks(a.elapsed_time(b) / 1e3 / steps, ws)
    return sec, proof, clk


def _e2e_proofs(P, hp, circuit, steps, ws):
    """The same proof end to end from HOST buffers: every step copies the
    witness (advice and instance Lagrange columns) from pinned host memory
    into the device columns (the advice in groups of columns, overlapped with
    the commitments and transforms of the groups already copied), proves, and
    reads the proof (every commitment and evaluation) back to the host."""
    host_adv = torch.empty(circuit.advice.shape, dtype=torch.int64, pin_memory=True)
    host_adv.copy_(circuit.advice)
    host_inst = torch.empty(circuit.instance.shape, dtype=torch.int64, pin_memory=True)
    host_inst.copy_(circuit.instance)
    h2d = (host_adv.numel() + host_inst.numel()) * 8

    stage = P.HostStage(host_adv, circuit.advice)

    def one():
        # the instance column first, the advice columns in groups while phase
        # 1 commits and transforms the groups already on the device
        circuit.instance.copy_(host_inst, non_blocking=True)
        return hp.prove(stage=stage)

    proof = one()
    torch.cuda.synchronize()
    barrier(ws)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        proof = one()
    b.record()
    torch.cuda.synchronize()
    sec = max_over_ranks(a.elapsed_time(b) / 1e3 / steps, ws)
    # the proof comes back as affine commitments (96-byte Jacobian points
    # read per MSM) and evaluations (32 bytes each)
    d2h = sum(len(p) for _, p in proof["commitments"]) * 96 + len(proof["evals"]) * 32
    del host_adv, host_inst
    return {"value": round(sec, 4), "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": steps, "digest": proof_digest(proof)}


def cpu_baseline_pipeline(counts, k, reps=1):
    """The oracle (C restatement, OpenMP on all host cores) on a bounded
    sample of the proof's work: one MSM of 2^16 points (Pippenger) and one
    NTT of 2^20 points, scaled to the proof's MSM and NTT counts at 2^k by
    the number of points (n log n for the NTTs).  The quotient's elementwise
    work and the host steps are left out, so the estimate is a lower bound."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    m_log, t_log = 16, 20
    d = O.rand_fr(1 << m_log, 3)
    sc = O.rand_fr(1 << m_log, 4)
    bases = O.g1_gen_bases(d)
    a = O.rand_fr(1 << t_log, 5)
    t0 = time.perf_counter()
    for _ in range(reps):
        O.msm(bases, sc)
    t_msm = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        O.ntt(a, t_log)
    t_ntt = (time.perf_counter() - t0) / reps
    n = 1 << k
    est = counts["msm"] * t_msm * n / (1 << m_log) + counts["ntt_n"] * t_ntt * (n * k) / ((1 << t_log) * t_log)
    return {"value": round(est, 2), "unit": "s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"one MSM of 2^{m_log} points ({t_msm:.2f} s) and one NTT of 2^{t_log} ({t_ntt:.2f} s) on "
                      f"the oracle, scaled to {counts['msm']} MSMs and {counts['ntt_n']} NTTs of 2^{k} "
                      f"(elementwise quotient work and host steps not counted)"}


def run_pipeline(args):
    ws, rank, local = dist_setup()
    device = torch.device("cuda", local)
    zkp = importlib.import_module("zkwasm-prover_b200")
    zkp.load_library()
    P = _prover()
    shape = _shape(P, args)
    circuit = P.Circuit(shape, seed=PIPE_SEED + rank)
    hp = P.HotPath(circuit, "batched")
    hp.ntt_events = []
    lib = zkp.load_library()
    # library entry-point calls of one proof (each launches one or more of
    # this library's kernels; the MSM pipelines and NTTs several)
    lib.calls = {}
    hp.prove()
    calls_per_proof = dict(lib.calls)
    lib.calls = None
    clocks = ClockSampler(local) if rank == 0 else None
    sec, proof, clk = _time_proofs(hp, args.steps, args.warmup, ws, clocks, profile=args.profile_range)
    digest = proof_digest(proof)
    phases = dict(hp.phase_s)
    learned_picks = dict(hp.learned_picks)
    # the dominant kernel: the coset transforms of the quotient (two NTT
    # passes per launch group), timed by the events recorded inside the
    # timed region (the last `steps` proofs' groups)
    evs = hp.ntt_events
    per_proof = len(evs) // (args.steps + args.warmup + 1)
    timed = evs[-per_proof * args.steps:]
    ntt_ms = sum(e[0].elapsed_time(e[1]) for e in timed)
    ntt_cols = sum(e[2] for e in timed)
    hp.ntt_events = None
    # the fused constraint pass against the reference's kernels one family at
    # a time on the same coset (and both against the proof's h)
    fused_vs_separate = hp.coset_fused_vs_separate()
    counts = hp.counts()
    memory = {"pk_coset_cache_gib": round(hp.pk_cache_bytes / 2 ** 30, 1),
              "peak_allocated_gib": round(torch.cuda.max_memory_allocated() / 2 ** 30, 1),
              "device_gib": round(torch.cuda.get_device_properties(device).total_memory / 2 ** 30, 1)}
    e2e = _e2e_proofs(P, hp, circuit, max(1, min(args.steps, 3)), ws)
    launches = _launch_count(calls_per_proof, shape)
    del hp
    gc.collect()
    torch.cuda.empty_cache()
    # the plain schedule (the reference host's one-kernel-per-column calls
    # through this library) on the same circuit, for the batched/plain ratio
    plain = None
    if not args.no_plain:
        hpp = P.HotPath(circuit, "plain")
        psec, pproof, _ = _time_proofs(hpp, max(1, min(args.steps, 3)), 1, ws)
        plain = {"s_per_proof": round(psec, 4), "phases_s": {k_: round(v, 4) for k_, v in hpp.phase_s.items()},
                 "steps": max(1, min(args.steps, 3)), "same_proof_as_batched": proof_digest(pproof) == digest}
        del hpp
        gc.collect()
        torch.cuda.empty_cache()
    out = None
    if rank == 0:
        n = shape.n
        peak_hbm, peak_kind = load_peaks()
        mont_rate = calib_mont_rate(zkp, device)
        # per launch group: read 32 coefficient columns, write 32 coset columns
        # (algorithmic bytes; the intermediate pass round trip is not counted),
        # (n/2) log n butterfly products + n twist products per column
        groups = len(timed)
        avg_ms = ntt_ms / max(1, groups)
        cols_per = ntt_cols / max(1, groups)
        bytes_per = cols_per * 2 * n * 32
        mults_per = cols_per * (n // 2 * shape.k + n)
        achieved = bytes_per / (avg_ms / 1e3) / 1e9
        extra = {}
        if ws == 1 and not args.no_extras:
            extra = pipeline_extras(args, P, zkp, device)
        cpu = cpu_baseline_pipeline(counts, shape.k) if ws == 1 and not args.no_cpu_baseline else None
        out = {
            "metric": f"k={shape.k} proof hot-path wall time (s/proof), batched+learned schedule",
            "value": round(sec, 4),
            "unit": "s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(sec * 1e3, 2),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "bn254-fr / bn254-fq (8x u32 Montgomery)",
            "data": "synthetic seeded circuit generated on the device; witness satisfies every constraint",
            "config": {"workload": ("SHPLONK proof hot path, " if args.config == "e" else "GWC proof hot path, ") +
                                   f"k={shape.k}, {shape.advice} advice, {shape.fixed} fixed, 1 instance, "
                                   f"{shape.lookups} logup lookups, {shape.shuffles} shuffles, {shape.perm} "
                                   f"permutation columns, degree {shape.degree} (extended domain "
                                   f"2^{shape.k + shape.ext_bits})",
                       "schedule": "batched+learned: MSM pipelines of 8 over SRS tables or plain bases as the "
                                   "learned table-or-plain model picks, batched NTTs, per-coset fused quotient "
                                   "(zkp_eval_h_fused) and coset combine, batched evaluations",
                       "parallelism": f"replicas x{ws}", "proofs_per_s": round(ws / sec, 4),
                       "l2": "every step streams > 100 GB of columns through HBM; no flush needed",
                       "transcript": "seeded BLAKE2b stand-in over every commitment and evaluation"},
            "proof_digest": digest,
            "phases_s": {k_: round(v, 4) for k_, v in phases.items()},
            "learned_msm_picks_per_proof": learned_picks,
            "quotient_coset_fused_vs_separate": fused_vs_separate,
            "plain": plain,
            "speedup_vs_plain": round(plain["s_per_proof"] / sec, 3) if plain else None,
            "e2e": e2e,
            "gpu_launches": launches * args.steps,
            "library_calls_per_proof": calls_per_proof,
            "roofline": {
                "bound": "hbm", "achieved": round(achieved, 2), "peak": peak_hbm, "unit": "GB/s",
                "frac": round(achieved / peak_hbm, 4), "traffic": coset_traffic(cols_per, shape.k),
                "kernel": "ntt_pass_kernel via zkp_ntt_batch_twisted (coset transforms of the quotient)",
                "launch_groups": groups, "avg_group_ms": round(avg_ms, 4), "columns_per_group": cols_per,
                "peak_kind": peak_kind, "note": "integer-pipe bound: see roofline_int"},
            "roofline_int": {
                "bound": "int", "unit": "Gmul/s",
                "achieved": round(mults_per / (avg_ms / 1e3) / 1e9, 2),
                "peak": round(mont_rate / 1e9, 2),
                "frac": round(mults_per / (avg_ms / 1e3) / mont_rate, 4),
                "peak_kind": "measured Fr Montgomery products/s (zkp_calib_mont_rate)"},
            "counts": counts,
            "memory": memory,
            "cpu_baseline": cpu,
        }
        out.update(extra)
        if clk:
            out["clocks"] = clk
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


# kernels each library entry point launches at the proof's sizes (2^22, the
# batched MSM pipeline over a table), counted from the ncu launch list of one
# proof (1089 launches of this library's kernels); entry points not listed
# launch one kernel
KERNELS_PER_CALL = {"zkp_msm_batch_table": 14, "zkp_ntt_batch_twisted": 2, "zkp_ntt_batch": 2, "ntt": 2,
                    "calc_m": 2, "prepare_table_lookup": 1, "logup_sum_input_inv": 1, "eval_logup_z_compose": 6,
                    "zkp_permutation_z": 4, "zkp_shuffle_z": 4, "zkp_powers": 2, "zkp_poly_divide_linear": 9,
                    "zkp_poly_eval_batch": 2}
NO_KERNEL = {"zkp_msm_batch_table_scratch_bytes", "zkp_scan_scratch_elems", "zkp_poly_divide_scratch_elems",
             "zkp_poly_eval_batch_scratch_elems", "zkp_msm_batch_table_default_window"}


def coset_traffic(columns, log_n):
    """DRAM bytes of one coset-transform launch group of `columns` columns of
    2^log_n, from the committed ncu capture (profiles/coset_ntt_traffic.json,
    per column), or None for another size or when ntt.cu no longer hashes to
    the captured source (a stale figure is not reported)."""
    import hashlib

    prof = os.path.join(ROOT, "profiles", "coset_ntt_traffic.json")
    src = os.path.join(ROOT, "zkwasm-prover_b200", "csrc", "ntt.cu")
    if not (os.path.exists(prof) and os.path.exists(src)):
        return None
    with open(prof) as f:
        d = json.load(f)
    if d.get("log_n") != log_n:
        return None
    with open(src, "rb") as f:
        if hashlib.sha256(f.read()).hexdigest() != d.get("source_sha256"):
            return None
    return round(d["bytes_per_column"] * columns)


def _launch_count(calls, shape):
    """This library's kernels launched by one proof of the batched schedule,
    from its entry-point calls."""
    return sum(cnt * KERNELS_PER_CALL.get(name, 1) for name, cnt in calls.items() if name not in NO_KERNEL)


def pipeline_extras(args, P, zkp, device):
    """Smaller companions of the headline on one GPU: the GWC proof of
    k = 20 (40 advice columns, degree 4) in both schedules, and the batched
    NTT phase of 64 columns of 2^20 extended to 2^23, and 256 uneven MSMs
    (2^14..2^22) plain and batched."""
    out = {}
    if args.config == "e":
        shape = P.gwc_shape(20)
        c = P.Circuit(shape, seed=PIPE_SEED)
        res = {}
        for sched in ("batched", "plain"):
            hp = P.HotPath(c, sched)
            sec, proof, _ = _time_proofs(hp, 3, 1, 1)
            res[sched] = {"s_per_proof": round(sec, 4), "digest": proof_digest(proof)}
            del hp
            gc.collect()
        res["speedup_vs_plain"] = round(res["plain"]["s_per_proof"] / res["batched"]["s_per_proof"], 3)
        res["same_proof"] = res["plain"]["digest"] == res["batched"]["digest"]
        out["gwc_proof_k20"] = res
        del c
        torch.cuda.empty_cache()
    ph = ExtendPhase(zkp, device, columns=64, log_n=20, ext_bits=3, chunk=8, seed=1)
    for _ in range(2):
        ph.step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(3):
        ph.step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / 3
    out["ntt_phase_64x2^20_to_2^23"] = {"ms_per_step": round(ms, 3), "unit": "GB/s",
                                 "value": round(64 * ph.bytes_per_column() / (ms / 1e3) / 1e9, 2),
                                 "workload": "64 columns x 2^20 Lagrange -> iNTT -> coset NTT on 2^23 (shift 7)"}
    del ph
    torch.cuda.empty_cache()
    out["msm_256_uneven_2^14..2^22"] = msm_uneven(zkp, device, one_window_sweep=False)
    return out


def run_pipeline_reference(args):
    """The reference arm: the proof's work on the host cores through the
    oracle (the reference's CPU path is Rust and halo2, absent here), as an
    estimate from a bounded sample; and, as an extra key, the same proof
    through the reference's own CUDA kernels rebuilt for sm_100a (its host's
    one-kernel-per-column schedule; the CPU steps of its host through the
    oracle)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    torch.cuda.set_device(0)
    P = _prover()
    shape = _shape(P, args)
    counts = {"msm": 0, "ntt_n": 0}
    # the proof's unit counts in the reference's own schedule
    s = shape
    E = 1 << s.ext_bits
    counts["msm"] = (s.advice + 1) + s.lookups + (s.perm_chunks + s.shuffles) + (s.lookups + 1) + (s.degree - 1) + (
        2 if s.multiopen == "shplonk" else 3)
    ext_cols = (5 * s.gates + s.gates) + 2 + s.perm_chunks + 2 * s.perm + 4 * s.lookups + 3 * s.shuffles
    counts["ntt_n"] = (s.advice + 1) + 2 * s.lookups + s.perm_chunks + s.shuffles + (ext_cols + 1) * E * (
        s.k + s.ext_bits) // s.k + 4
    vals = []
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_baseline_pipeline(counts, shape.k)
    for _ in range(max(1, min(args.steps, 3))):
        vals.append(cpu_baseline_pipeline(counts, shape.k))
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[0])
    cb["value"] = v
    out = {
        "impl": "reference",
        "metric": f"k={shape.k} proof hot-path wall time (s/proof), batched+learned schedule",
        "value": v, "unit": "s", "n_gpus": ws, "steps": len(vals), "warmup": min(args.warmup, 1),
        "ms_per_step": round(v * 1e3, 1), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "bn254-fr", "data": "synthetic, seeded",
        "config": {"workload": f"k={shape.k} {'SHPLONK' if args.config == 'e' else 'GWC'} proof hot path",
                   "sample": cb["sample"]},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_gpu:
        out["reference_gpu_sm100a"] = reference_pipeline_gpu(P, shape)
    print(json.dumps(out))


def reference_pipeline_gpu(P, shape):
    """The proof through the reference's kernels (oracle/_ref), plain schedule."""
    path = os.path.join(ROOT, "oracle", "_ref", "libzkwasm_prover_kernel_ref.so")
    if not os.path.exists(path) or not torch.cuda.is_available():
        return {"unavailable": "oracle/_ref not built or no GPU"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from host_work import OracleHostWork
    import ref_cases

    c = P.Circuit(shape, seed=PIPE_SEED)
    hp = P.HotPath(c, "plain", symbols=ref_cases.load_ref(), host_work=OracleHostWork())
    t0 = time.perf_counter()
    proof = hp.prove()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    return {"proof_s": round(sec, 3), "phases_s": {k: round(v, 4) for k, v in hp.phase_s.items()},
            "proof_digest": proof_digest(proof),
            "flow": "the reference host's schedule (src/lib.rs, src/eval_h.rs, src/multiopen.rs) through the "
                    "reference's 27 symbols; permutation/shuffle products and multi-open divisions on the host "
                    "(oracle C, as the reference runs them on its CPU); one proof after none untimed"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--columns", type=int, default=64)
    ap.add_argument("--log-n", type=int, default=20)
    ap.add_argument("--ext-bits", type=int, default=3)
    ap.add_argument("--chunk", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--montgomery-tables", action="store_true",
                    help="multiply by Montgomery-form twiddles instead of (w, w') pairs")
    ap.add_argument("--no-msm", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--no-rows", action="store_true", help="skip the per-row kernel timings")
    ap.add_argument("--msm-only", action="store_true", help="time only single MSMs (sizes from --msm-log-sizes)")
    ap.add_argument("--msm-log-sizes", default="18,22")
    ap.add_argument("--msm-uneven", action="store_true", help="256 uneven MSMs 2^14..2^22 (about a minute)")
    ap.add_argument("--rows-only", action="store_true",
                    help="time only the per-row kernels (with --impl reference: the reference's kernels)")
    ap.add_argument("--ntt-phase", action="store_true",
                    help="the batched NTT phase as the headline (64 columns of 2^20 -> 2^23)")
    ap.add_argument("--timeline", action="store_true",
                    help="one proof under CUPTI tracing: device busy time and per-kernel device time")
    ap.add_argument("--coset-ntt", action="store_true",
                    help="time only the quotient's coset transform (--cols columns of 2^--k)")
    ap.add_argument("--cols", type=int, default=8)
    ap.add_argument("--config", default="e", choices=["d", "e"],
                    help="proof hot path: e = SHPLONK k = 22, 120 advice, degree 9; d = GWC k = 20, 40 advice, degree 4")
    ap.add_argument("--k", type=int, default=None)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-schedule comparison")
    ap.add_argument("--no-extras", action="store_true", help="skip the k = 20 GWC proof and the NTT phase companions")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the timed proofs with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.k is None:
        args.k = 22 if args.config == "e" else 20
    if args.rows_only:
        run_rows_only(args)
    elif args.ntt_phase and args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference":
        run_pipeline_reference(args)
    elif args.msm_only:
        run_msm_only(args)
    elif args.msm_uneven:
        run_msm_uneven(args)
    elif args.coset_ntt:
        run_coset_ntt(args)
    elif args.timeline:
        run_timeline(args)
    elif args.ntt_phase:
        run_ours(args)
    else:
        run_pipeline(args)


if __name__ == "__main__":
    main()
