"""The proving hot path of one proof, phase by phase, through this library.

This drives the library in the order the reference's prover issues its GPU
work (src/lib.rs:205-1194; quotient src/eval_h.rs:410-1199; multi-open
src/multiopen.rs), over a seeded synthetic circuit:

  1. advice and instance commitments (MSM over the Lagrange SRS) and their
     inverse NTTs                                       src/lib.rs:297-366
  2. lookup multiplicities m (prepare_table_lookup, calc_m) and their
     commitments                                        src/lib.rs:390-528
  3. logup sums z, permutation and shuffle grand products, their
     commitments (z of lookups and the random polynomial over the
     coefficient SRS)                                   src/lib.rs:530-977
  4. the quotient h on the extended domain, divided by Z_H, its
     coefficients and the commitments of its pieces     src/eval_h.rs:410-586
  5. evaluations of every queried polynomial at x, wx, w^-(b+1) x
                                                        src/lib.rs:1024-1090
  6. multi-open: SHPLONK (src/multiopen.rs:283-547) or GWC (:63-170).

Challenges come from a stand-in transcript (BLAKE2b over a seed and every
commitment and evaluation so far, reduced mod r), since the halo2 transcript is
not in the reference tree; every challenge therefore depends on every earlier
result, as in the real prover.

Two schedules run the same proof:

* ``plain``   - the reference host's schedule through the reference-compatible
  symbols only: one msm() per column with the reference's window rule and
  scratch sizing, then batch_msm_collect; one ntt() per column; every
  quotient column extended to the whole 2^(k+e) domain, one kernel per
  constraint family (src/eval_h.rs).  The symbols may come from this library
  or from any library with the reference's ABI.  The steps the reference runs
  on the CPU (permutation and shuffle products, the multi-open divisions) go
  through ``host_work``: by default this library's device entry points.
* ``batched`` - whole phases per launch: MSM pipelines over tables of the SRS
  (zkp_msm_batch_table), batched NTTs, the quotient per coset of the
  extended domain with every constraint in one fused pass (zkp_eval_h_fused)
  and one radix-E combine (zkp_coset_combine), batched evaluations and the
  multi-open divisions on the device.

Both give the same commitments and evaluations, bit for bit.
"""
from __future__ import annotations

import ctypes
import hashlib
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import abi
from . import host as H

# ---------------------------------------------------------------- field constants (public BN254 parameters)

R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
Q_MOD = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
GENERATOR = 7
TWO_ADICITY = 28
# halo2's DELTA = GENERATOR^(2^S) (src/permutation.rs:51, 94) and ZETA, the
# cube root of unity of the extended-domain coset (src/eval_h.rs:620-623;
# halo2curves' value, equal to the GLV lambda of G1)
DELTA = pow(GENERATOR, 1 << TWO_ADICITY, R_MOD)
ZETA = 0x30644E72E131A029048B6E193FD84104CC37A73FEC2BC5E9B8CA0B2D36636F23
MONT_R = (1 << 256) % R_MOD


def omega(log_n: int) -> int:
    """Primitive 2^log_n-th root of unity: ROOT_OF_UNITY squared S - log_n
    times (src/profile.rs:193-196)."""
    w = pow(GENERATOR, (R_MOD - 1) >> TWO_ADICITY, R_MOD)
    for _ in range(log_n, TWO_ADICITY):
        w = w * w % R_MOD
    return w


def limbs(x: int, mont=True) -> list:
    v = (x % R_MOD) * MONT_R % R_MOD if mont else x
    return [(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)]


def _to_device(h: torch.Tensor, device) -> torch.Tensor:
    """Host tensor -> device through pinned memory, without waiting for the
    work queued on the stream (a pageable copy would; the caching host
    allocator keeps the pinned block until the copy has run)."""
    if torch.device(device).type != "cuda":
        return h.to(device)
    return h.pin_memory().to(device, non_blocking=True)


def fr_tensor(xs, device="cuda") -> torch.Tensor:
    """Python ints -> (len, 4) int64 Montgomery-form tensor."""
    a = np.array([limbs(int(x)) for x in xs], dtype=np.uint64).reshape(-1, 4)
    return _to_device(torch.from_numpy(a.view(np.int64)), device)


def fr_ints(t: torch.Tensor) -> list:
    a = t.detach().cpu().contiguous().numpy().view(np.uint64).reshape(-1, 4)
    rinv = pow(MONT_R, -1, R_MOD)
    return [(int(r[0]) | int(r[1]) << 64 | int(r[2]) << 128 | int(r[3]) << 192) * rinv % R_MOD for r in a]


def jac_to_affine(rows) -> list:
    """Jacobian (X, Y, Z) in Montgomery Fq, 12 words each -> affine (x, y) ints
    ((0, 0) for the identity)."""
    a = np.asarray(rows, dtype=np.uint64).reshape(-1, 12)
    rinv = pow((1 << 256) % Q_MOD, -1, Q_MOD)
    out = []
    for r in a:
        v = [(int(r[4 * j]) | int(r[4 * j + 1]) << 64 | int(r[4 * j + 2]) << 128 | int(r[4 * j + 3]) << 192) * rinv
             % Q_MOD for j in range(3)]
        x, y, z = v
        if z == 0:
            out.append((0, 0))
            continue
        zi = pow(z, -1, Q_MOD)
        zi2 = zi * zi % Q_MOD
        out.append((x * zi2 % Q_MOD, y * zi2 * zi % Q_MOD))
    return out


class Transcript:
    """Stand-in for the halo2 transcript: each challenge is BLAKE2b of the seed,
    everything absorbed so far and a counter, reduced mod r."""

    def __init__(self, seed: int):
        self.h = hashlib.blake2b(b"zkwasm-prover_b200 hot path" + seed.to_bytes(8, "little"), digest_size=64)
        self.count = 0

    def points(self, pts):
        for x, y in pts:
            self.h.update(x.to_bytes(32, "little") + y.to_bytes(32, "little"))

    def scalars(self, xs):
        for x in xs:
            self.h.update(int(x).to_bytes(32, "little"))

    def challenge(self) -> int:
        self.count += 1
        h = self.h.copy()
        h.update(b"challenge" + self.count.to_bytes(4, "little"))
        c = int.from_bytes(h.digest(), "little") % R_MOD
        self.h.update(c.to_bytes(32, "little"))
        return c


# ---------------------------------------------------------------- circuit shape


@dataclass
class Shape:
    """Column counts of the synthetic circuit (gwc_shape, shplonk_shape): one
    degree-4 gate q (a b c + d) - e = 0 per group of five advice columns with its
    own selector, logup lookups of single advice columns (values < 2^16) into a
    2^16 range table, shuffles of advice column pairs, copy-constraint cycles
    over the permutation columns, `blinding` blinding rows."""
    k: int
    advice: int
    fixed: int
    lookups: int
    shuffles: int
    perm: int
    degree: int
    blinding: int = 4
    instance_rows: int = 8
    multiopen: str = "shplonk"

    @property
    def n(self):
        return 1 << self.k

    @property
    def usable(self):
        return self.n - (self.blinding + 1)

    @property
    def gates(self):
        return (self.advice - self.lookups - 2 * self.shuffles) // 5

    @property
    def chunk_len(self):
        return self.degree - 2

    @property
    def ext_bits(self):
        return max(1, math.ceil(math.log2(self.degree - 1)))

    @property
    def perm_chunks(self):
        return (self.perm + self.chunk_len - 1) // self.chunk_len


def gwc_shape(k=20):
    """GWC proof, k = 20: 40 advice, 10 fixed, 1 instance column, 6 lookups,
    2 shuffles, 20 permutation columns, degree 4 (extended domain 4n)."""
    return Shape(k=k, advice=40, fixed=10, lookups=6, shuffles=2, perm=20, degree=4, multiopen="gwc")


def shplonk_shape(k=22):
    """SHPLONK proof, k = 22: 120 advice, 30 fixed, 24 lookups, 4 shuffles, 60
    permutation columns, quotient degree 8 (extended domain 8n = 2^25)."""
    return Shape(k=k, advice=120, fixed=30, lookups=24, shuffles=4, perm=60, degree=9, multiopen="shplonk")


# ---------------------------------------------------------------- device helpers


def lib():
    return abi.load_library()


def _st(stream=None):
    return H.stream_handle(stream)


def _p(t):
    return 0 if t is None else t.data_ptr()


def rand_fr(n: int, gen: torch.Generator, device="cuda") -> torch.Tensor:
    """Seeded uniform values below 2^253 (all below r), Montgomery form."""
    t = torch.randint(-(2 ** 63), 2 ** 63 - 1, (n, 4), dtype=torch.int64, device=device, generator=gen)
    t[:, 3] &= (1 << 61) - 1
    abi.check(lib().zkp_fr_to_mont(t.data_ptr(), t.data_ptr(), n, _st()), "zkp_fr_to_mont")
    return t


def small_fr(vals: torch.Tensor) -> torch.Tensor:
    """Non-negative int64 values -> Montgomery-form Fr."""
    t = torch.zeros((vals.shape[0], 4), dtype=torch.int64, device=vals.device)
    t[:, 0] = vals
    abi.check(lib().zkp_fr_to_mont(t.data_ptr(), t.data_ptr(), t.shape[0], _st()), "zkp_fr_to_mont")
    return t


def field_op(res, l, r, op, n, l_c=None, r_c=None, l_rot=0, r_rot=0, sym=None, stream=None):
    L = sym or lib()
    abi.check(L.field_op(_p(res), _p(l), l_rot, _p(l_c), _p(r), r_rot, _p(r_c), n, op, _st(stream)), "field_op")


def ptr_array(ptrs, device="cuda") -> torch.Tensor:
    return _to_device(torch.tensor([int(p) for p in ptrs], dtype=torch.int64), device)


def omega_table(sym, w: int, log_n: int, may_bit_reversed: int) -> torch.Tensor:
    """generate_omega_buffers (src/cuda/ntt.rs:15-34) through `sym`: [1, w]
    uploaded, then expand_omega_buffer."""
    buf = torch.zeros((1 << log_n, 4), dtype=torch.int64, device="cuda")
    buf[:2] = fr_tensor([1, w])
    torch.cuda.synchronize()
    abi.check(sym.expand_omega_buffer(buf.data_ptr(), log_n, may_bit_reversed), "expand_omega_buffer")
    torch.cuda.synchronize()
    return buf


class Tables:
    """Twiddle tables of one domain size, built by the library `sym` the way
    the reference host builds them (src/cuda/ntt.rs:15-59): the ntt() tables
    of w and w^-1 (whatever layout that library's expand_omega_buffer writes
    for may_bit_reversed = 1) with their pq radix tables, the natural w^i table
    (may_bit_reversed = 0) that the multi-open kernels read, and n^-1."""

    def __init__(self, log_n: int, sym=None):
        sym = sym or lib()
        self.log_n = log_n
        n = 1 << log_n
        w = omega(log_n)
        wi = pow(w, -1, R_MOD)
        self.w = w
        self.tw = omega_table(sym, w, log_n, 1)
        self.tw_inv = omega_table(sym, wi, log_n, 1)
        self.natural = omega_table(sym, w, log_n, 0)
        self.n_inv = fr_tensor([pow(n, -1, R_MOD)])
        max_deg = min(8, log_n)
        self.pq = fr_tensor([pow(pow(w, n >> max_deg, R_MOD), i, R_MOD) for i in range(max(1, (1 << max_deg) >> 1))])
        self.pq_inv = fr_tensor([pow(pow(wi, n >> max_deg, R_MOD), i, R_MOD) for i in range(max(1, (1 << max_deg) >> 1))])


def ntt_raw(sym, s_buf, tmp_buf, tables: Tables, inverse: bool, divisor=None, stream=None):
    """ntt_raw (src/cuda/ntt.rs:61-93) through `sym`; the result ends in s_buf."""
    swap = ctypes.c_bool(False)
    abi.check(sym.ntt(s_buf.data_ptr(), tmp_buf.data_ptr(), (tables.pq_inv if inverse else tables.pq).data_ptr(),
                      (tables.tw_inv if inverse else tables.tw).data_ptr(), _p(divisor), tables.log_n, 8,
                      ctypes.addressof(swap), _st(stream)), "ntt")
    if swap.value:
        s_buf.copy_(tmp_buf)


def ntt_cols(buf, tables: Tables, ncols: int, inverse: bool, tmp=None, stream=None):
    """In-place (through tmp) batched NTT / iNTT of ncols contiguous columns."""
    n = 1 << tables.log_n
    tmp = torch.empty_like(buf) if tmp is None else tmp
    res = ctypes.c_int(0)
    abi.check(lib().zkp_ntt_batch(buf.data_ptr(), tmp.data_ptr(), (tables.tw_inv if inverse else tables.tw).data_ptr(),
                                  tables.n_inv.data_ptr() if inverse else 0, tables.log_n, ncols, n,
                                  ctypes.addressof(res), _st(stream)), "zkp_ntt_batch")
    if res.value:
        buf.copy_(tmp)


NTT_CHUNK = 32
MSM_BATCH = 8


def ntt_into(out, src, tables: Tables, ncols: int, inverse: bool, in_mul=None, tmp=None, stream=None, events=None):
    """Out-of-place batched transform of ncols contiguous columns, NTT_CHUNK
    columns per launch: out = NTT(src * in_mul) (or iNTT scaled by n^-1);
    tables from this library (natural order).  events: optional list that
    receives (start, end, columns) CUDA events around each launch group."""
    n = 1 << tables.log_n
    step = min(ncols, NTT_CHUNK)
    tmp = torch.empty((step * n, 4), dtype=torch.int64, device="cuda") if tmp is None else tmp
    o = out.reshape(-1, 4)
    sr = src.reshape(-1, 4)
    for c0 in range(0, ncols, step):
        cnt = min(step, ncols - c0)
        if events is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), cnt)
            ev[0].record(stream)
        abi.check(lib().zkp_ntt_batch_twisted(o[c0 * n:].data_ptr(), sr[c0 * n:].data_ptr(), tmp.data_ptr(),
                                              (tables.tw_inv if inverse else tables.tw).data_ptr(), _p(in_mul),
                                              tables.n_inv.data_ptr() if inverse else 0, tables.log_n, cnt, n, n,
                                              0, _st(stream)), "zkp_ntt_batch_twisted")
        if events is not None:
            ev[1].record(stream)
            events.append(ev)


def _ntt_into_pairs(out, src, tw_pairs, in_mul_pairs, ncols: int, log_n: int, tmp, events=None, stream=None):
    """ntt_into's forward transform over (w, w') pair tables."""
    n = 1 << log_n
    step = min(ncols, NTT_CHUNK)
    o = out.reshape(-1, 4)
    sr = src.reshape(-1, 4)
    for c0 in range(0, ncols, step):
        cnt = min(step, ncols - c0)
        if events is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), cnt)
            ev[0].record(stream)
        abi.check(lib().zkp_ntt_batch_twisted(o[c0 * n:].data_ptr(), sr[c0 * n:].data_ptr(), tmp.data_ptr(),
                                              tw_pairs.data_ptr(), in_mul_pairs.data_ptr(), 0, log_n, cnt, n, n,
                                              1, _st(stream)), "zkp_ntt_batch_twisted")
        if events is not None:
            ev[1].record(stream)
            events.append(ev)


def powers(base: int, w: int, n: int, out=None) -> torch.Tensor:
    """out[i] = base * w^i."""
    out = torch.empty((n, 4), dtype=torch.int64, device="cuda") if out is None else out
    b, ww = fr_tensor([base]), fr_tensor([w])
    abi.check(lib().zkp_powers(out.data_ptr(), b.data_ptr(), ww.data_ptr(), n, _st()), "zkp_powers")
    return out


# ---------------------------------------------------------------- the circuit


class Circuit:
    """Proving key and witness of the synthetic circuit, generated on the GPU
    from one seed.  Column roles (advice): lookup inputs, shuffle pairs
    (input, shuffled copy), then five columns (a, b, c, d, e) per gate and any
    remainder; (fixed): the range table, one selector per gate, then constants;
    the permutation columns are the instance column, the fixed constants and
    the gates' a, b, c, d columns (then the remainder) up to `perm`.  The
    witness satisfies every constraint on the usable rows; blinding rows are
    random."""

    def __init__(self, shape: Shape, seed: int = 1, device="cuda"):
        s = self.shape = shape
        n, u, k = s.n, s.usable, s.k
        self.n, self.u, self.k = n, u, k
        G = s.gates
        if G < 1 or 1 + G > s.fixed:
            raise ValueError("shape leaves no room for the gates and their selectors")
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
        self.gen = gen
        L = lib()
        # roles
        self.lookup_cols = list(range(s.lookups))
        self.shuffle_pairs = [(s.lookups + 2 * i, s.lookups + 2 * i + 1) for i in range(s.shuffles)]
        g0 = s.lookups + 2 * s.shuffles
        self.gate_cols = [tuple(g0 + 5 * g + j for j in range(5)) for g in range(G)]
        rest = list(range(g0 + 5 * G, s.advice))
        self.table_col = 0
        self.selector_cols = [1 + g for g in range(G)]
        const_cols = list(range(1 + G, s.fixed))
        perm = [("instance", 0)] + [("fixed", c) for c in const_cols]
        perm += [("advice", c) for g in self.gate_cols for c in g[:4]] + [("advice", c) for c in rest]
        if len(perm) < s.perm:
            raise ValueError("not enough columns for the permutation")
        self.perm_cols = perm[:s.perm]
        # values
        self.advice = torch.empty((s.advice, n, 4), dtype=torch.int64, device=device)
        for c in range(s.advice):
            self.advice[c] = rand_fr(n, gen)
        self.fixed = torch.empty((s.fixed, n, 4), dtype=torch.int64, device=device)
        self.instance = torch.zeros((1, n, 4), dtype=torch.int64, device=device)
        self.instance[0, :s.instance_rows] = rand_fr(s.instance_rows, gen)
        lim = min(1 << 16, 1 << (k - 1))
        self.table_values = lim
        ar = torch.arange(n, device=device, dtype=torch.int64)
        self.fixed[self.table_col] = small_fr(ar % lim)
        for c in self.lookup_cols:
            self.advice[c, :u] = small_fr(torch.randint(0, lim, (u,), device=device, generator=gen))
        for a, b in self.shuffle_pairs:
            self.advice[b, :u] = self.advice[a, torch.randperm(u, device=device, generator=gen)]
        for c in self.selector_cols:
            bits = torch.randint(0, 2, (n,), device=device, generator=gen)
            bits[u:] = 0
            self.fixed[c] = small_fr(bits)
        for c in const_cols:
            self.fixed[c] = rand_fr(n, gen)
        self._permutation(gen)
        # gates: e = a b c + d where q = 1
        t = torch.empty((n, 4), dtype=torch.int64, device=device)
        for g, (ca, cb, cc, cd, ce) in enumerate(self.gate_cols):
            field_op(t, self.advice[ca], self.advice[cb], 1, n)
            field_op(t, t, self.advice[cc], 1, n)
            field_op(t, t, self.advice[cd], 0, n)
            q = self.fixed[self.selector_cols[g], :, 0] != 0
            self.advice[ce] = torch.where(q[:, None], t, self.advice[ce])
        # Lagrange basis vectors l_0, l_last (row u) and l_active (rows < u)
        one = fr_tensor([1])[0]
        self.l0 = torch.zeros((n, 4), dtype=torch.int64, device=device)
        self.l0[0] = one
        self.l_last = torch.zeros((n, 4), dtype=torch.int64, device=device)
        self.l_last[u] = one
        self.l_active = torch.zeros((n, 4), dtype=torch.int64, device=device)
        self.l_active[:u] = one
        # seeded blinding tails of the grand products and the random polynomial
        self.z_tails = rand_fr(n - u - 1, gen)
        self.random_poly = rand_fr(n, gen)
        torch.cuda.synchronize()
        del L

    def column(self, kind, idx):
        return {"advice": self.advice, "fixed": self.fixed, "instance": self.instance}[kind][idx]

    def _permutation(self, gen):
        """Copy-constraint cycles of three cells over the usable rows of the
        permutation columns (half the cells), equal values along each cycle,
        and the sigma columns delta^c' w^r' of the cell each cell maps to."""
        s, n, u = self.shape, self.n, self.u
        P = s.perm
        dev = self.advice.device
        # identity: delta^c w^r
        wt = powers(1, omega(self.k), n)
        ident = torch.empty((P, n, 4), dtype=torch.int64, device=dev)
        for c in range(P):
            field_op(ident[c], wt, None, 2, n, l_c=fr_tensor([pow(DELTA, c, R_MOD)]))
        m = (P * u // 2) // 3 * 3
        sel = torch.randperm(P * u, device=dev, generator=gen)[:m]
        cells = (sel // u) * n + (sel % u)
        a, b, c = cells[0::3], cells[1::3], cells[2::3]
        mapping = torch.arange(P * n, device=dev, dtype=torch.int64)
        mapping[a], mapping[b], mapping[c] = b, c, a
        self.sigma = ident.view(P * n, 4)[mapping].view(P, n, 4)
        vals = torch.stack([self.column(kd, i) for kd, i in self.perm_cols]).view(P * n, 4)
        gv = rand_fr(a.shape[0], gen)
        vals[a], vals[b], vals[c] = gv, gv, gv
        vals = vals.view(P, n, 4)
        for j, (kd, i) in enumerate(self.perm_cols):
            self.column(kd, i).copy_(vals[j])
        del ident, mapping, vals


# ---------------------------------------------------------------- witness from host memory


class HostStage:
    """Copies the advice columns from pinned host memory into the circuit's
    device columns in groups of `group` columns on a copy stream, one event
    per group; the prover waits on a group's event before its first use."""

    def __init__(self, host_advice: torch.Tensor, dev_advice: torch.Tensor, group: int = MSM_BATCH):
        self.host, self.dev, self.group = host_advice, dev_advice, group
        self.stream = torch.cuda.Stream()
        self.events = []
        ngroups = -(-host_advice.shape[0] // group)
        self.h_dev = torch.zeros((ngroups, 8), dtype=torch.int32, device="cuda")
        self.h_host = torch.zeros((ngroups, 8), dtype=torch.int32, pin_memory=True)

    def start(self, histograms: bool = False):
        """Queues every group's copy; with histograms, also the scalar
        histogram of each group's first column right behind its copy (the
        learned MSM choice reads it without waiting for the compute stream)."""
        # the copies overwrite the columns: order them after the work already queued
        self.stream.wait_stream(torch.cuda.current_stream())
        self.events = []
        with torch.cuda.stream(self.stream):
            for gi, g0 in enumerate(range(0, self.host.shape[0], self.group)):
                g1 = min(self.host.shape[0], g0 + self.group)
                self.dev[g0:g1].copy_(self.host[g0:g1], non_blocking=True)
                if histograms:
                    self.h_dev[gi].zero_()
                    abi.check(lib().zkp_scalar_histogram(self.dev[g0].data_ptr(), self.dev.shape[1],
                                                         self.h_dev[gi].data_ptr(), _st(self.stream)),
                              "zkp_scalar_histogram")
                    self.h_host[gi].copy_(self.h_dev[gi], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.stream)
                self.events.append((g0, g1, ev))

    def wait(self, lo: int, hi: int):
        for g0, g1, ev in self.events:
            if g0 < hi and g1 > lo:
                torch.cuda.current_stream().wait_event(ev)

    def histogram(self, gi: int) -> list:
        """The histogram features of group gi's first column: waits for that
        group's copy only."""
        self.events[gi][2].synchronize()
        v = self.h_host[gi].numpy()[:7].astype(np.float64)
        return list(v / max(1.0, v.sum()))


# ---------------------------------------------------------------- host-side steps


class DeviceHostWork:
    """The steps the reference runs on the CPU (src/permutation.rs,
    src/shuffle.rs, the divisions of src/multiopen.rs) through this library's
    device entry points."""

    def permutation_products(self, ctx, cols, sigmas, beta, gamma):
        s, n, u = ctx.shape, ctx.n, ctx.u
        L = lib()
        scratch = H.empty_fr(n + L.zkp_scan_scratch_elems(n))
        zall = ctx._ws("perm_z", (s.perm_chunks, n, 4))
        zs = []
        bt, gt = fr_tensor([beta]), fr_tensor([gamma])
        for j in range(s.perm_chunks):
            c0, c1 = j * s.chunk_len, min(s.perm, (j + 1) * s.chunk_len)
            pc = ptr_array([c.data_ptr() for c in cols[c0:c1]])
            ps = ptr_array([c.data_ptr() for c in sigmas[c0:c1]])
            db = fr_tensor([beta * pow(DELTA, c, R_MOD) for c in range(c0, c1)])
            z = zall[j]
            init = zs[-1][u:u + 1] if zs else fr_tensor([1])
            abi.check(L.zkp_permutation_z(z.data_ptr(), pc.data_ptr(), ps.data_ptr(), c1 - c0, bt.data_ptr(),
                                          gt.data_ptr(), db.data_ptr(), ctx.own_n.natural.data_ptr(), init.data_ptr(), n,
                                          scratch.data_ptr(), _st()), "zkp_permutation_z")
            zs.append(z)
        return zs

    def shuffle_products(self, ctx, pairs, beta):
        n = ctx.n
        L = lib()
        scratch = H.empty_fr(n + L.zkp_scan_scratch_elems(n))
        zs = []
        betas = fr_tensor([beta])
        zall = ctx._ws("shuffle_z", (len(pairs), n, 4))
        for j, (inp, tab) in enumerate(pairs):
            z = zall[j]
            # the pointer arrays stay referenced until the call returns: a
            # temporary freed inside the argument list can be handed out again
            # to the next one before the kernel reads it
            pi, pt = ptr_array([inp.data_ptr()]), ptr_array([tab.data_ptr()])
            abi.check(L.zkp_shuffle_z(z.data_ptr(), pi.data_ptr(), pt.data_ptr(), betas.data_ptr(), 1, n,
                                      scratch.data_ptr(), _st()), "zkp_shuffle_z")
            zs.append(z)
        return zs

    def divide_linear(self, ctx, a, z: int):
        """(a(X) - a(z)) / (X - z) with the reference's layout (q[n-1] = 0)."""
        n = a.shape[0]
        L = lib()
        q = torch.empty_like(a)
        scratch = H.empty_fr(L.zkp_poly_divide_scratch_elems(n))
        zh = np.array(limbs(z), dtype=np.uint64)
        abi.check(L.zkp_poly_divide_linear(q.data_ptr(), a.data_ptr(), zh.ctypes.data, n, scratch.data_ptr(), _st()),
                  "zkp_poly_divide_linear")
        return q


# ---------------------------------------------------------------- the prover


class HotPath:
    """One proof's hot path over a Circuit.  ``schedule``: "plain" or
    "batched"; ``symbols``: the library whose reference-compatible symbols the
    plain schedule calls (default: this one); ``host_work``: the CPU-side steps
    (default: DeviceHostWork)."""

    def __init__(self, circuit: Circuit, schedule="batched", symbols=None, host_work=None, seed=7, srs_seed=11,
                 pair_tables=False, pk_cache_gib=None, group=None, learned=True):
        if schedule not in ("plain", "batched"):
            raise ValueError(schedule)
        self.c = circuit
        self.shape = circuit.shape
        self.n, self.u, self.k = circuit.n, circuit.u, circuit.k
        self.schedule = schedule
        self.sym = symbols or lib()
        self.hw = host_work or DeviceHostWork()
        self.seed = seed
        # when set to a list, the batched quotient's coset transforms append
        # (start, end, columns) CUDA events to it (benchmark instrumentation)
        self.ntt_events = None
        # batched schedule: coset transforms over Montgomery tables, or over
        # (w, w') known-factor tables (pair_tables; at 2^22 the radix-2^11
        # passes run no faster with them: 1.028 against 0.994 ms a column);
        # proving-key coset values cached up to pk_cache_gib (None: as much as
        # the proof's memory leaves, 0: none)
        self.pair_tables = pair_tables
        self.pk_cache_gib = pk_cache_gib
        self.pk_cos = {}
        self._wsd = {}
        # batched schedule: MSM pipelines over the table or the plain bases as
        # the learned table-or-plain model picks (with learned windows for the
        # plain ones); learned=False keeps every pipeline on the table
        self.learned = learned and schedule == "batched"
        self.learned_picks = {}
        if self.learned:
            from . import choices, schedule as S

            self._choice_msm = choices.ChoiceModel.load("msm_table")
            self._window_model = S.Model.load()
        # batched schedule on several GPUs: a torch.distributed process group
        # whose ranks (one per GPU, each with the same circuit) share the
        # proof: commitments by column ranges, the quotient by cosets (shard.py)
        self.group = group
        if group is not None:
            from . import shard

            self.rank, self.world = shard.rank_world(group)
            if schedule != "batched":
                raise ValueError("sharding needs the batched schedule")
        else:
            self.rank, self.world = 0, 1
        s = self.shape
        self.E = 1 << s.ext_bits
        self.ek = self.k + s.ext_bits
        # tables of this library (batched entry points, proving-key setup) and,
        # for the plain schedule, of the symbol library
        self.own_n = Tables(self.k)
        self.tab_n = Tables(self.k, self.sym) if schedule == "plain" else self.own_n
        self.tab_N = Tables(self.ek, self.sym) if schedule == "plain" else None
        # SRS: seeded 62-bit multiples of G for the coefficient and the Lagrange
        # bases (same MSM work as [tau^i] G; known discrete logs)
        g = torch.Generator(device="cuda")
        g.manual_seed(srs_seed)
        self.srs_k = torch.randint(0, 2 ** 62, (2, self.n), dtype=torch.int64, device="cuda", generator=g)
        self.g = torch.empty((self.n, 8), dtype=torch.int64, device="cuda")
        self.g_lagrange = torch.empty((self.n, 8), dtype=torch.int64, device="cuda")
        for t, kk in ((self.g, self.srs_k[0]), (self.g_lagrange, self.srs_k[1])):
            abi.check(lib().zkp_g1_multiples(t.data_ptr(), kk.data_ptr(), self.n, _st()), "zkp_g1_multiples")
        self._pk()
        if schedule == "batched":
            self._batched_setup()
        torch.cuda.synchronize()

    # ------------------------------------------------------------ setup

    def _pk(self):
        """Coefficient forms of the proving key's columns (fixed, sigma, l_0,
        l_last, l_active), as the reference's pk holds them."""
        c, s, n = self.c, self.shape, self.n
        self.fixed_coeff = c.fixed.clone()
        ntt_cols(self.fixed_coeff, self.own_n, s.fixed, True)
        self.sigma_coeff = c.sigma.clone()
        ntt_cols(self.sigma_coeff, self.own_n, s.perm, True)
        self.l_coeff = torch.stack([c.l0, c.l_last, c.l_active])
        ntt_cols(self.l_coeff, self.own_n, 3, True)

    def _batched_setup(self):
        n, E = self.n, self.E
        L = lib()
        # MSM tables of both SRS bases at the batch-table width
        na = (ctypes.c_uint32 * 1)(n)
        self.tc = L.zkp_msm_batch_table_default_window(ctypes.addressof(na), 1)
        self.table_g, _ = H.msm_table_build(self.g, n, self.tc)
        self.table_gl, _ = H.msm_table_build(self.g_lagrange, n, self.tc)
        # per-coset twists (zeta w_N^j)^i, the rows' X and the combine tables
        wN = omega(self.ek)
        self.coset_twist = torch.empty((E, n, 4), dtype=torch.int64, device="cuda")
        self.coset_x = torch.empty((E, n, 4), dtype=torch.int64, device="cuda")
        for j in range(E):
            sj = ZETA * pow(wN, j, R_MOD) % R_MOD
            powers(1, sj, n, self.coset_twist[j])
            powers(sj, self.tab_n.w, n, self.coset_x[j])
        self.winv_N = powers(1, pow(wN, -1, R_MOD), n)
        zn = [(pow(ZETA * pow(wN, j, R_MOD), n, R_MOD) - 1) % R_MOD for j in range(E)]
        self.t_inv = [pow(z, -1, R_MOD) for z in zn]
        wE_inv = pow(pow(wN, n, R_MOD), -1, R_MOD)
        einv = pow(E, -1, R_MOD)
        zinv = pow(ZETA, -1, R_MOD)
        # the fused pass already divides each coset's values by Z_H (its
        # `scale`), so the combine's per-coset factors are 1
        self.combine_consts = fr_tensor([1] * E + [pow(wE_inv, kk, R_MOD) for kk in range(E)] +
                                        [pow(zinv, kk, R_MOD) * einv % R_MOD for kk in range(3)])
        self.t_inv_dev = fr_tensor(self.t_inv)
        # known-factor (w, w') forms of the forward twiddles and the coset twists
        if self.pair_tables:
            self.tab_pairs = torch.empty((2 * n, 4), dtype=torch.int64, device="cuda")
            abi.check(L.zkp_shoup_pairs(self.tab_pairs.data_ptr(), self.tab_n.tw.data_ptr(), n, _st()),
                      "zkp_shoup_pairs")
            self.coset_twist_pairs = torch.empty((E, 2 * n, 4), dtype=torch.int64, device="cuda")
            for j in range(E):
                abi.check(L.zkp_shoup_pairs(self.coset_twist_pairs[j].data_ptr(), self.coset_twist[j].data_ptr(), n,
                                            _st()), "zkp_shoup_pairs")
        self._workspaces()
        self._cache_pk_cosets()
        self._alloc_quotient_workspace()

    def _ws(self, name, shape, dtype=torch.int64):
        """A per-proof buffer: allocated once for the batched schedule (a
        prover runs proof after proof, and at k = 22 the proof's buffers take
        most of the 180 GB; allocating them per proof fragments HBM), fresh
        for the plain schedule (the reference host's per-call allocations)."""
        if self.schedule != "batched":
            return torch.empty(shape, dtype=dtype, device="cuda")
        t = self._wsd.get(name)
        if t is None or tuple(t.shape) != tuple(shape):
            t = torch.empty(shape, dtype=dtype, device="cuda")
            self._wsd[name] = t
        return t

    def _workspaces(self):
        """The batched schedule's per-proof buffers, allocated at setup."""
        s, n, E = self.shape, self.n, self.E
        A, L_ = s.advice, s.lookups
        for name, shape in (("adv_coeff", (A, n, 4)), ("inst_coeff", (1, n, 4)), ("m", (L_, n, 4)),
                            ("m_coeff", (L_, n, 4)), ("lookup_z", (L_, n, 4)),
                            ("perm_z", (s.perm_chunks, n, 4)), ("shuffle_z", (s.shuffles, n, 4)),
                            ("ntt_tmp", (NTT_CHUNK * n, 4)), ("hc", (E, n, 4)), ("hg", (E, n, 4)),
                            ("h_coeff", (E * n, 4))):
            self._ws(name, shape)
        # the pipeline's scratch is not monotonic in the MSM count (the
        # reduction's threads are shared out over the batch): the largest over
        # every count a pipeline of the proof can have
        nbytes = 0
        for cnt in range(1, MSM_BATCH + 2):
            na = (ctypes.c_uint32 * cnt)(*([n] * cnt))
            nbytes = max(nbytes, lib().zkp_msm_batch_table_scratch_bytes(ctypes.addressof(na), cnt, n, self.tc))
        self._ws("msm_scratch", (max(1, nbytes),), torch.uint8)

    def _quotient_rows(self):
        """(name, source, columns) of every column group the quotient reads,
        the witness's first."""
        s = self.shape
        dyn = [("adv", "adv_coeff", s.advice), ("inst", "inst_coeff", 1), ("pz", "perm_z", s.perm_chunks),
               ("m", "m_coeff", s.lookups), ("lz", "lookup_z", s.lookups), ("sz", "shuffle_z", s.shuffles)]
        pk = [("fixed", "fixed_coeff", s.fixed), ("sigma", "sigma_coeff", s.perm), ("l", "l_coeff", 3)]
        return [g for g in dyn if g[2] > 0], [g for g in pk if g[2] > 0]

    def _alloc_quotient_workspace(self):
        """One coset of every column the quotient transforms per proof: the
        witness's and the proving key's not cached for every coset."""
        dyn, pk = self._quotient_rows()
        work = dyn + [g for g in pk if not all((g[0], j) in self.pk_cos for j in range(self.E))]
        rows = sum(g[2] for g in work)
        self._ws("ev", (max(1, rows), self.n, 4))

    def _cache_pk_cosets(self):
        """Coset values of the proving key's columns (fixed, then l_0 / l_last /
        l_active, then sigma, one coset at a time), computed once and kept in
        HBM as far as the memory a proof needs leaves room, as halo2's pk keeps
        its fixed and permutation cosets; the quotient then transforms only the
        witness's columns."""
        s, n, E = self.shape, self.n, self.E
        self.pk_cos = {}
        if self.pk_cache_gib is not None:
            budget = self.pk_cache_gib * (1 << 30)
        else:
            # what is left once the per-proof buffers (allocated already) and
            # the quotient's workspace for the witness's columns are set aside,
            # less a margin for the proof's small buffers
            torch.cuda.empty_cache()
            free, _ = torch.cuda.mem_get_info()
            dyn, _ = self._quotient_rows()
            budget = free - sum(g[2] for g in dyn) * n * 32 - (14 << 30)
        tmp = self._ws("ntt_tmp", (NTT_CHUNK * n, 4))
        order = [("fixed", self.fixed_coeff, s.fixed), ("l", self.l_coeff, 3), ("sigma", self.sigma_coeff, s.perm)]
        used = 0
        if self.world > 1:
            from . import shard

            mine = shard.coset_ranks(E, self.world)[self.rank]
        else:
            mine = list(range(E))
        for name, src, cnt in order:
            for j in mine:
                size = cnt * n * 32
                if used + size > budget:
                    break
                t = torch.empty((cnt, n, 4), dtype=torch.int64, device="cuda")
                self._coset_ntt(t, src, cnt, j, tmp)
                self.pk_cos[(name, j)] = t
                used += size
        self.pk_cache_bytes = used
        torch.cuda.synchronize()

    # ------------------------------------------------------------ MSM helpers

    def _msm_plain(self, bases, cols):
        """src/cuda/msm.rs:239-455: one msm() per column with the reference
        host's sizing, then batch_msm_collect; affine results."""
        if not cols:
            return []
        b = _RefMsm(self.sym, bases, cols, self.n)
        b.enqueue()
        return jac_to_affine(b.results())

    def _msm_batched(self, lagrange: bool, cols):
        if not cols:
            return []
        table = self.table_gl if lagrange else self.table_g
        bases = self.g_lagrange if lagrange else self.g
        # pipelines of MSM_BATCH MSMs: at 2^22 over the c = 19 table, 8 a
        # pipeline run at 13.05 ms an MSM against 13.64 for 16 and 14.21 for 32
        parts = [cols[i:i + MSM_BATCH] for i in range(0, len(cols), MSM_BATCH)]
        # every pipeline's schedule choice before the first launch: the
        # histograms and the model run once for the whole call, so the
        # pipelines queue back to back with no host round trip between them
        picks = self._msm_picks(parts)
        outs = [self._msm_part(table, bases, part, pick) for part, pick in zip(parts, picks)]
        torch.cuda.synchronize()
        return jac_to_affine(torch.cat(outs).cpu().numpy().view(np.uint64))

    def _msm_picks(self, parts, hists=None):
        """For each pipeline: None (over the SRS table) or the scalar
        histogram features (over the plain bases, with a learned window), as
        the learned table-or-plain choice predicts faster for the pipeline's
        size, count and scalar distribution.  hists: the features when the
        caller has them (then the model runs on a side stream, so reading its
        answer does not wait for the work queued on the compute stream)."""
        if not self.learned:
            return [None] * len(parts)
        from . import schedule as S

        recs = lambda hs: [{"n": self.n, "batch": len(p), "hist": h} for p, h in zip(parts, hs)]
        if hists is None:
            hists = S.histograms([p[0] for p in parts])
            table = self._choice_msm.pick_many(recs(hists), [0, 1])
        else:
            if getattr(self, "_pick_stream", None) is None:
                self._pick_stream = torch.cuda.Stream()
            with torch.cuda.stream(self._pick_stream):
                table = self._choice_msm.pick_many(recs(hists), [0, 1])
        return [None if t == 1 else h for t, h in zip(table, hists)]

    def _msm_part(self, table, bases, part, pick=None):
        """One MSM pipeline: over the SRS table (pick None), or over the plain
        bases with the learned window for the histogram features `pick`."""
        n = self.n
        ns = [n] * len(part)
        if self.learned:
            from . import schedule as S

            if pick is not None:
                feats = S.shape_features(n, len(part), pick)
                c = self._window_model.pick(feats)
                ws = [c] * len(part)
                na = (ctypes.c_uint32 * len(part))(*ns)
                ca = (ctypes.c_int * len(part))(*ws)
                nbytes = lib().zkp_msm_batch_scratch_bytes(ctypes.addressof(na), ctypes.addressof(ca), len(part))
                scratch = self._wsd.get("msm_plain_scratch")
                if scratch is None or scratch.numel() < nbytes:
                    scratch = torch.empty(max(1, nbytes), dtype=torch.uint8, device="cuda")
                    self._wsd["msm_plain_scratch"] = scratch
                self.learned_picks["plain"] = self.learned_picks.get("plain", 0) + 1
                return H.msm_batch(bases, part, ns, ws, scratch=scratch)
            self.learned_picks["table"] = self.learned_picks.get("table", 0) + 1
        return H.msm_batch_table(table, n, self.tc, part, ns, scratch=self._wsd.get("msm_scratch"))

    def commit(self, lagrange: bool, cols):
        if self.schedule == "plain":
            return self._msm_plain(self.g_lagrange if lagrange else self.g, cols)
        if self.world > 1:
            from . import shard

            a, b = shard.column_ranges(len(cols), self.world)[self.rank]
            return shard.gather_points(self._msm_batched(lagrange, cols[a:b]), self.group)
        return self._msm_batched(lagrange, cols)

    def intt_many(self, cols):
        """In-place iNTT of each column (list of (n, 4) tensors)."""
        if self.schedule == "plain":
            tmp = H.empty_fr(self.n)
            for c in cols:
                ntt_raw(self.sym, c, tmp, self.tab_n, True, self.tab_n.n_inv)
        elif cols:
            st = _stacked(cols)
            if st.data_ptr() == cols[0].data_ptr() and len(cols) <= NTT_CHUNK and "ntt_tmp" in self._wsd:
                # consecutive rows of one workspace: one batched launch group
                tmp = self._wsd["ntt_tmp"][:len(cols) * self.n].view(st.shape)
                ntt_cols(st, self.tab_n, len(cols), True, tmp=tmp)
            else:
                for c in cols:
                    ntt_cols(c, self.tab_n, 1, True)

    def counts(self):
        """Work units of one proof in this schedule: MSMs of n points, NTTs of
        n points (batched) or of n and 2^(k+e) points (plain), and the
        polynomials whose coset values the quotient needs."""
        s = self.shape
        msm = (s.advice + 1) + s.lookups + (s.perm_chunks + s.shuffles) + (s.lookups + 1) + (s.degree - 1)
        msm += 2 if s.multiopen == "shplonk" else 3
        cols = s.advice + 1 + s.perm_chunks + 2 * s.lookups + s.shuffles + s.fixed + s.perm + 3
        return {"msm": msm, "quotient_columns": cols, "cosets": self.E,
                "ntt_n": (s.advice + 1) + 2 * s.lookups + s.perm_chunks + s.shuffles + cols * self.E + self.E + 2}

    # ------------------------------------------------------------ the proof

    def prove(self, stage=None):
        """Runs phases 1-6; returns the proof stand-in: every commitment
        (affine ints) and evaluation, in transcript order.  stage: a
        HostStage bringing the advice columns in from host memory during
        phase 1 (batched schedule).

        Python's automatic garbage collection is paused while the proof runs
        (reference counting still frees its objects; any left in cycles wait
        for the first collection after it): a full collection, tens of ms
        with the proving key's objects alive, landing at a phase boundary,
        where the device waits for the host, stalled the device."""
        import gc

        enabled = gc.isenabled()
        gc.disable()
        try:
            return self._prove(stage)
        finally:
            if enabled:
                gc.enable()

    def _prove(self, stage):
        s, c, n, u = self.shape, self.c, self.n, self.u
        tr = Transcript(self.seed)
        proof = {"commitments": [], "evals": []}
        self.phase_s = {}
        self.learned_picks = {}
        t0 = [time.perf_counter()]

        def absorb(name, pts):
            tr.points(pts)
            proof["commitments"].append((name, pts))

        def mark(phase):
            # wall time of each phase (the transcript synchronises at every challenge)
            torch.cuda.synchronize()
            t = time.perf_counter()
            self.phase_s[phase] = t - t0[0]
            t0[0] = t

        # 1. advice and instance
        adv = [c.advice[i] for i in range(s.advice)]
        inst = [c.instance[0]]
        if self.schedule == "plain":
            com = self.commit(True, adv + inst)
            self.adv_coeff = c.advice.clone()
            self.inst_coeff = c.instance.clone()
            self.intt_many([self.adv_coeff[i] for i in range(s.advice)] + [self.inst_coeff[0]])
        elif stage is not None and self.world == 1:
            # the witness arrives from host memory: commit and transform each
            # group of columns as soon as its copy has landed, while later
            # groups are still crossing PCIe (src/lib.rs overlaps the copies
            # of its columns with the MSMs of earlier ones the same way)
            self.adv_coeff = self._ws("adv_coeff", tuple(c.advice.shape))
            self.inst_coeff = self._ws("inst_coeff", tuple(c.instance.shape))
            stage.start(histograms=self.learned)
            outs = []
            for gi, a0 in enumerate(range(0, s.advice, MSM_BATCH)):
                a1 = min(s.advice, a0 + MSM_BATCH)
                stage.wait(a0, a1)
                part = adv[a0:a1] + (inst if a1 == s.advice else [])
                pick = self._msm_picks([part], [stage.histogram(gi)])[0] if self.learned else None
                outs.append(self._msm_part(self.table_gl, self.g_lagrange, part, pick))
                ntt_into(self.adv_coeff[a0:a1], c.advice[a0:a1], self.tab_n, a1 - a0, True,
                         tmp=self._wsd["ntt_tmp"])
            ntt_into(self.inst_coeff, c.instance, self.tab_n, 1, True)
            torch.cuda.synchronize()
            com = jac_to_affine(torch.cat(outs).cpu().numpy().view(np.uint64))
        else:
            com = self.commit(True, adv + inst)
            self.adv_coeff = self._ws("adv_coeff", tuple(c.advice.shape))
            ntt_into(self.adv_coeff, c.advice, self.tab_n, s.advice, True, tmp=self._wsd.get("ntt_tmp"))
            self.inst_coeff = self._ws("inst_coeff", tuple(c.instance.shape))
            ntt_into(self.inst_coeff, c.instance, self.tab_n, 1, True, tmp=self._wsd.get("ntt_tmp"))
        absorb("instance", com[s.advice:])
        absorb("advice", com[:s.advice])
        theta = tr.challenge()
        mark("1 advice commit + iNTT")

        # 2. lookup multiplicities
        self.m = self._ws("m", (s.lookups, n, 4))
        self.m.zero_()
        self._lookup_m()
        absorb("lookup_m", self.commit(True, [self.m[i] for i in range(s.lookups)]))
        beta, gamma = tr.challenge(), tr.challenge()
        self.beta, self.gamma, self.theta = beta, gamma, theta
        mark("2 lookup m")

        # 3. logup z, permutation and shuffle products
        self._logup_z(beta)
        perm_vals = [c.column(kd, i) for kd, i in c.perm_cols]
        self.perm_z = self.hw.permutation_products(self, perm_vals, [c.sigma[j] for j in range(s.perm)], beta, gamma)
        self.shuffle_z = self.hw.shuffle_products(self, [(c.advice[a], c.advice[b]) for a, b in c.shuffle_pairs], beta)
        for z in self.perm_z + self.shuffle_z:
            z[u + 1:] = c.z_tails
        perm_com = self.commit(True, self.perm_z)
        self.intt_many(self.perm_z)
        shuffle_com = self.commit(True, self.shuffle_z)
        self.intt_many(self.shuffle_z)
        lz_com = self.commit(False, [self.lookup_z[i] for i in range(s.lookups)] + [c.random_poly])
        absorb("permutation_z", perm_com)
        absorb("lookup_z", lz_com[:-1])
        absorb("shuffle_z", shuffle_com)
        absorb("random", lz_com[-1:])
        y = tr.challenge()
        self.y = y
        mark("3 grand products + commits")

        # 4. quotient
        if self.schedule == "plain":
            h_coeff = self._quotient_plain(y, beta, gamma)
        else:
            h_coeff = self._quotient_batched(y, beta, gamma)
        self.h_coeff = h_coeff
        # quotient_poly_degree pieces (src/eval_h.rs:512-545); with a valid
        # witness h has degree below degree (n - 1) - n, so the coefficients
        # past the pieces are zero
        pieces = [h_coeff[i * n:(i + 1) * n] for i in range(s.degree - 1)]
        mark("4a quotient h")
        absorb("h_pieces", self.commit(False, pieces))
        x = tr.challenge()
        self.x = x
        mark("4b h commits")

        # 5. evaluations
        xn = pow(x, n, R_MOD)
        h_fold = pieces[-1].clone()
        xn_t = fr_tensor([xn])
        for i in range(len(pieces) - 2, -1, -1):
            field_op(h_fold, h_fold, pieces[i], 0, n, l_c=xn_t, sym=self.sym if self.schedule == "plain" else None)
        self.h_fold = h_fold
        queries = self._queries(x)
        evals = self._evaluate(queries)
        tr.scalars(evals)
        proof["evals"] = evals
        mark("5 evaluations")

        # 6. multi-open
        if s.multiopen == "shplonk":
            absorb("multiopen", self._shplonk(tr, queries, evals))
        else:
            absorb("multiopen", self._gwc(tr, queries, evals))
        mark("6 multiopen")
        proof["challenges"] = {"theta": theta, "beta": beta, "gamma": gamma, "y": y, "x": x}
        return proof

    # ------------------------------------------------------------ phase 2, 3 details

    def _lookup_m(self):
        s, n, u, k = self.shape, self.n, self.u, self.k
        c = self.c
        words = [torch.empty(n * 8, dtype=torch.int32, device="cuda") for _ in range(6)]
        table = c.fixed[c.table_col]
        for i, col in enumerate(c.lookup_cols):
            if self.schedule == "plain" or i == 0:
                # the reference prepares the table of every lookup (src/lib.rs:425-445);
                # the batched schedule prepares the shared range table once
                abi.check(self.sym.prepare_table_lookup(table.data_ptr(), words[0].data_ptr(), words[1].data_ptr(),
                                                        words[2].data_ptr(), words[3].data_ptr(), words[4].data_ptr(),
                                                        words[5].data_ptr(), n * 32, k, u, _st()),
                          "prepare_table_lookup")
            abi.check(self.sym.calc_m(self.m[i].data_ptr(), table.data_ptr(), c.advice[col].data_ptr(),
                                      words[3].data_ptr(), words[4].data_ptr(), words[0].data_ptr(),
                                      words[1].data_ptr(), words[5].data_ptr(), n * 32, k, u, _st()), "calc_m")

    def _logup_z(self, beta):
        """src/lib.rs:586-720: sum of 1/(input + beta), z by
        eval_logup_z_compose (table used as scratch), then m and z to
        coefficients."""
        s, n, u = self.shape, self.n, self.u
        c = self.c
        bt = fr_tensor([beta])
        self.lookup_z = self._ws("lookup_z", (s.lookups, n, 4))
        last = torch.zeros((max(1, s.lookups), 4), dtype=torch.int64, device="cuda")
        ssum = H.empty_fr(n)
        tmp = H.empty_fr(n)
        tcopy = H.empty_fr(n)
        for i, col in enumerate(c.lookup_cols):
            abi.check(self.sym.logup_sum_input_inv(ssum.data_ptr(), c.advice[col].data_ptr(), tmp.data_ptr(),
                                                   bt.data_ptr(), 0, n, _st()), "logup_sum_input_inv")
            tcopy.copy_(c.fixed[c.table_col])
            abi.check(self.sym.eval_logup_z_compose(self.lookup_z[i].data_ptr(), ssum.data_ptr(), tcopy.data_ptr(),
                                                    self.m[i].data_ptr(), bt.data_ptr(), last[i].data_ptr(), u, n,
                                                    _st()), "eval_logup_z_compose")
        # m (committed in Lagrange form above) and z to coefficients
        self.m_coeff = self._ws("m_coeff", (s.lookups, n, 4))
        self.m_coeff.copy_(self.m)
        if self.schedule == "plain":
            self.intt_many([self.m_coeff[i] for i in range(s.lookups)] + [self.lookup_z[i] for i in range(s.lookups)])
        else:
            ntt_cols(self.m_coeff, self.tab_n, s.lookups, True)
            ntt_cols(self.lookup_z, self.tab_n, s.lookups, True)

    # ------------------------------------------------------------ phase 4: plain (the reference's schedule)

    def _extend(self, coeff, out=None, tmp=None):
        """copy_and_extended_ntt (src/eval_h.rs:324-337): n coefficients ->
        zeta coset values on the 2^(k+e) domain."""
        N = self.n << self.shape.ext_bits
        out = torch.empty((N, 4), dtype=torch.int64, device="cuda") if out is None else out
        out[:self.n].copy_(coeff)
        abi.check(self.sym.extended_prepare(out.data_ptr(), self._coset_powers.data_ptr(), 3, self.n, N, 0, _st()),
                  "extended_prepare")
        tmp = torch.empty_like(out) if tmp is None else tmp
        ntt_raw(self.sym, out, tmp, self.tab_N, False)
        return out

    def _quotient_plain(self, y, beta, gamma):
        s, c, n, u = self.shape, self.c, self.n, self.u
        E, N = self.E, self.n << self.shape.ext_bits
        sym = self.sym
        st = _st()
        self._coset_powers = fr_tensor([ZETA, pow(ZETA, -1, R_MOD)])
        tmpN = torch.empty((N, 4), dtype=torch.int64, device="cuda")
        h = torch.zeros((N, 4), dtype=torch.int64, device="cuda")
        yt, bt, gt = fr_tensor([y]), fr_tensor([beta]), fr_tensor([gamma])
        # gates, grouped as analyze_expr_tree groups them (at most 27 distinct
        # columns per group for k < 23, else 10; src/analyze.rs:31)
        limit = 27 if self.k < 23 else 10
        G = s.gates
        groups, cur, cols = [], [], set()
        for g in range(G):
            need = {("f", c.selector_cols[g])} | {("a", x) for x in c.gate_cols[g]}
            if len(cols | need) > limit and cur:
                groups.append(cur)
                cur, cols = [], set()
            cur.append(g)
            cols |= need
        if cur:
            groups.append(cur)
        ext = {}
        for grp in groups:
            keep = {}
            for g in grp:
                for key in [("f", c.selector_cols[g])] + [("a", x) for x in c.gate_cols[g]]:
                    if key not in keep:
                        keep[key] = ext.pop(key) if key in ext else self._extend(
                            self.fixed_coeff[key[1]] if key[0] == "f" else self.adv_coeff[key[1]], tmp=tmpN)
            ext = keep
            v, rots, keepalive = [], [], []
            for g in grp:
                co = pow(y, G - 1 - g, R_MOD)
                q = keep[("f", c.selector_cols[g])]
                a, b, cc, d, e = [keep[("a", x)] for x in c.gate_cols[g]]
                for coeff, fs in ((co, [q, a, b, cc]), (co, [q, d]), ((-co) % R_MOD, [q, e])):
                    ct = fr_tensor([coeff])
                    keepalive.append(ct)
                    v.append(ct.data_ptr())
                    v.extend(f.data_ptr() for f in fs)
                    rots.extend([0] * len(fs))
                    v.append(0)
            vd = ptr_array(v)
            rd = torch.tensor(rots, dtype=torch.int32, device="cuda")
            abi.check(sym.field_op_batch_mul_sum(h.data_ptr(), vd.data_ptr(), rd.data_ptr(), len(v), N, st),
                      "field_op_batch_mul_sum")
            torch.cuda.synchronize()
        ext.clear()
        l0 = self._extend(self.l_coeff[0], tmp=tmpN)
        ll = self._extend(self.l_coeff[1], tmp=tmpN)
        la = self._extend(self.l_coeff[2], tmp=tmpN)
        last_rot = (n - (s.blinding + 1)) << s.ext_bits
        rot1 = 1 << s.ext_bits
        # permutation (src/eval_h.rs:664-810)
        if s.perm_chunks:
            zext = [self._extend(z, tmp=tmpN) for z in self.perm_z]
            abi.check(sym.permutation_eval_h_p1(h.data_ptr(), zext[0].data_ptr(), zext[-1].data_ptr(), l0.data_ptr(),
                                                ll.data_ptr(), yt.data_ptr(), N), "permutation_eval_h_p1")
            sets = ptr_array([z.data_ptr() for z in zext])
            abi.check(sym.permutation_eval_h_p2(h.data_ptr(), sets.data_ptr(), l0.data_ptr(), ll.data_ptr(),
                                                yt.data_ptr(), len(zext), last_rot, N), "permutation_eval_h_p2")
            torch.cuda.synchronize()
            curr_delta = beta * ZETA % R_MOD
            l_res = torch.empty((N, 4), dtype=torch.int64, device="cuda")
            r_res = torch.empty((N, 4), dtype=torch.int64, device="cuda")
            for j, zj in enumerate(zext):
                r_acc = zj
                l_acc = torch.empty_like(zj)
                # buffer_copy_with_shift (src/cuda/bn254.rs:154-177): l_acc = z(w X)
                l_acc[:N - rot1].copy_(r_acc[rot1:])
                l_acc[N - rot1:].copy_(r_acc[:rot1])
                for ci in range(j * s.chunk_len, min(s.perm, (j + 1) * s.chunk_len)):
                    kd, idx = c.perm_cols[ci]
                    val = {"advice": self.adv_coeff, "fixed": self.fixed_coeff, "instance": self.inst_coeff}[kd][idx]
                    r_res[:n].copy_(val)
                    abi.check(sym.extended_prepare(r_res.data_ptr(), self._coset_powers.data_ptr(), 3, n, N, 0, st),
                              "extended_prepare")
                    diff = fr_tensor([gamma, curr_delta])
                    field_op(r_res, r_res, diff, 0, 2, sym=sym)
                    ntt_raw(sym, r_res, tmpN, self.tab_N, False)
                    field_op(r_acc, r_acc, r_res, 1, N, sym=sym)
                    l_res.zero_()
                    l_res[:n].copy_(val)
                    abi.check(sym.permutation_eval_h_l(l_res.data_ptr(), bt.data_ptr(), gt.data_ptr(),
                                                       self.sigma_coeff[ci].data_ptr(), n, st), "permutation_eval_h_l")
                    self._extend(l_res[:n], out=l_res, tmp=tmpN)
                    field_op(l_acc, l_acc, l_res, 1, N, sym=sym)
                    curr_delta = curr_delta * DELTA % R_MOD
                field_op(l_acc, l_acc, r_acc, 3, N, sym=sym)
                field_op(l_acc, l_acc, la, 1, N, sym=sym)
                field_op(h, h, l_acc, 0, N, l_c=yt, sym=sym)
                torch.cuda.synchronize()
            del zext, l_res, r_res
        # logup lookups (src/eval_h.rs:814-1049), one input per set
        for i, col in enumerate(c.lookup_cols):
            mext = self._extend(self.m_coeff[i], tmp=tmpN)
            inp = self._ntt_and_extend(c.advice[col], bt, tmpN)
            prod = torch.empty_like(inp)
            psum = torch.empty_like(inp)
            sets = ptr_array([inp.data_ptr()])
            abi.check(sym.logup_eval_h_inputs_product_sum(prod.data_ptr(), psum.data_ptr(), sets.data_ptr(), 1, N, st),
                      "logup_eval_h_inputs_product_sum")
            zext = self._extend(self.lookup_z[i], tmp=tmpN)
            text = self._ntt_and_extend(c.fixed[c.table_col], bt, tmpN)
            abi.check(sym.logup_eval_h(h.data_ptr(), prod.data_ptr(), psum.data_ptr(), text.data_ptr(), mext.data_ptr(),
                                       zext.data_ptr(), zext.data_ptr(), l0.data_ptr(), ll.data_ptr(), la.data_ptr(),
                                       yt.data_ptr(), rot1, N, st), "logup_eval_h")
            torch.cuda.synchronize()
            del mext, inp, prod, psum, zext, text
        # shuffles (src/eval_h.rs:1051-1128)
        betas = fr_tensor([pow(beta, i + 1, R_MOD) for i in range(16)])
        for (a, b), z in zip(c.shuffle_pairs, self.shuffle_z):
            zext = self._extend(z, tmp=tmpN)
            ia = self._extend(self.adv_coeff[a], tmp=tmpN)
            ib = self._extend(self.adv_coeff[b], tmp=tmpN)
            pa, pb = ptr_array([ia.data_ptr()]), ptr_array([ib.data_ptr()])
            abi.check(sym.shuffle_eval_h_v2(h.data_ptr(), pa.data_ptr(), pb.data_ptr(), betas.data_ptr(), 1,
                                            zext.data_ptr(), l0.data_ptr(), ll.data_ptr(), la.data_ptr(), yt.data_ptr(),
                                            rot1, N), "shuffle_eval_h_v2")
            torch.cuda.synchronize()
            del zext, ia, ib
        del l0, ll, la
        # divide by Z_H, back to coefficients, undo the coset (src/eval_h.rs:463-510)
        wN = omega(self.ek)
        t_eval = fr_tensor([pow((pow(ZETA * pow(wN, j, R_MOD), n, R_MOD) - 1) % R_MOD, -1, R_MOD) for j in range(E)])
        abi.check(sym.field_mul_zip(h.data_ptr(), t_eval.data_ptr(), E, N), "field_mul_zip")
        ntt_raw(sym, h, tmpN, self.tab_N, True, self.tab_N.n_inv)
        back = fr_tensor([pow(ZETA, -1, R_MOD), ZETA])
        abi.check(sym.extended_prepare(h.data_ptr(), back.data_ptr(), 3, n, N, 1, st), "extended_prepare")
        torch.cuda.synchronize()
        return h

    def _ntt_and_extend(self, lagrange, bt, tmpN):
        """ntt_and_extend_ntt (src/eval_h.rs:339-383): values + beta -> iNTT ->
        extended."""
        n, N = self.n, self.n << self.shape.ext_bits
        buf = torch.empty((N, 4), dtype=torch.int64, device="cuda")
        field_op(buf[:n], lagrange, None, 0, n, r_c=bt, sym=self.sym)
        ntt_raw(self.sym, buf[:n], tmpN[:n], self.tab_n, True, self.tab_n.n_inv)
        return self._extend(buf[:n], out=buf, tmp=tmpN)

    # ------------------------------------------------------------ phase 4: batched (per coset)

    def _quotient_batched(self, y, beta, gamma):
        s, c, n, u = self.shape, self.c, self.n, self.u
        E = self.E
        L = lib()
        st = _st()
        # every coefficient column the constraints read: the witness's, and the
        # proving key's (fixed, sigma, l_0 / l_last / l_active) unless their
        # coset values are cached (setup)
        dyn, pk = self._quotient_rows()
        src = {"adv_coeff": self.adv_coeff, "inst_coeff": self.inst_coeff, "m_coeff": self.m_coeff,
               "lookup_z": self.lookup_z, "fixed_coeff": self.fixed_coeff, "sigma_coeff": self.sigma_coeff,
               "l_coeff": self.l_coeff, "perm_z": _stacked(self.perm_z), "shuffle_z": _stacked(self.shuffle_z)}
        groups = [(name, src[key], cnt) for name, key, cnt in dyn + pk]
        # rows of the per-coset workspace: every group that is not cached for all cosets
        work = [w for w in groups if not all((w[0], j) in self.pk_cos for j in range(E))]
        total = sum(w[2] for w in work)
        ev = self._ws("ev", (max(1, total), n, 4))
        off, base = {}, 0
        for name, _, cnt in work:
            off[name] = base
            base += cnt
        tmp = self._ws("ntt_tmp", (NTT_CHUNK * n, 4))
        yt, bt, gt = fr_tensor([y]), fr_tensor([beta]), fr_tensor([gamma])
        G = s.gates
        coeffs = fr_tensor([pow(y, G - 1 - g, R_MOD) if t < 2 else (-pow(y, G - 1 - g, R_MOD)) % R_MOD
                            for g in range(G) for t in range(3)])
        dbeta = fr_tensor([beta * pow(DELTA, j, R_MOD) for j in range(s.perm)])
        betas = fr_tensor([pow(beta, i + 1, R_MOD) for i in range(16)])
        shuffle_len = torch.ones(max(1, s.shuffles), dtype=torch.int32, device="cuda")
        # one rotation (0) per column entry of the gate terms: 4 + 2 + 2 a gate
        gate_rots = torch.zeros(max(1, 8 * G), dtype=torch.int32, device="cuda")
        kinds = {"advice": "adv", "fixed": "fixed", "instance": "inst"}
        hc = self._ws("hc", (E, n, 4))
        hc.zero_()
        if self.world > 1:
            from . import shard

            mine = shard.coset_ranks(E, self.world)[self.rank]
        else:
            mine = list(range(E))
        for j in mine:
            # this coset's values of every column not cached
            for name, src, cnt in work:
                if (name, j) in self.pk_cos:
                    continue
                self._coset_ntt(ev[off[name]:off[name] + cnt], src, cnt, j, tmp)

            def col(name, i, j=j, pk_cos=self.pk_cos):
                # no reference to self: the last coset's resolver is kept on
                # the prover, and a cycle would hold its HBM past `del`
                cached = pk_cos.get((name, j))
                return cached[i] if cached is not None else ev[off[name] + i]

            # the argument block of zkp_eval_h_fused for this coset
            v = []
            for g in range(G):
                q = col("fixed", c.selector_cols[g])
                a, b, cc, d, e = [col("adv", x) for x in c.gate_cols[g]]
                for t, fs in enumerate(([q, a, b, cc], [q, d], [q, e])):
                    v.append(coeffs[3 * g + t].data_ptr())
                    v.extend(f.data_ptr() for f in fs)
                    v.append(0)
            assert sum(1 for x in v if x) - 3 * G == 8 * G, "gate term layout"
            gate_terms = ptr_array(v)
            perm_cols = ptr_array([col(kinds[kd], i).data_ptr() for kd, i in c.perm_cols])
            perm_sig = ptr_array([col("sigma", i).data_ptr() for i in range(s.perm)])
            perm_z = ptr_array([col("pz", i).data_ptr() for i in range(len(self.perm_z))])
            lk = []
            for i, cl in enumerate(c.lookup_cols):
                lk += [col("adv", cl).data_ptr(), col("fixed", c.table_col).data_ptr(), col("m", i).data_ptr(),
                       col("lz", i).data_ptr()]
            lookup_cols = ptr_array(lk) if lk else None
            sh = []
            for i, (a_, b_) in enumerate(c.shuffle_pairs):
                sh += [col("sz", i).data_ptr(), col("adv", a_).data_ptr(), col("adv", b_).data_ptr()]
            shuffle_cols = ptr_array(sh) if sh else None
            args = _EvalHArgs()
            args.n = n
            args.rot_scale = 1
            args.y = yt.data_ptr()
            args.gate_terms, args.gate_rots, args.gate_terms_n = gate_terms.data_ptr(), gate_rots.data_ptr(), len(v)
            args.l0, args.l_last, args.l_active = col("l", 0).data_ptr(), col("l", 1).data_ptr(), col("l", 2).data_ptr()
            args.beta, args.gamma = bt.data_ptr(), gt.data_ptr()
            args.perm_chunks, args.perm_chunk_len, args.perm_cols_n = len(self.perm_z), s.chunk_len, s.perm
            args.perm_last_rot = -(s.blinding + 1)
            args.perm_z, args.perm_cols, args.perm_sigmas = perm_z.data_ptr(), perm_cols.data_ptr(), perm_sig.data_ptr()
            args.perm_dbeta = dbeta.data_ptr()
            args.lookups, args.lookup_cols = s.lookups, _p(lookup_cols)
            args.shuffles, args.shuffle_cols = s.shuffles, _p(shuffle_cols)
            args.shuffle_group_len, args.shuffle_betas = shuffle_len.data_ptr(), betas.data_ptr()
            args.x = self.coset_x[j].data_ptr()
            args.scale = self.t_inv_dev[j].data_ptr()
            abi.check(L.zkp_eval_h_fused(hc[j].data_ptr(), ctypes.byref(args), st), "zkp_eval_h_fused")
            # keep this coset's pointer arrays referenced until the kernel has
            # read them, and the last coset's inputs for coset_fused_vs_separate
            self._keep = (gate_terms, perm_cols, perm_sig, perm_z, lookup_cols, shuffle_cols)
            self._last_coset = {"j": j, "col": col, "args": args, "h": hc[j],
                                "keep": (gate_terms, gate_rots, perm_cols, perm_sig, perm_z, lookup_cols, shuffle_cols,
                                         coeffs, yt, bt, gt, dbeta, betas, shuffle_len)}
        if self.world > 1:
            shard.gather_cosets(hc, mine, E, self.group)
        # back to the 2^(k+e) coefficients of h
        g = self._ws("hg", (E, n, 4))
        ntt_into(g, hc, self.tab_n, E, True, tmp=tmp)
        out = self._ws("h_coeff", (E * n, 4))
        abi.check(L.zkp_coset_combine(out.data_ptr(), g.data_ptr(), n, self.winv_N.data_ptr(),
                                      self.combine_consts.data_ptr(), self.k, s.ext_bits, st), "zkp_coset_combine")
        torch.cuda.synchronize()
        self._keep = None
        return out

    def coset_fused_vs_separate(self, reps=3):
        """The last proof's last coset evaluated again two ways: one
        zkp_eval_h_fused launch, and the reference symbols one constraint
        family at a time on the same coset rows (field_op_batch_mul_sum,
        permutation_eval_h_p1 / p2, field_op for the chunk products,
        logup_eval_h, shuffle_eval_h_v2, field_op for 1/Z_H), as the
        reference's quotient runs them on its extended buffers.  Returns the
        device milliseconds of each and whether both equal the proof's h on
        that coset."""
        ctx = self._last_coset
        n = self.n
        L = lib()
        st = _st()
        h_f = torch.empty((n, 4), dtype=torch.int64, device="cuda")
        h_s = torch.empty((n, 4), dtype=torch.int64, device="cuda")

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

        fused_ms = timed(lambda: abi.check(L.zkp_eval_h_fused(h_f.data_ptr(), ctypes.byref(ctx["args"]), st),
                                           "zkp_eval_h_fused"))
        launches = [0]
        sep_ms = timed(lambda: self._coset_separate(h_s, ctx, launches))
        return {"rows": n, "coset": ctx["j"], "fused_ms": round(fused_ms, 3), "separate_ms": round(sep_ms, 3),
                "separate_launches": launches[0] // (reps + 1),
                "equal": bool(torch.equal(h_f, ctx["h"]) and torch.equal(h_s, ctx["h"]))}

    def _coset_separate(self, h, ctx, launches):
        s, c, n = self.shape, self.c, self.n
        col, j = ctx["col"], ctx["j"]
        (gate_terms, gate_rots, _, _, _, _, _, _, yt, bt, gt, dbeta, betas, _) = ctx["keep"]
        L = lib()
        st = _st()
        cnt = [0]

        def fo(res, l, r, op, l_c=None, r_c=None, l_rot=0):
            field_op(res, l, r, op, n, l_c=l_c, r_c=r_c, l_rot=l_rot)
            cnt[0] += 1

        h.zero_()
        args = ctx["args"]
        abi.check(L.field_op_batch_mul_sum(h.data_ptr(), args.gate_terms, args.gate_rots, args.gate_terms_n, n, st),
                  "field_op_batch_mul_sum")
        l0, ll, la = col("l", 0), col("l", 1), col("l", 2)
        zs = [col("pz", i) for i in range(s.perm_chunks)]
        abi.check(L.permutation_eval_h_p1(h.data_ptr(), zs[0].data_ptr(), zs[-1].data_ptr(), l0.data_ptr(),
                                          ll.data_ptr(), yt.data_ptr(), n), "permutation_eval_h_p1")
        sets = ptr_array([z.data_ptr() for z in zs])
        abi.check(L.permutation_eval_h_p2(h.data_ptr(), sets.data_ptr(), l0.data_ptr(), ll.data_ptr(), yt.data_ptr(),
                                          len(zs), -(s.blinding + 1), n), "permutation_eval_h_p2")
        cnt[0] += 3
        kinds = {"advice": "adv", "fixed": "fixed", "instance": "inst"}
        X = self.coset_x[j]
        Lb, Rb, t = (torch.empty((n, 4), dtype=torch.int64, device="cuda") for _ in range(3))
        ci = 0
        for zj in zs:
            fo(Lb, zj, None, 2, l_rot=1)
            Rb.copy_(zj)
            for _ in range(s.chunk_len):
                if ci == s.perm:
                    break
                kd, idx = c.perm_cols[ci]
                v, sg = col(kinds[kd], idx), col("sigma", ci)
                fo(t, sg, v, 0, l_c=bt)
                fo(t, t, None, 0, r_c=gt)
                fo(Lb, Lb, t, 1)
                fo(t, X, v, 0, l_c=dbeta[ci:ci + 1])
                fo(t, t, None, 0, r_c=gt)
                fo(Rb, Rb, t, 1)
                ci += 1
            fo(Lb, Lb, Rb, 3)
            fo(Lb, Lb, la, 1)
            fo(h, h, Lb, 0, l_c=yt)
        ones = fr_tensor([1] * 1).expand(n, 4).contiguous()
        for i, cl in enumerate(c.lookup_cols):
            fo(Lb, col("adv", cl), None, 0, r_c=bt)
            fo(Rb, col("fixed", c.table_col), None, 0, r_c=bt)
            abi.check(L.logup_eval_h(h.data_ptr(), Lb.data_ptr(), ones.data_ptr(), Rb.data_ptr(),
                                     col("m", i).data_ptr(), col("lz", i).data_ptr(), col("lz", i).data_ptr(),
                                     l0.data_ptr(), ll.data_ptr(), la.data_ptr(), yt.data_ptr(), 1, n, st),
                      "logup_eval_h")
            cnt[0] += 1
        for i, (a_, b_) in enumerate(c.shuffle_pairs):
            pa, pb = ptr_array([col("adv", a_).data_ptr()]), ptr_array([col("adv", b_).data_ptr()])
            abi.check(L.shuffle_eval_h_v2(h.data_ptr(), pa.data_ptr(), pb.data_ptr(), betas.data_ptr(), 1,
                                          col("sz", i).data_ptr(), l0.data_ptr(), ll.data_ptr(), la.data_ptr(),
                                          yt.data_ptr(), 1, n), "shuffle_eval_h_v2")
            cnt[0] += 1
        fo(h, h, None, 2, l_c=self.t_inv_dev[j:j + 1])
        launches[0] += cnt[0]

    def _coset_ntt(self, out, src, cnt, j, tmp):
        """Coset j of cnt coefficient columns: NTT_n of c_k (zeta w_N^j)^k, over
        (w, w') pair tables when the schedule uses them."""
        if self.pair_tables:
            _ntt_into_pairs(out, src, self.tab_pairs, self.coset_twist_pairs[j], cnt, self.k, tmp,
                            events=self.ntt_events)
        else:
            ntt_into(out, src, self.tab_n, cnt, False, in_mul=self.coset_twist[j], tmp=tmp, events=self.ntt_events)

    # ------------------------------------------------------------ phase 5

    def _queries(self, x):
        """(name, poly tensor, rotation) in the order of src/lib.rs:1084-1150."""
        s, c, n = self.shape, self.c, self.n
        b = s.blinding + 1
        q = []
        if any(kd == "instance" for kd, _ in c.perm_cols):
            q.append(("instance0", self.inst_coeff[0], 0))
        for i in range(s.advice):
            q.append((f"advice{i}", self.adv_coeff[i], 0))
        for j, z in enumerate(self.perm_z):
            q += [(f"perm_z{j}", z, 0), (f"perm_z{j}", z, 1)]
        for j in range(len(self.perm_z) - 2, -1, -1):
            q.append((f"perm_z{j}", self.perm_z[j], -b))
        for i in range(s.lookups):
            q += [(f"m{i}", self.m_coeff[i], 0), (f"lz{i}", self.lookup_z[i], 0), (f"lz{i}", self.lookup_z[i], 1)]
        for j, z in enumerate(self.shuffle_z):
            q += [(f"sz{j}", z, 0), (f"sz{j}", z, 1)]
        for i in range(s.fixed):
            q.append((f"fixed{i}", self.fixed_coeff[i], 0))
        for j in range(s.perm):
            q.append((f"sigma{j}", self.sigma_coeff[j], 0))
        q.append(("h", self.h_fold, 0))
        q.append(("random", self.c.random_poly, 0))
        w = self.tab_n.w
        pts = {0: x, 1: x * w % R_MOD, -b: x * pow(w, -b, R_MOD) % R_MOD}
        return [(nm, t, r, pts[r]) for nm, t, r in q]

    def _evaluate(self, queries):
        """Every (polynomial, point) pair once, in query order of first
        appearance."""
        n = self.n
        pairs = []
        seen = {}
        for nm, t, r, pt in queries:
            if (nm, r) not in seen:
                seen[(nm, r)] = len(pairs)
                pairs.append((nm, t, pt))
        out = [0] * len(pairs)
        if self.schedule == "plain":
            res = H.empty_fr(n)
            for i, (nm, t, pt) in enumerate(pairs):
                xt = fr_tensor([pow(pt, 1 << d, R_MOD) for d in range(self.k)])
                abi.check(self.sym.poly_eval(t.data_ptr(), res.data_ptr(), xt.data_ptr(), n, _st()), "poly_eval")
                out[i] = fr_ints(res[:1])[0]
        else:
            L = lib()
            by_pt = {}
            for i, (nm, t, pt) in enumerate(pairs):
                by_pt.setdefault(pt, []).append(i)
            for pt, idx in by_pt.items():
                pw = powers(1, pt, n)
                polys = ptr_array([pairs[i][1].data_ptr() for i in idx])
                res = H.empty_fr(len(idx))
                scratch = H.empty_fr(L.zkp_poly_eval_batch_scratch_elems(len(idx)))
                abi.check(L.zkp_poly_eval_batch(res.data_ptr(), polys.data_ptr(), len(idx), pw.data_ptr(), n,
                                                scratch.data_ptr(), _st()), "zkp_poly_eval_batch")
                vals = fr_ints(res)
                for i, v_ in zip(idx, vals):
                    out[i] = v_
        self._eval_map = {(pairs[i][0], pairs[i][2]): out[i] for i in range(len(pairs))}
        return out

    # ------------------------------------------------------------ phase 6

    def _gwc(self, tr, queries, evals):
        """src/multiopen.rs:63-170: per rotation, W = sum_q v^(len-1-idx) p_q,
        (W - W(z)) / (X - z), one commitment each."""
        n = self.n
        v = tr.challenge()
        by_rot = {}
        for nm, t, r, pt in queries:
            by_rot.setdefault(r, []).append((nm, t, pt))
        coms = []
        sym = self.sym if self.schedule == "plain" else None
        for r in sorted(by_rot):
            grp = by_rot[r]
            ln = len(grp)
            W = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
            ev = 0
            for idx, (nm, t, pt) in enumerate(grp):
                vp = pow(v, ln - 1 - idx, R_MOD)
                field_op(W, W, t, 0, n, r_c=fr_tensor([vp]), sym=sym)
                ev = (ev + self._eval_map[(nm, pt)] * vp) % R_MOD
            W[0:1] = fr_tensor([(fr_ints(W[0:1])[0] - ev) % R_MOD])
            q = self.hw.divide_linear(self, W, grp[0][2])
            coms.append(q)
        return self.commit(False, coms)

    def _shplonk(self, tr, queries, evals):
        """src/multiopen.rs:283-547."""
        n, k = self.n, self.k
        sym = self.sym if self.schedule == "plain" else None
        y2 = tr.challenge()
        v = tr.challenge()
        rot_pt = {}
        for nm, t, r, pt in queries:
            rot_pt.setdefault(r, pt)
        super_rots = sorted(rot_pt)
        super_pts = [rot_pt[r] for r in super_rots]
        poly_rots, order, tens = {}, [], {}
        for nm, t, r, pt in queries:
            if nm not in poly_rots:
                poly_rots[nm] = set()
                order.append(nm)
                tens[nm] = t
            poly_rots[nm].add(r)
        sets = {}
        for nm in order:
            sets.setdefault(tuple(sorted(poly_rots[nm])), []).append(nm)
        rotation_sets = []
        for rs in sorted(sets):
            pts = [rot_pt[r] for r in rs]
            polys = sets[rs]
            vb = tens[polys[0]].clone()
            acc = _lagrange_interpolate(pts, [self._eval_map[(polys[0], p)] for p in pts])
            yt = fr_tensor([y2])
            for nm in polys[1:]:
                field_op(vb, vb, tens[nm], 0, n, l_c=yt, sym=sym)
                e2 = _lagrange_interpolate(pts, [self._eval_map[(nm, p)] for p in pts])
                acc = [(a * y2 + b) % R_MOD for a, b in zip(acc, e2)]
            rotation_sets.append((pts, vb, acc))
        omegas = self.tab_n.natural
        hx = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
        vt = fr_tensor([v])
        tmp = H.empty_fr(n)
        pb = H.empty_fr(n)
        L = self.sym
        for pts, vb, acc in rotation_sets:
            pb.copy_(vb)
            ev = fr_tensor(acc)
            field_op(pb, pb, ev, 3, len(acc), sym=sym)
            diffs = [p for p in super_pts if p not in pts]
            ntt_raw(L, pb, tmp, self.tab_n, False)
            dt = fr_tensor(diffs) if diffs else fr_tensor([0])
            abi.check(L.shplonk_h_x_merge(hx.data_ptr(), vt.data_ptr(), pb.data_ptr(), omegas.data_ptr(),
                                          dt.data_ptr(), len(diffs), n), "shplonk_h_x_merge")
        spt = fr_tensor(super_pts)
        abi.check(L.shplonk_h_x_div_points(hx.data_ptr(), omegas.data_ptr(), spt.data_ptr(), len(super_pts), n),
                  "shplonk_h_x_div_points")
        ntt_raw(L, hx, tmp, self.tab_n, True, self.tab_n.n_inv)
        c1 = self.commit(False, [hx])
        tr.points(c1)
        uu = tr.challenge()
        zt = 1
        for p in super_pts:
            zt = zt * (uu - p) % R_MOD
        parts = []
        for pts, vb, acc in rotation_sets:
            ev = 0
            for cf in reversed(acc):
                ev = (ev * uu + cf) % R_MOD
            vb[0:1] = fr_tensor([(fr_ints(vb[0:1])[0] - ev) % R_MOD])
            zi = 1
            for p in super_pts:
                if p not in pts:
                    zi = zi * (uu - p) % R_MOD
            parts.append((vb, zi))
        z0inv = pow(parts[0][1], -1, R_MOD)
        fz = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
        for vb, zi in parts:
            field_op(fz, fz, vb, 0, n, l_c=vt, r_c=fr_tensor([zi]), sym=sym)
        field_op(fz, fz, hx, 3, n, r_c=fr_tensor([zt]), sym=sym)
        field_op(fz, fz, None, 2, n, l_c=fr_tensor([z0inv]), sym=sym)
        lx = self.hw.divide_linear(self, fz, uu)
        return c1 + self.commit(False, [lx])


def _stacked(ts):
    """The columns of a list as one (count, n, 4) tensor: the list's own
    storage when its entries are consecutive rows of one tensor (the batched
    schedule's workspaces), else a copy."""
    if not ts:
        return None
    base = ts[0]
    row = base.numel() * base.element_size()
    if all(t.data_ptr() == base.data_ptr() + i * row for i, t in enumerate(ts)):
        return torch.as_strided(base, (len(ts),) + tuple(base.shape), (base.numel(),) + tuple(base.stride()))
    return torch.stack(ts)


def _lagrange_interpolate(points, evals):
    """Coefficients of the polynomial through (points[i], evals[i])
    (halo2's lagrange_interpolate, used by src/multiopen.rs:324, 358)."""
    m = len(points)
    coeffs = [0] * m
    for j in range(m):
        # basis polynomial l_j = prod_{i != j} (X - x_i) / (x_j - x_i)
        num = [1]
        den = 1
        for i in range(m):
            if i == j:
                continue
            num = [(a - points[i] * b) % R_MOD for a, b in zip([0] + num, num + [0])]
            den = den * (points[j] - points[i]) % R_MOD
        f = evals[j] * pow(den, -1, R_MOD) % R_MOD
        for d in range(len(num)):
            coeffs[d] = (coeffs[d] + f * num[d]) % R_MOD
    return coeffs


class _EvalHArgs(ctypes.Structure):
    """zkp_eval_h_args (include/zkwasm_prover_kernel.h)."""
    P = ctypes.c_void_p
    _fields_ = [("n", ctypes.c_uint32), ("rot_scale", ctypes.c_int), ("y", P),
                ("gate_terms", P), ("gate_rots", P), ("gate_terms_n", ctypes.c_int),
                ("l0", P), ("l_last", P), ("l_active", P), ("x", P), ("beta", P), ("gamma", P),
                ("perm_chunks", ctypes.c_int), ("perm_chunk_len", ctypes.c_int), ("perm_cols_n", ctypes.c_int),
                ("perm_last_rot", ctypes.c_int),
                ("perm_z", P), ("perm_cols", P), ("perm_sigmas", P), ("perm_dbeta", P),
                ("lookups", ctypes.c_int), ("lookup_cols", P),
                ("shuffles", ctypes.c_int), ("shuffle_cols", P), ("shuffle_group_len", P), ("shuffle_betas", P),
                ("scale", P)]


class _RefMsm(H.ReferenceMsmBatch):
    """host.ReferenceMsmBatch through a given symbol table."""

    def __init__(self, sym, points, scalars, length):
        super().__init__(points, scalars, length)
        self.sym = sym

    def enqueue(self):
        st = H.stream_handle(self.stream)
        for i, s in enumerate(self.scalars):
            err = self.sym.msm(self.curve_buf.data_ptr() + i * self.region * 96, self.points.data_ptr(), s.data_ptr(),
                               self.idx[0].data_ptr(), self.idx[1].data_ptr(), self.idx[2].data_ptr(),
                               self.idx[3].data_ptr(), self.sort_buf.data_ptr(), self.acc_idx[i].data_ptr(),
                               self.length, self.windows, self.c, self.threads, self.worker,
                               self.sort_buf.numel() * 4, 1, st)
            abi.check(err, "msm")
        r = self.remain
        abi.check(self.sym.batch_msm_collect(r[0].data_ptr(), r[1].data_ptr(), r[2].data_ptr(), r[3].data_ptr(),
                                             self.regions.data_ptr(), self.worker, self.windows, self.c, self.count,
                                             st), "batch_msm_collect")
