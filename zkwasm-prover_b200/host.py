"""Host-side mirror of the reference's GPU wrappers for the proving hot path.

Function names, arguments and buffer sizing follow the reference's Rust
wrappers (src/cuda/ntt.rs, src/cuda/msm.rs, src/cuda/bn254.rs); device buffers
are torch tensors (int64 storage, 4 words per field element, 8 per affine
point, 12 per Jacobian point).  Every call goes through the C ABI of
libzkwasm_prover_kernel.so and raises on a CUDA error status.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import abi

MAX_DEG = 8  # src/cuda/ntt.rs:13


def lib():
    return abi.load_library()


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("zkwasm-prover_b200 needs a CUDA device; there is no CPU fallback")


def stream_handle(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def to_device(arr, device="cuda") -> torch.Tensor:
    """numpy uint64 array -> int64 tensor on the device (same bits)."""
    _require_cuda()
    a = np.ascontiguousarray(np.asarray(arr, dtype=np.uint64))
    return torch.from_numpy(a.view(np.int64)).to(device)


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().contiguous().numpy().view(np.uint64)


def empty_fr(n: int, device="cuda") -> torch.Tensor:
    _require_cuda()
    return torch.empty((n, 4), dtype=torch.int64, device=device)


def zeros_fr(n: int, device="cuda") -> torch.Tensor:
    _require_cuda()
    return torch.zeros((n, 4), dtype=torch.int64, device=device)


def ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def ptr_array(tensors) -> torch.Tensor:
    """Device array of device pointers (the reference's T** arguments)."""
    _require_cuda()
    return torch.tensor([t.data_ptr() for t in tensors], dtype=torch.int64, device="cuda")


# ---------------------------------------------------------------- ntt.rs


def generate_omega_buffers(omega, log_n: int, may_bit_reversed: bool = True, stream=None) -> torch.Tensor:
    """src/cuda/ntt.rs:15-34: upload [1, omega] and expand to w^i, i < 2^log_n."""
    buf = zeros_fr(1 << log_n)
    one = np.asarray(omega, np.uint64).reshape(1, 4)
    from_host = np.zeros((2, 4), np.uint64)
    from_host[0] = _mont_one()
    from_host[1] = one
    buf[:2].copy_(to_device(from_host))
    torch.cuda.synchronize()
    abi.check(lib().expand_omega_buffer(ptr(buf), log_n, int(may_bit_reversed)), "expand_omega_buffer")
    torch.cuda.synchronize()
    return buf


def _mont_one():
    # 2^256 mod r as 4 u64 limbs
    r = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
    one = (1 << 256) % r
    return np.array([(one >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)], np.uint64)


def generate_ntt_buffers(omega, log_n: int):
    """src/cuda/ntt.rs:36-59: (omegas_buf, pq_buf).  The pq table is unused by
    this library's ntt and kept as a one-element placeholder."""
    omegas = generate_omega_buffers(omega, log_n, True)
    pq = zeros_fr(1)
    return omegas, pq


def ntt_raw(s_buf, tmp_buf, pq_buf, omegas_buf, log_n: int, intt_divisor=None, stream=None):
    """src/cuda/ntt.rs:61-93: returns (s_buf, tmp_buf), swapped when the result
    landed in tmp."""
    swap = ctypes.c_bool(False)
    err = lib().ntt(ptr(s_buf), ptr(tmp_buf), ptr(pq_buf), ptr(omegas_buf), ptr(intt_divisor), log_n, MAX_DEG,
                    ctypes.addressof(swap), stream_handle(stream))
    abi.check(err, "ntt")
    if swap.value:
        return tmp_buf, s_buf
    return s_buf, tmp_buf


def extended_prepare(s, coset_powers, coset_powers_n: int, size: int, extended_size: int, to_coset: bool,
                     stream=None):
    """src/cuda/ntt.rs:111-135."""
    abi.check(lib().extended_prepare(ptr(s), ptr(coset_powers), coset_powers_n, size, extended_size,
                                     1 if to_coset else 0, stream_handle(stream)), "extended_prepare")


# ---------------------------------------------------------------- msm.rs


def msm_window_bits(msm_count: int, length: int) -> int:
    """src/cuda/msm.rs:105: the reference's window heuristic (its scratch sizing)."""
    def log2_ceil(x):
        return max(0, (x - 1).bit_length())
    return min(log2_ceil(msm_count), 3) + 10 + max(log2_ceil(length), 22) - 22


class ReferenceMsmBatch:
    """The buffers and calls of src/cuda/msm.rs:239-455 through the drop-in
    msm + batch_msm_collect symbols, with the reference's scratch sizing:
    one region of (windows << c) + 2 * workers Jacobian points per MSM, a
    shared sort buffer of 3 * length * windows u32, and the device array of
    region pointers batch_msm_collect takes."""

    def __init__(self, points_buf, scalar_bufs, length: int, stream=None):
        threads, bits = 64, 254
        self.points, self.scalars, self.length = points_buf, list(scalar_bufs), length
        self.count = count = len(self.scalars)
        self.c = c = msm_window_bits(count, length)
        self.windows = windows = (bits + c - 1) // c
        bucket_size = windows << c
        max_worker = 128 * 512
        self.worker = (length + threads - 1) // threads * threads if length < max_worker else max_worker
        self.threads = threads
        self.region = bucket_size + self.worker * 2
        self.curve_buf = torch.empty((count * self.region, 12), dtype=torch.int64, device="cuda")
        single = length * windows
        self.sort_buf = torch.empty(max(1, single * 3), dtype=torch.int32, device="cuda")
        self.idx = [torch.empty(max(1, single), dtype=torch.int32, device="cuda") for _ in range(4)]
        self.acc_idx = [torch.empty(max(1, self.worker * 2), dtype=torch.int32, device="cuda") for _ in range(count)]
        # device arrays of the per-MSM region pointers and of the worker
        # remainders inside each region (src/cuda/msm.rs:387-420): this
        # library's batch_msm_collect reads the regions only, the reference's
        # kernels all five
        base = self.curve_buf.data_ptr()
        bucket = windows << c

        def ptrs(xs):
            return torch.tensor(xs, dtype=torch.int64, device="cuda")

        self.regions = ptrs([base + i * self.region * 96 for i in range(count)])
        self.remain = (ptrs([a.data_ptr() for a in self.acc_idx]),
                       ptrs([base + (i * self.region + bucket) * 96 for i in range(count)]),
                       ptrs([a.data_ptr() + self.worker * 4 for a in self.acc_idx]),
                       ptrs([base + (i * self.region + bucket + self.worker) * 96 for i in range(count)]))
        self.stream = stream

    def enqueue(self):
        """msm per column, then batch_msm_collect; no host synchronisation."""
        st = stream_handle(self.stream)
        for i, s in enumerate(self.scalars):
            err = lib().msm(self.curve_buf.data_ptr() + i * self.region * 96, ptr(self.points), ptr(s),
                            ptr(self.idx[0]), ptr(self.idx[1]), ptr(self.idx[2]), ptr(self.idx[3]),
                            ptr(self.sort_buf), ptr(self.acc_idx[i]), self.length, self.windows, self.c,
                            self.threads, self.worker, self.sort_buf.numel() * 4, 1, st)
            abi.check(err, "msm")
        r = self.remain
        abi.check(lib().batch_msm_collect(ptr(r[0]), ptr(r[1]), ptr(r[2]), ptr(r[3]), ptr(self.regions), self.worker,
                                          self.windows, self.c, self.count, st), "batch_msm_collect")

    def results(self):
        """Jacobian results as a numpy (count, 12) uint64 array (synchronises)."""
        torch.cuda.synchronize()
        return to_host(torch.stack([self.curve_buf[i * self.region] for i in range(self.count)]))


def batch_msm(points_buf, scalar_bufs, length: int, stream=None):
    """src/cuda/msm.rs:239-455 through the drop-in msm + batch_msm_collect
    symbols, with the reference's scratch sizing.  Returns Jacobian points as a
    numpy (B, 12) uint64 array."""
    b = ReferenceMsmBatch(points_buf, scalar_bufs, length, stream)
    b.enqueue()
    return b.results()


def msm_scratch(n: int, window_bits: int = 0) -> torch.Tensor:
    nbytes = lib().zkp_msm_scratch_bytes(n, window_bits)
    return torch.empty(max(1, nbytes), dtype=torch.uint8, device="cuda")


def msm(points_buf, scalars_buf, n: int | None = None, window_bits: int = 0, scratch=None, out=None, stream=None):
    """One MSM through zkp_msm; returns the 96-byte Jacobian result as a (12,)
    int64 device tensor (no host synchronisation)."""
    n = scalars_buf.shape[0] if n is None else n
    if scratch is None:
        scratch = msm_scratch(n, window_bits)
    if out is None:
        out = torch.empty(12, dtype=torch.int64, device="cuda")
    err = lib().zkp_msm(ptr(out), ptr(points_buf), ptr(scalars_buf), n, window_bits, ptr(scratch),
                        scratch.numel(), stream_handle(stream))
    abi.check(err, "zkp_msm")
    return out


def msm_table_build(bases_buf, nsrs: int | None = None, window_bits: int = 0, stream=None, table=None):
    """zkp_msm_table_build: the table of pre-multiplied bases (and their
    endomorphism images) for MSMs over the resident bases_buf[:nsrs];
    window_bits 0 picks the library's width for nsrs points; table, if
    given, is a device buffer of at least zkp_msm_table_bytes.  Returns
    (table, window_bits)."""
    nsrs = bases_buf.shape[0] if nsrs is None else nsrs
    c = window_bits or lib().zkp_msm_table_default_window(nsrs)
    nbytes = lib().zkp_msm_table_bytes(nsrs, c)
    if nbytes == 0:
        raise ValueError(f"unsupported table window width {c}")
    if table is None:
        table = torch.empty(nbytes // 8, dtype=torch.int64, device="cuda")
    elif table.numel() * table.element_size() < nbytes:
        raise ValueError(f"table buffer holds {table.numel() * table.element_size()} bytes, {nbytes} needed")
    abi.check(lib().zkp_msm_table_build(ptr(table), ptr(bases_buf), nsrs, c, stream_handle(stream)),
              "zkp_msm_table_build")
    return table, c


def msm_table(table, nsrs: int, window_bits: int, scalars_buf, n: int | None = None, scratch=None, out=None,
              stream=None):
    """One MSM over a table from msm_table_build (same nsrs and window_bits);
    returns the 96-byte Jacobian result as a (12,) int64 device tensor."""
    n = scalars_buf.shape[0] if n is None else n
    if scratch is None:
        nbytes = lib().zkp_msm_table_scratch_bytes(n, window_bits)
        scratch = torch.empty(max(1, nbytes), dtype=torch.uint8, device="cuda")
    if out is None:
        out = torch.empty(12, dtype=torch.int64, device="cuda")
    err = lib().zkp_msm_table(ptr(out), ptr(table), nsrs, window_bits, ptr(scalars_buf), n, ptr(scratch),
                              scratch.numel(), stream_handle(stream))
    abi.check(err, "zkp_msm_table")
    return out


def msm_batch_table(table, nsrs: int, window_bits: int, scalar_bufs, ns, scratch=None, out=None, stream=None,
                    ptrs=None):
    """zkp_msm_batch_table: len(scalar_bufs) MSMs over prefixes of the bases
    of one table (msm_table_build); returns (count, 12) int64 Jacobian points.
    ptrs: the device array of scalar pointers, prepared beforehand (required
    under CUDA-graph capture, where no host-to-device copy may run)."""
    count = len(scalar_bufs)
    n_arr = (ctypes.c_uint32 * count)(*[int(x) for x in ns])
    ptrs = ptr_array(scalar_bufs) if ptrs is None else ptrs
    if scratch is None:
        nbytes = lib().zkp_msm_batch_table_scratch_bytes(ctypes.addressof(n_arr), count, nsrs, window_bits)
        if nbytes == 0:
            raise ValueError("batch does not fit one table pipeline")
        scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    if out is None:
        out = torch.empty((count, 12), dtype=torch.int64, device="cuda")
    err = lib().zkp_msm_batch_table(ptr(out), ptr(table), nsrs, window_bits, ptr(ptrs), ctypes.addressof(n_arr),
                                    count, ptr(scratch), scratch.numel(), stream_handle(stream))
    abi.check(err, "zkp_msm_batch_table")
    out._keep = (ptrs, scratch)
    return out


def msm_batch(bases_buf, scalar_bufs, ns, windows=None, scratch=None, out=None, stream=None, ptrs=None):
    """zkp_msm_batch: one pipeline for len(scalar_bufs) MSMs over the prefix
    bases_buf[:ns[i]]; returns (count, 12) int64 Jacobian points on the device.
    ptrs: the device array of scalar pointers, prepared beforehand (required
    under CUDA-graph capture, where no host-to-device copy may run)."""
    count = len(scalar_bufs)
    n_arr = (ctypes.c_uint32 * count)(*[int(x) for x in ns])
    c_arr = None if windows is None else (ctypes.c_int * count)(*[int(x) for x in windows])
    ptrs = ptr_array(scalar_bufs) if ptrs is None else ptrs
    if scratch is None:
        nbytes = lib().zkp_msm_batch_scratch_bytes(ctypes.addressof(n_arr),
                                                   None if c_arr is None else ctypes.addressof(c_arr), count)
        scratch = torch.empty(max(1, nbytes), dtype=torch.uint8, device="cuda")
    if out is None:
        out = torch.empty((count, 12), dtype=torch.int64, device="cuda")
    err = lib().zkp_msm_batch(ptr(out), ptr(bases_buf), ptr(ptrs), ctypes.addressof(n_arr),
                              None if c_arr is None else ctypes.addressof(c_arr), count, ptr(scratch),
                              scratch.numel(), stream_handle(stream))
    abi.check(err, "zkp_msm_batch")
    out._keep = (ptrs, scratch)  # keep device operands alive with the result
    return out


# ---------------------------------------------------------------- batched phases


def twist_tables(shift, w_ext, log_n: int, ext_bits: int, tw, stream=None) -> torch.Tensor:
    """Coset tables for zkp_extend_batch (tw: natural w_n table)."""
    t = empty_fr(lib().zkp_coset_table_elems(log_n, ext_bits))
    sh = to_device(np.asarray(shift, np.uint64).reshape(1, 4))
    we = to_device(np.asarray(w_ext, np.uint64).reshape(1, 4))
    abi.check(lib().zkp_coset_twist_tables(ptr(t), ptr(sh), ptr(we), log_n, ext_bits, ptr(tw),
                                           stream_handle(stream)), "zkp_coset_twist_tables")
    torch.cuda.synchronize()
    return t


def extend_batch(ext_out, coeff_out, lagrange_in, ncols: int, log_n: int, ext_bits: int, tw_inv, n_inv, tw, twist,
                 scratch, stage_events=None, stream=None):
    """zkp_extend_batch: iNTT of ncols Lagrange columns, then the coset
    evaluation on the 2^ext_bits-times larger domain.  stage_events: optional
    ctypes array of 5 cudaEvent_t handles recorded around the stages."""
    abi.check(lib().zkp_extend_batch(ptr(ext_out), ptr(coeff_out), ptr(lagrange_in), ncols, log_n, ext_bits,
                                     ptr(tw_inv), ptr(n_inv), ptr(tw), ptr(twist), ptr(scratch),
                                     None if stage_events is None else ctypes.addressof(stage_events),
                                     stream_handle(stream)), "zkp_extend_batch")


def extend_tables(tw, tw_inv, n_inv, shift, w_ext, log_n: int, ext_bits: int, stream=None) -> torch.Tensor:
    """Tables of zkp_extend_batch_tables: every twiddle, twist and scale as a
    (w, w') pair for products by a known factor (tw, tw_inv: natural w_n and
    w_n^-1 tables; n_inv on the device; shift, w_ext as Montgomery limbs)."""
    t = empty_fr(lib().zkp_extend_table_elems(log_n, ext_bits))
    sh = to_device(np.asarray(shift, np.uint64).reshape(1, 4))
    we = to_device(np.asarray(w_ext, np.uint64).reshape(1, 4))
    abi.check(lib().zkp_extend_tables(ptr(t), ptr(tw), ptr(tw_inv), ptr(n_inv), ptr(sh), ptr(we), log_n, ext_bits,
                                      stream_handle(stream)), "zkp_extend_tables")
    torch.cuda.synchronize()
    return t


def extend_batch_tables(ext_out, coeff_out, lagrange_in, ncols: int, log_n: int, ext_bits: int, tables, scratch,
                        stage_events=None, stream=None):
    """zkp_extend_batch_tables: extend_batch over the pair tables of
    extend_tables."""
    abi.check(lib().zkp_extend_batch_tables(ptr(ext_out), ptr(coeff_out), ptr(lagrange_in), ncols, log_n, ext_bits,
                                            ptr(tables), ptr(scratch),
                                            None if stage_events is None else ctypes.addressof(stage_events),
                                            stream_handle(stream)), "zkp_extend_batch_tables")


def ntt_batch(buf, tmp, omegas, log_n: int, ncols: int, scale=None, stream=None):
    res = ctypes.c_int(0)
    abi.check(lib().zkp_ntt_batch(ptr(buf), ptr(tmp), ptr(omegas), ptr(scale), log_n, ncols, 1 << log_n,
                                  ctypes.addressof(res), stream_handle(stream)), "zkp_ntt_batch")
    return tmp if res.value else buf


def ntt_default_plan(log_n: int) -> list:
    rad = (ctypes.c_int * 4)()
    k = lib().zkp_ntt_default_plan(log_n, ctypes.addressof(rad))
    return [rad[i] for i in range(k)]


def ntt_batch_plan(buf, tmp, omegas, log_n: int, ncols: int, radices, scale=None, stream=None):
    """zkp_ntt_batch with the pass radices given (log2 each)."""
    rad = (ctypes.c_int * len(radices))(*[int(r) for r in radices])
    res = ctypes.c_int(0)
    abi.check(lib().zkp_ntt_batch_plan(ptr(buf), ptr(tmp), ptr(omegas), ptr(scale), log_n, ncols, 1 << log_n,
                                       ctypes.addressof(rad), len(radices), ctypes.addressof(res),
                                       stream_handle(stream)), "zkp_ntt_batch_plan")
    return tmp if res.value else buf


def scan_scratch(n: int) -> torch.Tensor:
    return empty_fr(max(1, lib().zkp_scan_scratch_elems(n)))


def batch_inverse(out, inp, c=None, accumulate=False, scratch=None, stream=None):
    """out = (accumulate ? out : 0) + 1 / (inp + c); scratch from scan_scratch(n)
    (or None for one field inversion per 2048 elements)."""
    abi.check(lib().zkp_batch_inverse(ptr(out), ptr(inp), ptr(c), inp.shape[0], int(accumulate), ptr(scratch),
                                      stream_handle(stream)), "zkp_batch_inverse")


def grand_product(out, inp, init=None, scratch=None, stream=None):
    n = inp.shape[0]
    scratch = scan_scratch(n) if scratch is None else scratch
    abi.check(lib().zkp_grand_product(ptr(out), ptr(inp), n, ptr(init), ptr(scratch), stream_handle(stream)),
              "zkp_grand_product")


def grand_sum(out, inp, init=None, scratch=None, stream=None):
    n = inp.shape[0]
    scratch = scan_scratch(n) if scratch is None else scratch
    abi.check(lib().zkp_grand_sum(ptr(out), ptr(inp), n, ptr(init), ptr(scratch), stream_handle(stream)),
              "zkp_grand_sum")


# ------------------------------------------------------------- host staging


class HostPool:
    """Page-locked (optionally huge-page) host chunks for column transfers
    (zkp_host_pool_*; replaces src/hugetlb.rs).  flags: 1 = pin, 2 = huge pages."""

    PIN, HUGE = 1, 2

    def __init__(self, chunk_bytes: int, chunks_per_block: int = 2, flags: int = 3):
        self.chunk = chunk_bytes
        self.h = lib().zkp_host_pool_create(chunk_bytes, chunks_per_block, flags)
        if not self.h:
            raise MemoryError("zkp_host_pool_create failed")

    def alloc(self, nbytes: int) -> int:
        p = lib().zkp_host_pool_alloc(self.h, nbytes)
        if not p:
            raise MemoryError("zkp_host_pool_alloc failed")
        return p

    def free(self, p: int):
        if lib().zkp_host_pool_free(self.h, p) != 0:
            raise ValueError("pointer not from this pool (or freed twice)")

    def stats(self):
        b, u = ctypes.c_size_t(), ctypes.c_size_t()
        lib().zkp_host_pool_stats(self.h, ctypes.byref(b), ctypes.byref(u))
        return b.value, u.value

    @staticmethod
    def view(p: int, nbytes: int, dtype=np.uint8) -> np.ndarray:
        """numpy view of pool memory (no copy)."""
        buf = (ctypes.c_char * nbytes).from_address(p)
        return np.frombuffer(buf, dtype=dtype)

    def close(self):
        if self.h:
            lib().zkp_host_pool_destroy(self.h)
            self.h = None


class CopyQueue:
    """Bounded asynchronous copy queue (zkp_copy_queue_*; replaces
    src/async_copy_queue.rs)."""

    H2D, D2H, D2D = 1, 2, 3  # cudaMemcpyKind

    def __init__(self, max_in_flight: int = 2, device: int = 0):
        self.h = lib().zkp_copy_queue_create(max_in_flight, device)
        if not self.h:
            raise RuntimeError("zkp_copy_queue_create failed")

    def push(self, dst: int, src: int, nbytes: int, kind: int, after=None):
        abi.check(lib().zkp_copy_queue_push(self.h, dst, src, nbytes, kind, stream_handle(after)),
                  "zkp_copy_queue_push")

    def sync(self):
        abi.check(lib().zkp_copy_queue_sync(self.h), "zkp_copy_queue_sync")

    def close(self):
        if self.h:
            lib().zkp_copy_queue_destroy(self.h)
            self.h = None
