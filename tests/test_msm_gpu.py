"""MSM parity on the GPU: zkp_msm and the reference-compatible msm +
batch_msm_collect pair (with the reference host's scratch sizing,
src/cuda/msm.rs:239-455) against the oracle, compared as affine points."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _jac_to_aff(O, j):
    return O.g1_jac_to_aff(np.asarray(j, np.uint64).reshape(-1, 12))


def _run(gpu, bases, scalars, c=0):
    H = gpu.host
    out = H.msm(H.to_device(bases), H.to_device(scalars), n=scalars.shape[0], window_bits=c)
    torch.cuda.synchronize()
    return H.to_host(out)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 100, 1000])
def test_msm_small_vs_oracle(O, gpu, n):
    d = O.rand_fr(n, 10 + n)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 20 + n)
    got = _jac_to_aff(O, _run(gpu, bases, s))
    assert (got == O.msm(bases, s)).all()


@pytest.mark.parametrize("c", [4, 8, 11, 13, 16])
def test_msm_window_widths(O, gpu, c):
    n = 3000
    d = O.rand_fr(n, 31)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 32)
    assert (_jac_to_aff(O, _run(gpu, bases, s, c)) == O.msm_known_dlog(d, s)).all()


def test_msm_edge_cases(O, gpu):
    n = 512
    d = O.rand_fr(n, 41)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 42)
    s[0:50] = 0                               # zero scalars
    s[50:60] = O.fr(O.R_MOD - 1)              # r - 1 (all-ones-ish digits)
    s[60:70] = O.fr(1)
    bases[70:80] = 0                          # identity bases (0, 0)
    d[70:80] = 0
    s[80:90] = O.fr((1 << 253) + 1)           # top window set
    bases[100] = bases[101]                   # repeated point -> doubling branch
    d[100] = d[101]
    s[100] = s[101]
    assert (_jac_to_aff(O, _run(gpu, bases, s)) == O.msm_known_dlog(d, s)).all()


def test_msm_all_scalars_equal(O, gpu):
    # one bucket per window holds every point: runs span many accumulation slices
    n = 1 << 14
    d = O.rand_fr(n, 51)
    bases = O.g1_gen_bases(d)
    s = np.repeat(O.rand_fr(1, 52), n, axis=0)
    assert (_jac_to_aff(O, _run(gpu, bases, s)) == O.msm_known_dlog(d, s)).all()


@pytest.mark.parametrize("c", [9, 12, 14, 18])
def test_msm_narrow_top_window(O, gpu, c):
    # 254 = q c + 1 or 2: the top window has 1-2 bits, so a handful of buckets
    # there hold every point and the merge reduces runs over thousands of slices
    n = 1 << 16
    d = O.rand_fr(n, 53)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 54 + c)
    assert (_jac_to_aff(O, _run(gpu, bases, s, c)) == O.msm_known_dlog(d, s)).all()


def test_msm_few_distinct_scalars(O, gpu):
    # witness-like columns: 90% of the scalars take one of three values
    n = 1 << 15
    d = O.rand_fr(n, 55)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 56)
    rng = np.random.default_rng(57)
    pick = rng.random(n)
    vals = O.fr_vec([1, 2, (1 << 64) + 3])
    s[pick < 0.3] = vals[0]
    s[(pick >= 0.3) & (pick < 0.6)] = vals[1]
    s[(pick >= 0.6) & (pick < 0.9)] = vals[2]
    for c in (0, 10, 16):
        assert (_jac_to_aff(O, _run(gpu, bases, s, c)) == O.msm_known_dlog(d, s)).all(), c


def test_msm_zero_result_and_empty(O, gpu):
    d = O.rand_fr(2, 61)
    bases = O.g1_gen_bases(d)
    # [k]P + [k](-P) = identity
    bases[1] = bases[0]
    bases[1, 4:] = O.neg(bases[0, 4:], 1)
    s = np.repeat(O.rand_fr(1, 62), 2, axis=0)
    j = _run(gpu, bases, s)
    assert O.fq_ints(j[8:])[0] == 0
    H = gpu.host
    out = H.msm(H.to_device(bases), H.to_device(s), n=0)
    torch.cuda.synchronize()
    assert O.fq_ints(H.to_host(out)[8:])[0] == 0


def test_msm_known_dlog_2_18(O, gpu):
    # the single-MSM benchmark size (n = 2^18), reference test identity
    n = 1 << 18
    d = O.rand_fr(n, 71)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 72)
    assert (_jac_to_aff(O, _run(gpu, bases, s)) == O.msm_known_dlog(d, s)).all()


def test_g1_multiples_generator(O, gpu):
    # device-generated bases with known 64-bit discrete logs (benchmark data)
    H = gpu.host
    rng = np.random.default_rng(5)
    k = rng.integers(0, 2 ** 63, 4096, dtype=np.int64).astype(np.uint64)
    k[:3] = [0, 1, 2]
    kd = torch.from_numpy(k.view(np.int64)).cuda()
    out = torch.empty((k.shape[0], 8), dtype=torch.int64, device="cuda")
    gpu.abi.check(gpu.load_library().zkp_g1_multiples(out.data_ptr(), kd.data_ptr(), k.shape[0], H.stream_handle()))
    got = H.to_host(out)
    dl = O.fr_vec([int(x) for x in k])
    assert (got == O.g1_gen_bases(dl)).all()
    s = O.rand_fr(k.shape[0], 6)
    assert (_jac_to_aff(O, _run(gpu, got, s)) == O.msm_known_dlog(dl, s)).all()


def test_msm_batch_uneven(O, gpu):
    # uneven sizes over one base array, mixed scalar distributions, mixed
    # window widths, an empty MSM and a single-point MSM
    H = gpu.host
    nmax = 1 << 13
    d = O.rand_fr(nmax, 91)
    bases = H.to_device(O.g1_gen_bases(d))
    rng = np.random.default_rng(92)
    ns = [nmax, 1000, 1, 0, 4096, 300, 2048, 5000]
    ws = [0, 9, 4, 0, 13, 6, 0, 11]
    cols = []
    for i, n in enumerate(ns):
        s = O.rand_fr(max(n, 1), 100 + i)[:n]
        if i == 4:  # small, witness-like scalars
            s = O.fr_vec([int(x) for x in rng.integers(0, 1 << 20, n)])
        if i == 6:  # sparse
            s[rng.random(n) < 0.9] = 0
        cols.append(s)
    dev_cols = [H.to_device(c) if c.shape[0] else H.empty_fr(1) for c in cols]
    out = H.msm_batch(bases, dev_cols, ns, ws)
    torch.cuda.synchronize()
    got = H.to_host(out)
    for i, (n, s) in enumerate(zip(ns, cols)):
        exp = O.msm_known_dlog(d[:n], s) if n else np.zeros((1, 8), np.uint64)
        assert (_jac_to_aff(O, got[i]) == exp).all(), i


def test_msm_batch_many_buckets(O, gpu):
    # 40 MSMs with 17-bit windows over the 127-bit GLV halves: 40 * 8 * 2^16 =
    # 21M buckets, more than one pass of the top-level bucket-offset scan
    # (4096 * 4096) covers
    H = gpu.host
    n = 512
    d = O.rand_fr(n, 95)
    bases = H.to_device(O.g1_gen_bases(d))
    cols = [O.rand_fr(n, 200 + i) for i in range(40)]
    ns, ws = [n] * 40, [17] * 40
    out = H.msm_batch(bases, [H.to_device(c) for c in cols], ns, ws)
    torch.cuda.synchronize()
    got = H.to_host(out)
    for i in (0, 17, 39):
        assert (_jac_to_aff(O, got[i]) == O.msm_known_dlog(d, cols[i])).all(), i


@pytest.mark.parametrize("n", [1 << 12, 1 << 16])
def test_reference_abi_batch_msm(O, gpu, n):
    # msm() per column + batch_msm_collect, buffers sized like src/cuda/msm.rs;
    # msm() places its scratch in the sort buffer and the region as fits
    H = gpu.host
    d = O.rand_fr(n, 81)
    bases = H.to_device(O.g1_gen_bases(d))
    cols = [O.rand_fr(n, 82 + i) for i in range(3)]
    cols[1][::3] = 0
    res = H.batch_msm(bases, [H.to_device(c) for c in cols], n)
    for i, c in enumerate(cols):
        assert (_jac_to_aff(O, res[i]) == O.msm_known_dlog(d, c)).all()


# ------------------------------------------------------- pre-multiplied base tables

def _table_run(gpu, table, nsrs, c, scalars):
    H = gpu.host
    out = H.msm_table(table, nsrs, c, H.to_device(scalars), n=scalars.shape[0])
    torch.cuda.synchronize()
    return H.to_host(out)


@pytest.mark.parametrize("c", [4, 7, 13, 22])
def test_msm_table_entries(O, gpu, c):
    # entry j 2N + i = [2^(c j) d_i] G and entry j 2N + N + i = [lambda 2^(c j) d_i] G
    N = 37
    d = O.rand_fr(N, 80 + c)
    d[5] = 0                                   # identity base
    bases = O.g1_gen_bases(d)
    H = gpu.host
    table, cc = H.msm_table_build(H.to_device(bases), N, c)
    assert cc == c
    torch.cuda.synchronize()
    t = H.to_host(table).reshape(-1, 8)
    W = (128 + c - 1) // c
    assert t.shape[0] == W * 2 * N
    dl = O.fr_ints(d)
    for j in range(W):
        m = pow(2, c * j, O.R_MOD)
        assert (t[j * 2 * N: j * 2 * N + N] == O.g1_gen_bases(O.fr_vec([x * m for x in dl]))).all(), j
        assert (t[j * 2 * N + N: (j + 1) * 2 * N] ==
                O.g1_gen_bases(O.fr_vec([x * m * O.GLV_LAMBDA for x in dl]))).all(), j


@pytest.mark.parametrize("c", [5, 9, 13, 16, 22])
def test_msm_table_widths(O, gpu, c):
    N = 3000
    d = O.rand_fr(N, 90)
    bases = O.g1_gen_bases(d)
    H = gpu.host
    table, _ = H.msm_table_build(H.to_device(bases), N, c)
    for n in (N, 1, 2, 777):                   # the whole table and prefixes of it
        s = O.rand_fr(n, 91 + n)
        got = _jac_to_aff(O, _table_run(gpu, table, N, c, s))
        assert (got == O.msm_known_dlog(d[:n], s)).all(), (c, n)


def test_msm_table_edge_cases(O, gpu):
    n = 2048
    d = O.rand_fr(n, 95)
    s = O.rand_fr(n, 96)
    s[0:50] = 0
    s[50:60] = O.fr(O.R_MOD - 1)
    s[60:70] = O.fr(1)
    d[70:80] = 0                               # identity bases
    s[80:90] = O.fr((1 << 253) + 1)
    d[100] = d[101]                            # repeated point: doubling in a bucket
    s[100] = s[101]
    s[200:1200] = s[3]                         # one bucket per window holds 1000 points
    bases = O.g1_gen_bases(d)
    H = gpu.host
    for c in (0, 8, 16):
        table, cc = H.msm_table_build(H.to_device(bases), n, c)
        got = _jac_to_aff(O, _table_run(gpu, table, n, cc, s))
        assert (got == O.msm_known_dlog(d, s)).all(), c


def test_msm_table_zero_result_and_empty(O, gpu):
    d = O.rand_fr(2, 97)
    d[1] = O.fr(O.R_MOD - O.fr_ints(d[:1])[0])  # base 1 = -base 0
    bases = O.g1_gen_bases(d)
    H = gpu.host
    table, c = H.msm_table_build(H.to_device(bases), 2, 0)
    s = np.repeat(O.rand_fr(1, 98), 2, axis=0)
    assert O.fq_ints(_table_run(gpu, table, 2, c, s)[8:])[0] == 0
    out = H.msm_table(table, 2, c, H.to_device(s), n=0)
    torch.cuda.synchronize()
    assert O.fq_ints(H.to_host(out)[8:])[0] == 0


def test_msm_table_2_18_matches_plain(O, gpu):
    # the benchmark size through the default table width, against the known
    # discrete log and the plain MSM on the same inputs
    n = 1 << 18
    d = O.rand_fr(n, 99)
    bases = O.g1_gen_bases(d)
    s = O.rand_fr(n, 100)
    H = gpu.host
    table, c = H.msm_table_build(H.to_device(bases), n, 0)
    got = _table_run(gpu, table, n, c, s)
    assert (_jac_to_aff(O, got) == O.msm_known_dlog(d, s)).all()
    assert (_jac_to_aff(O, got) == _jac_to_aff(O, _run(gpu, bases, s))).all()


def test_msm_table_rejects_bad_arguments(gpu):
    L = gpu.load_library()
    assert L.zkp_msm_table_bytes(100, 3) == 0 and L.zkp_msm_table_bytes(100, 23) == 0
    assert L.zkp_msm_table_scratch_bytes(100, 3) == 0
    # n above the table's points, and a table too large for 31-bit entry indices
    assert L.zkp_msm_table(1, 1, 10, 16, 1, 11, 1, 1 << 30, None) != 0
    assert L.zkp_msm_table_build(1, 1, 1 << 28, 4, None) != 0


@pytest.mark.parametrize("c", [6, 13, 16])
def test_msm_batch_table_uneven(O, gpu, c):
    # the uneven batch of test_msm_batch_uneven over one table of the bases
    H = gpu.host
    nmax = 1 << 13
    d = O.rand_fr(nmax, 191)
    bases = H.to_device(O.g1_gen_bases(d))
    table, _ = H.msm_table_build(bases, nmax, c)
    rng = np.random.default_rng(192)
    ns = [nmax, 1000, 1, 0, 4096, 300, 2048, 5000]
    cols = []
    for i, n in enumerate(ns):
        s = O.rand_fr(max(n, 1), 300 + i)[:n]
        if i == 4:
            s = O.fr_vec([int(x) for x in rng.integers(0, 1 << 20, n)])
        if i == 6:
            s[rng.random(n) < 0.9] = 0
        if i == 7:
            s[:2000] = s[0]                    # one bucket per window holds 2000 points
        cols.append(s)
    dev_cols = [H.to_device(x) if x.shape[0] else H.empty_fr(1) for x in cols]
    out = H.msm_batch_table(table, nmax, c, dev_cols, ns)
    torch.cuda.synchronize()
    got = H.to_host(out)
    for i, (n, s) in enumerate(zip(ns, cols)):
        exp = O.msm_known_dlog(d[:n], s) if n else np.zeros((1, 8), np.uint64)
        assert (_jac_to_aff(O, got[i]) == exp).all(), i


def test_msm_batch_table_many(O, gpu):
    # 300 MSMs share the reduction-thread budget (a few threads per bucket set)
    H = gpu.host
    nmax = 2048
    d = O.rand_fr(nmax, 193)
    bases = H.to_device(O.g1_gen_bases(d))
    c = 15
    table, _ = H.msm_table_build(bases, nmax, c)
    rng = np.random.default_rng(194)
    ns = [int(x) for x in rng.integers(1, nmax + 1, 300)]
    cols = [O.rand_fr(n, 400 + i) for i, n in enumerate(ns)]
    out = H.msm_batch_table(table, nmax, c, [H.to_device(x) for x in cols], ns)
    plain = H.msm_batch(bases, [H.to_device(x) for x in cols], ns, [c] * len(ns))
    torch.cuda.synchronize()
    got, ref = H.to_host(out), H.to_host(plain)
    for i in (0, 1, 150, 299):
        assert (_jac_to_aff(O, got[i]) == O.msm_known_dlog(d[:ns[i]], cols[i])).all(), i
    assert (_jac_to_aff(O, got) == _jac_to_aff(O, ref)).all()
