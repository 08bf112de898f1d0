"""Writes tests/golden/reference_kernels.json from the reference's own CUDA
kernels (cuda/bn254.cu + cuda/msm.cu rebuilt for sm_100a by `make -C oracle
ref` into oracle/_ref/).  Needs a GPU:

    python tests/golden/make_golden.py [OUT_DIR]

writes OUT_DIR/reference_kernels.json (default: this directory, where the
committed copy lives; on a machine whose results must be carried back, give a
directory that is copied back and copy the file here).

Inputs come from the oracle's seeded generators.  Each reference entry point
is called the way the reference's Rust host calls it:
  ntt / expand_omega_buffer   src/cuda/ntt.rs:15-93 (pq table of 128 entries)
  msm + batch_msm_collect     src/cuda/msm.rs:239-455 (batch of one)
  logup_sum_input_inv         src/lib.rs:643 (n >= 32768)
  eval_logup_z_compose        src/lib.rs:662
and every case of tests/ref_cases.py (the quotient, multi-open, coset and
lookup symbols) at n = 2^12 and 2^16, recorded as SHA-256 hashes of each
output under "kernels" (key "<case>@<n>").
"""
import ctypes
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402
import ref_cases as RC  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libzkwasm_prover_kernel_ref.so")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint64)


def p(t):
    return ctypes.c_void_p(t.data_ptr())


def ref_ntt(L, a, log_n, inverse):
    n = 1 << log_n
    w = O.omega(log_n)
    if inverse:
        w = pow(w, -1, O.R_MOD)
    max_deg = min(8, log_n)
    tw = pow(w, n >> max_deg, O.R_MOD)
    pq = O.fr_vec([pow(tw, i, O.R_MOD) for i in range((1 << max_deg) >> 1)])
    om = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
    om[:2] = dev(O.fr_vec([1, w]))
    torch.cuda.synchronize()
    assert L.expand_omega_buffer(p(om), log_n, 1) == 0
    buf, tmp = dev(a), torch.empty((n, 4), dtype=torch.int64, device="cuda")
    ninv = dev(O.fr(pow(n, -1, O.R_MOD)))
    swap = ctypes.c_bool(False)
    pqd = dev(pq)  # device buffers stay referenced until the kernels finish
    assert L.ntt(p(buf), p(tmp), p(pqd), p(om), p(ninv) if inverse else None, log_n, 8,
                 ctypes.byref(swap), None) == 0
    torch.cuda.synchronize()
    return host(tmp if swap.value else buf)


def ref_msm(L, bases, scalars):
    n = scalars.shape[0]
    threads, bits = 64, 254
    c = 0 + 10 + max((n - 1).bit_length(), 22) - 22
    windows = (bits + c - 1) // c
    bucket = windows << c
    worker = (n + threads - 1) // threads * threads if n < 128 * 512 else 128 * 512
    region = bucket + 2 * worker
    curve = torch.empty((region, 12), dtype=torch.int64, device="cuda")
    single = n * windows
    idx = [torch.empty(single, dtype=torch.int32, device="cuda") for _ in range(4)]
    sort = torch.empty(3 * single, dtype=torch.int32, device="cuda")
    acc = torch.empty(2 * worker, dtype=torch.int32, device="cuda")
    P = dev(bases)
    S = dev(scalars)
    err = L.msm(p(curve), p(P), p(S), p(idx[0]), p(idx[1]), p(idx[2]), p(idx[3]), p(sort), p(acc), n, windows, c,
                threads, worker, 3 * single * 4, 1, None)
    assert err == 0, err
    torch.cuda.synchronize()
    base = curve.data_ptr()
    ptrs = lambda xs: torch.tensor(xs, dtype=torch.int64, device="cuda")
    ri = ptrs([acc.data_ptr()])
    nri = ptrs([acc.data_ptr() + worker * 4])
    ra = ptrs([base + bucket * 96])
    nra = ptrs([base + (bucket + worker) * 96])
    bk = ptrs([base])
    err = L.batch_msm_collect(p(ri), p(ra), p(nri), p(nra), p(bk), worker, windows, c, 1, None)
    assert err == 0, err
    torch.cuda.synchronize()
    return host(curve[0:1])


def main(out):
    os.makedirs(out, exist_ok=True)
    L = ctypes.CDLL(REF)
    g = {}
    for k in (10, 13):
        a = O.rand_fr(1 << k, 7000 + k)
        g[f"ntt_in_{k}"] = a
        g[f"ntt_out_{k}"] = ref_ntt(L, a, k, False)
        g[f"intt_out_{k}"] = ref_ntt(L, a, k, True)
    for tag, n in (("msm_small", 100), ("msm_2_14", 1 << 14)):
        d = O.rand_fr(n, 8000 + n)
        s = O.rand_fr(n, 9000 + n)
        g[f"{tag}_dlogs"] = d
        g[f"{tag}_scalars"] = s
        g[f"{tag}_out"] = ref_msm(L, O.g1_gen_bases(d), s)
    n = 1 << 16
    inp = O.rand_fr(n, 10001)
    beta = O.rand_fr(1, 10002)
    s = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
    tmp = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    inp_d, beta_d = dev(inp), dev(beta)
    assert L.logup_sum_input_inv(p(s), p(inp_d), p(tmp), p(beta_d), 0, n, None) == 0
    torch.cuda.synchronize()
    g["logup_in"], g["logup_beta"], g["logup_sum"] = inp, beta, host(s)
    # eval_logup_z_compose on the sum above with a table and multiplicities
    table = O.rand_fr(n, 10003)
    m = O.fr_vec([i % 5 for i in range(n)])
    z = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    last = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
    s2, table_d, m_d = s.clone(), dev(table), dev(m)
    assert L.eval_logup_z_compose(p(z), p(s2), p(table_d), p(m_d), p(beta_d), p(last), n - 17, n, None) == 0
    torch.cuda.synchronize()
    g["logup_table"], g["logup_m"], g["logup_z"], g["logup_last_z"] = table, m, host(z), host(last)
    kernels = {}
    LR = RC.load_ref()
    for n in (1 << 12, 1 << 16):
        for case in RC.cases_for(n):
            kernels[f"{case.name}@{n}"] = {k: sha(v) for k, v in case.run(LR, RC.Dev(), n).items()}
    path = os.path.join(out, "reference_kernels.json")
    write_json(g, kernels, path)
    print("wrote", path, len(kernels), "kernel cases")


def sha(a):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a, np.uint64).tobytes()).hexdigest()


def write_json(g, kernels, path):
    """Compact fixture: seeds of the inputs, hashes of large outputs, small
    outputs in full."""
    out = {"generator": "tests/golden/make_golden.py on a B200 (reference cuda/bn254.cu + cuda/msm.cu rebuilt "
                        "for sm_100a)",
           "inputs": "oracle.rand_fr(n, seed) (splitmix64, rejection below r, Montgomery form)",
           "ntt": [], "msm": [], "logup": {}}
    for k in (10, 13):
        out["ntt"].append({"log_n": k, "seed": 7000 + k, "forward_sha256": sha(g[f"ntt_out_{k}"]),
                           "inverse_sha256": sha(g[f"intt_out_{k}"])})
    for tag, n in (("msm_small", 100), ("msm_2_14", 1 << 14)):
        out["msm"].append({"n": n, "dlog_seed": 8000 + n, "scalar_seed": 9000 + n,
                           "jacobian_out": [int(x) for x in g[f"{tag}_out"].reshape(-1)]})
    n = 1 << 16
    out["logup"] = {"n": n, "input_seed": 10001, "beta_seed": 10002, "table_seed": 10003, "m": "i % 5",
                    "last_z_index": n - 17, "sum_sha256": sha(g["logup_sum"]), "z_sha256": sha(g["logup_z"]),
                    "last_z": [int(x) for x in g["logup_last_z"].reshape(-1)]}
    out["kernels"] = kernels
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
