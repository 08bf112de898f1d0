"""The proof hot path (zkwasm-prover_b200/prover.py) on small circuits of the
benchmark's two shapes: the plain schedule (reference-compatible symbols, one
kernel per column), the batched schedule (phase pipelines, per-coset fused
quotient) and the plain schedule through the reference's own kernels (with the
CPU steps through the oracle, as the reference's host runs them) give the same
commitments and evaluations, bit for bit; the witness satisfies the circuit,
so the quotient's coefficients past its degree bound are zero; commitments
match the known-discrete-log identity of the SRS."""
import importlib
import os

import numpy as np
import pytest
import torch

import ref_cases as RC

pytestmark = pytest.mark.gpu


def _shapes(P, k=10):
    return {
        "gwc_deg4": P.Shape(k=k, advice=16, fixed=6, lookups=3, shuffles=1, perm=10, degree=4, multiopen="gwc"),
        "shplonk_deg9": P.Shape(k=k, advice=16, fixed=6, lookups=3, shuffles=1, perm=10, degree=9,
                                multiopen="shplonk"),
    }


@pytest.fixture(scope="module")
def P(gpu):
    return importlib.import_module("zkwasm-prover_b200.prover")


def _run(P, shape, schedule, symbols=None, host_work=None, seed=3, **kw):
    c = P.Circuit(shape, seed=seed)
    hp = P.HotPath(c, schedule, symbols=symbols, host_work=host_work, **kw)
    return hp, hp.prove()


# the batched schedule with (w, w') pair tables and every proving-key coset
# cached, with Montgomery tables and nothing cached, and with the cache holding
# only part of the cosets (the rest transformed per proof)
BATCHED = {"pairs_cached": {"pair_tables": True}, "montgomery_uncached": {"pair_tables": False, "pk_cache_gib": 0},
           "partly_cached": {"pk_cache_gib": 0.0003}, "tables_only": {"learned": False}}


@pytest.mark.parametrize("variant", sorted(BATCHED))
@pytest.mark.parametrize("name", ["gwc_deg4", "shplonk_deg9"])
def test_plain_and_batched_agree(P, name, variant):
    shape = _shapes(P)[name]
    hp_p, proof_p = _run(P, shape, "plain")
    hp_b, proof_b = _run(P, shape, "batched", **BATCHED[variant])
    if variant == "partly_cached":
        assert 0 < len(hp_b.pk_cos) < 3 * hp_b.E
    assert proof_p["challenges"] == proof_b["challenges"]
    for (na, a), (nb, b) in zip(proof_p["commitments"], proof_b["commitments"]):
        assert na == nb and a == b, na
    assert proof_p["evals"] == proof_b["evals"]
    assert torch.equal(hp_p.h_coeff, hp_b.h_coeff)


@pytest.mark.parametrize("schedule", ["plain", "batched"])
@pytest.mark.parametrize("name", ["gwc_deg4", "shplonk_deg9"])
def test_quotient_vanishes_past_degree_bound(P, name, schedule):
    """With a witness that satisfies every constraint, h = C / Z_H has degree
    at most degree (n - 1) - n; any wrong value anywhere makes the top
    coefficients nonzero."""
    shape = _shapes(P)[name]
    hp, _ = _run(P, shape, schedule)
    n = shape.n
    bound = shape.degree * (n - 1) - n
    top = hp.h_coeff[bound + 1:]
    assert top.shape[0] > 0
    assert not top.any(), f"{int((top != 0).any(dim=1).sum())} coefficients past {bound} are nonzero"
    # and a deliberately broken witness (one gate output changed) does not vanish
    c = P.Circuit(shape, seed=3)
    g = c.gate_cols[0]
    row = int(torch.nonzero(c.fixed[c.selector_cols[0], :c.u, 0]).flatten()[0])
    c.advice[g[4], row] = P.fr_tensor([12345])[0]
    hp2 = P.HotPath(c, schedule)
    hp2.prove()
    assert hp2.h_coeff[bound + 1:].any()


@pytest.mark.parametrize("name", ["gwc_deg4", "shplonk_deg9"])
def test_plain_through_reference_kernels(P, name):
    if not os.path.exists(RC.REF_LIB):
        pytest.skip("reference kernels not built (make -C oracle ref)")
    from host_work import OracleHostWork

    # k = 15: the reference's logup kernels need n >= 32768 (cuda/bn254.cu:1914-1934)
    shape = _shapes(P, k=15)[name]
    _, proof_b = _run(P, shape, "batched")
    _, proof_r = _run(P, shape, "plain", symbols=RC.load_ref(), host_work=OracleHostWork())
    for (na, a), (nb, b) in zip(proof_b["commitments"], proof_r["commitments"]):
        assert na == nb and a == b, na
    assert proof_b["evals"] == proof_r["evals"]


def test_commitments_match_known_dlogs(O, P):
    """An advice commitment over the Lagrange SRS equals [sum_i a_i k_i] G."""
    shape = _shapes(P)["gwc_deg4"]
    c = P.Circuit(shape, seed=5)
    hp = P.HotPath(c, "batched")
    proof = hp.prove()
    adv = dict(proof["commitments"])["advice"]
    kl = hp.srs_k[1].cpu().numpy().view(np.uint64)
    dl = O.fr_vec([int(x) for x in kl])
    for i in (0, shape.advice - 1):
        a = c.advice[i].cpu().numpy().view(np.uint64)
        exp = O.msm_known_dlog(dl, a)
        ex = [O.fq_ints(exp[:, :4])[0], O.fq_ints(exp[:, 4:])[0]]
        assert tuple(ex) == adv[i]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_schedule_same_proof(P, world):
    """The batched schedule sharded over `world` ranks (commitments by column
    ranges, quotient cosets round robin) gives the unsharded proof.  The ranks
    are threads on one GPU exchanging through the host (shard.ThreadGroup):
    their kernels never wait on one another."""
    import threading

    S = importlib.import_module("zkwasm-prover_b200.shard")
    shape = _shapes(P)["shplonk_deg9"]
    _, ref = _run(P, shape, "batched")
    g = S.ThreadGroup(world)
    proofs, errors = [None] * world, []

    def rank(r):
        try:
            c = P.Circuit(shape, seed=3)
            hp = P.HotPath(c, "batched", group=g.view(r))
            proofs[r] = hp.prove()
        except BaseException as e:  # noqa: BLE001
            errors.append(e)
            g.barrier.abort()

    ts = [threading.Thread(target=rank, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    assert not errors, errors
    for p in proofs:
        assert p["commitments"] == ref["commitments"] and p["evals"] == ref["evals"]


def test_witness_staged_from_host(P):
    """The advice columns copied in from pinned host memory group by group,
    overlapped with phase 1, give the same proof as resident columns."""
    shape = _shapes(P)["shplonk_deg9"]
    hp, ref = _run(P, shape, "batched")
    host = torch.empty(hp.c.advice.shape, dtype=torch.int64, pin_memory=True)
    host.copy_(hp.c.advice)
    hp.c.advice.zero_()
    stage = P.HostStage(host, hp.c.advice, group=3)
    for _ in range(2):
        proof = hp.prove(stage=stage)
        assert proof["commitments"] == ref["commitments"] and proof["evals"] == ref["evals"]


@pytest.mark.parametrize("name", ["gwc_deg4", "shplonk_deg9"])
def test_fused_coset_equals_separate_kernels(P, name):
    """The fused constraint pass of one coset equals the reference symbols run
    one constraint family at a time on the same coset rows."""
    hp, _ = _run(P, _shapes(P)[name], "batched")
    r = hp.coset_fused_vs_separate(reps=1)
    assert r["equal"], r
