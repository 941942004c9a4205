"""Batched joins: many uneven joins in one pipeline (one persistent probe kernel over all joins'
tasks) give exactly the per-join oracle results."""
import numpy as np
import pytest

from gpu_helpers import assert_same_pairs, dev, run_device

pytestmark = pytest.mark.gpu


def _batch(bj, torch, cases, **cfg):
    items, keep = [], []
    for rk, rv, sk, sv, cap in cases:
        d = [dev(torch, a) for a in (rk, rv, sk, sv)]
        o_r = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        o_s = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        keep.append((d, o_r, o_s))
        items.append(dict(r_key=d[0], r_val=d[1], n_r=len(rk), s_key=d[2], s_val=d[3], n_s=len(sk),
                          out_r=o_r, out_s=o_s, capacity=cap))
    with bj.Join(**cfg) as j:
        j.run_batch(items)
        counts = j.batch_counts(len(items))
    outs = []
    for (d, o_r, o_s), c, (_, _, _, _, cap) in zip(keep, counts, cases):
        n = min(int(c), cap)
        outs.append((int(c), o_r[:n].cpu().numpy().view(np.uint32), o_s[:n].cpu().numpy().view(np.uint32)))
    return outs


@pytest.mark.parametrize("bloom", [0, 1])
@pytest.mark.parametrize("graph", [0, 1])
def test_uneven_batch_matches_oracle(bj, oracle, torch_cuda, bloom, graph):
    rng = np.random.default_rng(10 + bloom)
    cases, exps = [], []
    for i in range(24):
        nr = int(rng.integers(0, 60_000)) if i % 7 else int(rng.integers(0, 50))
        ns = int(rng.integers(0, 4 * max(nr, 1) + 10))
        if i % 5 == 3:   # duplicate-heavy join
            rk = rng.integers(0, 64, nr, dtype=np.uint32)
            sk = rng.integers(0, 128, ns, dtype=np.uint32)
            rv = np.arange(nr, dtype=np.uint32)
            sv = np.arange(ns, dtype=np.uint32)
        else:
            rk, rv, sk, sv = bj.gen_host(100 + i, nr, ns, float(rng.uniform(0, 1)), zipf_s=1.0 if i % 2 else 0.0)
        e = oracle.pairs(rk, rv, sk, sv)
        exps.append(e)
        cases.append((rk, rv, sk, sv, len(e[0])))
    outs = _batch(bj, torch_cuda, cases, use_bloom=bloom, use_cuda_graph=graph, table_capacity=1024)
    for (c, r, s), (er, es) in zip(outs, exps):
        assert c == len(er)
        assert_same_pairs(oracle, r, s, er, es)


def test_batch_equals_single_joins(bj, oracle, torch_cuda):
    cases = []
    for i in range(5):
        rk, rv, sk, sv = bj.gen_host(500 + i, 40_000 * (i + 1), 90_000, 0.2)
        cases.append((rk, rv, sk, sv, 90_000))
    outs = _batch(bj, torch_cuda, cases, use_bloom=1)
    for (c, r, s), (rk, rv, sk, sv, cap) in zip(outs, cases):
        st, r1, s1, _ = run_device(bj, torch_cuda, rk, rv, sk, sv, cap=cap, use_bloom=1)
        assert st.count == c
        assert_same_pairs(oracle, r, s, r1, s1)


def test_batch_graph_replay_new_inputs(bj, oracle, torch_cuda):
    """The captured pipeline replays for a second batch of the same shape with different data."""
    shape = [(30_000, 70_000), (1000, 5000), (80_000, 80_000)]
    with bj.Join(use_bloom=1, use_cuda_graph=1) as j:
        for seed in (1, 2):
            items, keep, exps = [], [], []
            for i, (nr, ns) in enumerate(shape):
                rk, rv, sk, sv = bj.gen_host(seed * 10 + i, nr, ns, 0.3)
                exps.append(oracle.pairs(rk, rv, sk, sv))
                d = [dev(torch_cuda, a) for a in (rk, rv, sk, sv)]
                o_r = torch_cuda.empty(ns, dtype=torch_cuda.int32, device="cuda")
                o_s = torch_cuda.empty(ns, dtype=torch_cuda.int32, device="cuda")
                keep.append((d, o_r, o_s))
                items.append(dict(r_key=d[0], r_val=d[1], n_r=nr, s_key=d[2], s_val=d[3], n_s=ns,
                                  out_r=o_r, out_s=o_s, capacity=ns))
            j.run_batch(items)
            counts = j.batch_counts(len(items))
            for (d, o_r, o_s), c, (er, es) in zip(keep, counts, exps):
                assert c == len(er)
                assert_same_pairs(oracle, o_r[:c].cpu().numpy().view(np.uint32),
                                  o_s[:c].cpu().numpy().view(np.uint32), er, es)


def _skewed_cases(bj, oracle, n, seed):
    rng = np.random.default_rng(seed)
    cases, exps = [], []
    for i in range(n):
        nr = int(rng.integers(1000, 120_000))
        ns = 4 * nr
        rk, rv, sk, sv = bj.gen_host(seed * 100 + i, nr, ns, 0.1, zipf_s=1.0 if i % 2 else 0.0)
        e = oracle.pairs(rk, rv, sk, sv)
        exps.append(e)
        cases.append((rk, rv, sk, sv, len(e[0])))
    return cases, exps


def test_every_autotune_candidate_gives_the_oracle_pairs(bj, oracle, torch_cuda):
    """Each configuration the autotuner may pick (Bloom choice, table capacity, level-1 bits,
    partition fill, slices per SM) joins an uneven, partly Zipf-skewed batch to exactly the oracle's
    pairs: tuning changes the speed only."""
    cases, exps = _skewed_cases(bj, oracle, 6, 3)
    cands = bj.autotune_candidates(use_cuda_graph=1)
    assert len(cands) == 17
    for c in cands:
        outs = _batch(bj, torch_cuda, cases, **bj.config_dict(c))
        for (cnt, r, s), (er, es) in zip(outs, exps):
            assert cnt == len(er)
            assert_same_pairs(oracle, r, s, er, es)


def test_autotune_keeps_a_candidate_and_the_batch_stays_exact(bj, oracle, torch_cuda):
    cases, exps = _skewed_cases(bj, oracle, 8, 4)
    items, keep = [], []
    for rk, rv, sk, sv, cap in cases:
        d = [dev(torch_cuda, a) for a in (rk, rv, sk, sv)]
        o_r = torch_cuda.empty(max(cap, 1), dtype=torch_cuda.int32, device="cuda")
        o_s = torch_cuda.empty(max(cap, 1), dtype=torch_cuda.int32, device="cuda")
        keep.append((o_r, o_s))
        items.append(dict(r_key=d[0], r_val=d[1], n_r=len(rk), s_key=d[2], s_val=d[3], n_s=len(sk),
                          out_r=o_r, out_s=o_s, capacity=cap))
        keep.append(d)
    with bj.Join(use_cuda_graph=1) as j:
        chosen = j.autotune(items)
        # the handle's own defaults (0: automatic) stay when no candidate beats them
        assert chosen["table_capacity"] in (0, 1024, 2048, 4096) and chosen["slices_per_sm"] in (0, 8, 16, 32)
        j.run_batch(items)
        counts = j.batch_counts(len(items))
    for (o_r, o_s), c, (er, es) in zip(keep[0::2], counts, exps):
        assert c == len(er)
        assert_same_pairs(oracle, o_r[:c].cpu().numpy().view(np.uint32), o_s[:c].cpu().numpy().view(np.uint32), er, es)
