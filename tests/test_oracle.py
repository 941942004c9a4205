"""The oracle is pinned before it is trusted: against the reference generator's known answers and
the reference's own CPU join (golden fixtures), against an independent sort-merge join, and against
a pure-Python join on small inputs."""
import json
import os
from collections import defaultdict

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))


def load_case(c):
    rk = np.fromfile(os.path.join(GOLDEN, c["r_file"]), dtype=np.uint32)
    sk = np.fromfile(os.path.join(GOLDEN, c["s_file"]), dtype=np.uint32)
    rv = (np.arange(len(rk), dtype=np.int64) + 1).astype(np.uint32)
    sv = (np.arange(len(sk), dtype=np.int64) + 100000001).astype(np.uint32)
    return rk, rv, sk, sv


def py_join(rk, rv, sk, sv):
    idx = defaultdict(list)
    for k, v in zip(rk.tolist(), rv.tolist()):
        idx[k].append(v)
    out = [(r, s) for k, s in zip(sk.tolist(), sv.tolist()) for r in idx.get(k, ())]
    return sorted(out)


@pytest.mark.parametrize("case", MANIFEST, ids=[c["name"] for c in MANIFEST])
def test_golden_known_answer(oracle, case):
    rk, rv, sk, sv = load_case(case)
    assert len(rk) == case["R"] and len(sk) == case["S"]
    assert oracle.count(rk, sk) == case["k"] == case["ref_sanity_count"]
    a, b = oracle.pairs(rk, rv, sk, sv)
    assert len(a) == case["k"]
    a, b = oracle.sort_pairs(a, b)
    assert f"{oracle.digest(a, b):016x}" == case["pairs_digest"]
    c, d = oracle.sort_pairs(*oracle.sortmerge_pairs(rk, rv, sk, sv))
    assert np.array_equal(a, c) and np.array_equal(b, d)


@pytest.mark.parametrize("case", MANIFEST, ids=[c["name"] for c in MANIFEST])
def test_golden_against_live_reference(oracle, case):
    if not oracle.ref_available():
        pytest.skip("reference CPU join not built here (oracle/_ref)")
    rk, _, sk, _ = load_case(case)
    assert oracle.ref_count(rk, sk)[0] == case["k"]


@pytest.mark.parametrize("seed", range(6))
def test_random_with_duplicates_vs_python(oracle, seed):
    rng = np.random.default_rng(seed)
    nr, ns = rng.integers(0, 3000), rng.integers(0, 3000)
    hi = int(rng.integers(1, 4000))
    rk = rng.integers(0, hi, nr, dtype=np.uint32)
    sk = rng.integers(0, hi, ns, dtype=np.uint32)
    rv = rng.integers(0, 2**32, nr, dtype=np.uint64).astype(np.uint32)
    sv = rng.integers(0, 2**32, ns, dtype=np.uint64).astype(np.uint32)
    exp = py_join(rk, rv, sk, sv)
    a, b = oracle.pairs(rk, rv, sk, sv)
    assert oracle.count(rk, sk) == len(exp) == len(a)
    a, b = oracle.sort_pairs(a, b)
    assert list(zip(a.tolist(), b.tolist())) == exp
    c, d = oracle.sort_pairs(*oracle.sortmerge_pairs(rk, rv, sk, sv))
    assert np.array_equal(a, c) and np.array_equal(b, d)


def test_full_key_domain(oracle):
    edge = np.array([0, 1, 0x7FFFFFFF, 0x80000000, 0x80000001, 0xFFFFFFFE, 0xFFFFFFFF], np.uint32)
    rk = np.concatenate([edge, edge[:3]])
    sk = np.concatenate([edge, edge])
    rv = np.arange(len(rk), dtype=np.uint32)
    sv = np.arange(len(sk), dtype=np.uint32)
    exp = py_join(rk, rv, sk, sv)
    a, b = oracle.sort_pairs(*oracle.pairs(rk, rv, sk, sv))
    assert list(zip(a.tolist(), b.tolist())) == exp
    assert oracle.count(rk, sk) == len(exp) == 2 * (7 + 3)


def test_reference_drops_int_min_keys(oracle):
    """Documents the deliberate difference: the reference's table uses INT_MIN as EMPTY, so an R key
    0x80000000 never matches there, while the oracle (and the engine) match it."""
    if not oracle.ref_available():
        pytest.skip("reference CPU join not built here (oracle/_ref)")
    rk = np.array([5, 0x80000000, 9], np.uint32)
    sk = np.array([0x80000000, 5, 9, 9], np.uint32)
    assert oracle.count(rk, sk) == 4
    assert oracle.ref_count(rk, sk)[0] == 3


@pytest.mark.parametrize("seed", [1, 2])
def test_reference_agrees_on_duplicates(oracle, seed):
    """The reference's CPU join counts duplicates on both sides (src/sanity_check.cpp:36-41,55-60)."""
    if not oracle.ref_available():
        pytest.skip("reference CPU join not built here (oracle/_ref)")
    rng = np.random.default_rng(seed)
    rk = rng.integers(0, 500, 20000, dtype=np.uint32)
    sk = rng.integers(0, 900, 30000, dtype=np.uint32)
    assert oracle.ref_count(rk, sk)[0] == oracle.count(rk, sk)


def test_generator_known_answer(bj, oracle):
    for frac in (0.0, 0.001, 0.1, 0.5, 1.0):
        rk, rv, sk, sv = bj.gen_host(77, 50_000, 80_000, frac)
        assert oracle.count(rk, sk) == int(np.floor(frac * 80_000))


@pytest.mark.parametrize("seed,nr,ns,frac", [(42, 1000, 1000, 0.1), (7, 123457, 98765, 0.3), (3, 1, 1, 1.0),
                                             (9, 0, 10, 0.5), (5, 10, 0, 0.1), (11, 1 << 20, 1 << 21, 0.001)])
def test_oracle_generator_matches_engine_generator(bj, oracle, seed, nr, ns, frac):
    """The benchmark's CPU baseline and reference arm generate their inputs with the oracle's C
    restatement of the generator (so they load no engine library); it must equal the engine's own
    host generator row for row."""
    a = bj.gen_host(seed, nr, ns, frac)
    b = oracle.gen(seed, nr, ns, frac)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
