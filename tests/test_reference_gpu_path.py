"""The reference's own GPU path as a second oracle. oracle/_ref/ref_gpu_harness runs the reference's
partition, Bloom and probe kernels (src/kernel_functions.cu, src/vlsplit_hash_kernel.cu,
src/bloom.cu, compiled for sm_100a from the reference tree by `make -C oracle ref`) in gpu_main's
one-PE order for use_bf = 0 and use_bf = 10, and writes the pairs they produce. On the same inputs
the engine's pair multiset (through the C ABI) must equal the reference GPU path's, and both must
equal the CPU oracle's.

Values are the reference's synthesised payloads, row + 1 for R and row + 100000001 for S
(hash_kernel.cu:333-335), on both sides."""
import json
import os
import subprocess

import numpy as np
import pytest

from gpu_helpers import assert_same_pairs, run_device

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_harness")

needs_harness = pytest.mark.skipif(
    not os.path.exists(HARNESS),
    reason="oracle/_ref/ref_gpu_harness is not built (make -C oracle ref REF=<BRIG-Join tree>)")


def ref_vals(n_r, n_s):
    return ((np.arange(n_r) + 1).astype(np.uint32), (np.arange(n_s) + 100000001).astype(np.uint32))


def run_reference(tmp_path, rk, sk, p1, p2, bloom=None):
    """Runs the reference's GPU path; returns (count, overflow sub-buckets, survivors, r_vals, s_vals)."""
    rf, sf, pf = (str(tmp_path / n) for n in ("R.bin", "S.bin", "pairs.bin"))
    rk.astype(np.uint32).tofile(rf)
    sk.astype(np.uint32).tofile(sf)
    args = [HARNESS, "bf10" if bloom else "bf0", rf, sf, str(len(rk)), str(len(sk)), str(p1), str(p2), pf]
    if bloom:
        args += [str(bloom[0]), str(bloom[1])]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = dict(l.split() for l in r.stdout.splitlines() if len(l.split()) == 2)
    count = int(out["COUNT"])
    raw = np.fromfile(pf, dtype=np.uint32)
    assert len(raw) == 2 * count
    return count, int(out["OVERFLOW"]), int(out.get("SURVIVORS", len(sk))), raw[:count], raw[count:]


def engine_pairs(bj, torch, rk, rv, sk, sv, p1, p2, bloom):
    cfg = dict(partition_mode=bj.PART_MODULO, partition_size=p1, second_partition_size=p2)
    if bloom:
        cfg.update(use_bloom=1, bloom_bits_per_key=bloom[0] / len(rk), bloom_num_hashes=bloom[1])
    st, r, s, _ = run_device(bj, torch, rk, rv, sk, sv, cap=len(sk) + 16, **cfg)
    return st, r, s


@needs_harness
@pytest.mark.parametrize("case", [c for c in MANIFEST if c["R"] > 1], ids=lambda c: c["name"])
@pytest.mark.parametrize("p1,p2", [(16, 5), (512, 67)])
@pytest.mark.parametrize("use_bf", [0, 10])
def test_golden_cases_match_the_reference_gpu_path(bj, oracle, torch_cuda, tmp_path, case, p1, p2, use_bf):
    rk = np.fromfile(os.path.join(GOLDEN, case["r_file"]), dtype=np.uint32)
    sk = np.fromfile(os.path.join(GOLDEN, case["s_file"]), dtype=np.uint32)
    rv, sv = ref_vals(len(rk), len(sk))
    bloom = (10 * len(rk), 7) if use_bf == 10 else None
    count, _, surv, ref_r, ref_s = run_reference(tmp_path, rk, sk, p1, p2, bloom)
    assert count == case["k"] and count <= surv <= len(sk)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    assert_same_pairs(oracle, ref_r, ref_s, exp_r, exp_s)
    st, got_r, got_s = engine_pairs(bj, torch_cuda, rk, rv, sk, sv, p1, p2, bloom)
    assert st.count == count
    assert_same_pairs(oracle, got_r, got_s, ref_r, ref_s)


@needs_harness
@pytest.mark.parametrize("use_bf", [0, 10])
def test_config0_16M_x_16M_matches_the_reference_gpu_path(bj, oracle, torch_cuda, tmp_path, use_bf):
    """|R| = |S| = 2^24, 10% of S matching, the reference's README fan-out 512 (key % 512) with the
    second level its sizing rule gives at this size (67); use_bf = 10 with 10 bits per key, k = 7."""
    n = 1 << 24
    rk, _, sk, _ = oracle.gen(42, n, n, 0.1, want_vals=False)
    rv, sv = ref_vals(n, n)
    bloom = (10 * n, 7) if use_bf == 10 else None
    count, overflow, surv, ref_r, ref_s = run_reference(tmp_path, rk, sk, 512, 67, bloom)
    assert count == 1_677_721 and overflow == 0
    if use_bf:
        assert count <= surv < n // 4
    st, got_r, got_s = engine_pairs(bj, torch_cuda, rk, rv, sk, sv, 512, 67, bloom)
    assert st.count == count
    assert_same_pairs(oracle, got_r, got_s, ref_r, ref_s)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    assert_same_pairs(oracle, ref_r, ref_s, exp_r, exp_s)


@needs_harness
def test_oversized_sub_buckets_take_the_reference_nested_loop_path(bj, oracle, torch_cuda, tmp_path):
    """Sub-buckets of about 13,000 R keys, above the reference's 10,007-slot shared table: the reference
    probes every one by its nested-loop path (kernel_functions.cu:341-370) and the engine by its
    split path; the pairs are the same (R keys are distinct, so the nested loop's first-match stop
    loses nothing)."""
    n_r, n_s = 1 << 19, 1 << 17
    rk, _, sk, _ = oracle.gen(9, n_r, n_s, 0.5, want_vals=False)
    rv, sv = ref_vals(n_r, n_s)
    count, overflow, _, ref_r, ref_s = run_reference(tmp_path, rk, sk, 8, 5)
    assert overflow == 40 and count == n_s // 2
    st, got_r, got_s = engine_pairs(bj, torch_cuda, rk, rv, sk, sv, 8, 5, None)
    assert st.count == count
    assert_same_pairs(oracle, got_r, got_s, ref_r, ref_s)
