"""C-ABI checks that need no GPU: the library loads and exports every declared function, the
planner's fan-outs, argument validation, error reporting without a device, and the host generator."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest


def test_exports_every_declared_symbol(bj):
    names = bj.header_functions()
    assert len(names) >= 15
    lib = bj.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", bj.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert set(names) <= exported


def test_config_defaults(bj):
    cfg = bj.make_config()
    assert cfg.abi_version == bj.ABI_VERSION
    assert cfg.partition_mode == bj.PART_HASH
    assert cfg.bloom_bits_per_key == 10.0 and cfg.use_bloom == 0 and cfg.device == -1
    assert cfg.s_chunks == 0  # S in one piece
    assert cfg.wait_poll_limit == 0  # default bound of the kernels' waits
    assert cfg.partition_fill == 0 and cfg.slices_per_sm == 0
    # layout of brig_join_config: s_chunks, wait_poll_limit, partition_fill and slices_per_sm took
    # what were reserved slots, so the size is unchanged
    assert C.sizeof(bj.Config) == 88
    assert bj.Config.s_chunks.offset == 72 and bj.Config.wait_poll_limit.offset == 76
    assert bj.Config.partition_fill.offset == 80 and bj.Config.slices_per_sm.offset == 84


@pytest.mark.parametrize("n_r,n_s,kw,expect", [
    (1 << 24, 1 << 24, {}, (512, 16)),
    (640_000_000, 640_000_000, {"use_bloom": 1}, (512, 512)),
    (1 << 26, 1 << 30, {"use_bloom": 1}, (512, 64)),
    (1 << 24, 1 << 24, {"partition_mode": 1, "partition_size": 512}, (512, 67)),
    (640_000_000, 640_000_000, {"partition_mode": 1, "partition_size": 512}, (512, 407)),
    (4096, 16384, {}, (2, 1)),
    (3000, 16384, {}, (1, 1)),
    (0, 0, {}, (1, 1)),
])
def test_planner_fanouts(bj, n_r, n_s, kw, expect):
    p1, p2, ws = bj.plan(n_r, n_s, **kw)
    assert (p1, p2) == expect
    assert ws >= 8 * (n_r + n_s)


def test_planner_rejects_bad_configs(bj):
    with pytest.raises(bj.BrigError) as e:
        bj.plan(1000, 1000, partition_size=3)
    assert e.value.status == bj.BRIG_E_INVALID
    with pytest.raises(bj.BrigError) as e:
        bj.plan(1000, 1000, partition_mode=1, partition_size=5000)
    assert e.value.status == bj.BRIG_E_INVALID
    with pytest.raises(bj.BrigError) as e:
        bj.plan(1 << 33, 1000, partition_mode=1, partition_size=2)
    assert e.value.status == bj.BRIG_E_UNSUPPORTED
    with pytest.raises(bj.BrigError) as e:
        bj.plan(-1, 10)
    assert e.value.status == bj.BRIG_E_INVALID
    with pytest.raises(bj.BrigError) as e:
        bj.plan(1000, 1000, s_chunks=-2)
    assert e.value.status == bj.BRIG_E_INVALID
    cfg = bj.make_config()
    cfg.abi_version = 99
    assert bj.lib().brig_join_plan(C.byref(cfg), 10, 10, None, None, None) == bj.BRIG_E_INVALID
    assert "ABI" in bj.last_error()


def test_create_reports_missing_device(bj):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    cfg = bj.make_config()
    st = bj.lib().brig_join_create(C.byref(cfg), C.byref(h))
    assert st == bj.BRIG_E_CUDA and not h.value
    assert bj.last_error()


def test_null_arguments_rejected(bj):
    assert bj.lib().brig_join_run(None, None, None, 0, None, None, 0, None, None) == bj.BRIG_E_INVALID
    assert bj.lib().brig_join_get_stats(None, None) == bj.BRIG_E_INVALID
    assert bj.lib().brig_join_destroy(None) == bj.BRIG_OK
    assert bj.lib().brig_join_stage_name(0) == b"r_hist"
    assert bj.lib().brig_join_stage_name(3) == b"r_l2_hist"
    assert bj.lib().brig_join_stage_name(12) == b"probe"
    assert bj.lib().brig_join_stage_name(13) is None


def test_generator_properties(bj):
    nr, ns, frac = 200_000, 300_000, 0.1
    rk, rv, sk, sv = bj.gen_host(5, nr, ns, frac)
    assert np.array_equal(rv, np.arange(nr)) and np.array_equal(sv, np.arange(ns))
    assert len(np.unique(rk)) == nr and rk.min() >= 1 and rk.max() < 2**31
    match = sk < 2**31
    assert match.sum() == int(frac * ns)
    assert np.isin(sk[match], rk).all()
    nm = sk[~match]
    assert nm.min() >= 2**31 and nm.max() < 2**32 - 1 and len(np.unique(nm)) == len(nm)
    again = bj.gen_host(5, nr, ns, frac)
    assert all(np.array_equal(a, b) for a, b in zip((rk, rv, sk, sv), again))
    other = bj.gen_host(6, nr, ns, frac)
    assert not np.array_equal(rk, other[0])


def test_generator_zipf_skew(bj):
    nr, ns = 100_000, 400_000
    rk, _, sk, _ = bj.gen_host(9, nr, ns, 0.1, zipf_s=1.0)
    m = sk[sk < 2**31]
    assert len(m) == 40_000
    pos = {k: i for i, k in enumerate(rk.tolist())}
    ranks = np.array([pos[k] for k in m.tolist()])
    # Zipf(1) over 100k ranks: rank 1 has probability 1/H(n) ~ 8%, the top 10 ranks ~ 24%
    assert 0.06 < (ranks == 0).mean() < 0.11
    assert 0.18 < (ranks < 10).mean() < 0.30


def test_generator_rejects_bad_arguments(bj):
    L = bj.lib()
    assert L.brig_gen_host(1, -5, 10, 0.1, 0.0, None, None, None, None) == bj.BRIG_E_INVALID
    assert L.brig_gen_host(1, 10, 10, 1.5, 0.0, None, None, None, None) == bj.BRIG_E_INVALID
    assert L.brig_gen_host(1, 1 << 31, 10, 0.1, 0.0, None, None, None, None) == bj.BRIG_E_UNSUPPORTED


def test_compat_symbols_exported(bj):
    """The reference-named C++ entry points of include/brig_join_compat.h are exported."""
    out = subprocess.run(["nm", "-DC", "--defined-only", bj.LIB_PATH], capture_output=True, text=True).stdout
    for name in ["gpu_main(", "split_tables(", "partial_jointable_gpu_partition(",
                 "partial_jointable_gpu_partition_rs_split(", "partial_jointable_gpu_partition_r_only(",
                 "partial_jointable_gpu_partition_s_only(", "partial_jointable_gpu_run_only_s(",
                 "brig_compat_set_answer_capacity("]:
        assert name in out, name
    for g in ["partition_size", "second_partition_size", "thread_no", "block_no", "chunk_size"]:
        assert any(line.split()[-1] == g for line in out.splitlines() if line.strip()), g


def test_autotune_candidates_vary_one_dimension_each(bj):
    """The autotuner's search space: every candidate differs from the base in one tuned field."""
    base = bj.make_config(use_bloom=1)
    cands = bj.autotune_candidates(use_bloom=1)
    assert len(cands) == 4 + 3 + 4 + 3 + 3
    tuned = {"use_bloom", "bloom_bits_per_key", "bloom_num_hashes", "bloom_num_bits", "bloom_probe_level",
             "table_capacity", "max_level1_bits", "partition_fill", "slices_per_sm"}
    for c in cands:
        for name, _ in bj.Config._fields_:
            if name not in tuned:
                assert getattr(c, name) == getattr(base, name), name
    assert {c.table_capacity for c in cands} >= {1024, 2048, 4096}
    assert {c.max_level1_bits for c in cands} >= {7, 8, 9, 10}
    assert {c.partition_fill for c in cands} >= {50, 75, 100}
    assert {c.slices_per_sm for c in cands} >= {8, 16, 32}
    assert {(c.use_bloom, c.bloom_num_hashes) for c in cands} >= {(0, 0), (1, 6), (1, 7)}


def test_planner_partition_fill_and_slices(bj):
    """partition_fill sets the level-2 fan-out through the per-partition target."""
    p_default = bj.plan(1 << 26, 1 << 26)  # 75%: 3072 of 4096 per finest partition -> 2^15 partitions
    p_full = bj.plan(1 << 26, 1 << 26, partition_fill=100)  # 4096 -> 2^14
    assert p_full[0] == p_default[0] and 2 * p_full[1] == p_default[1]
    with pytest.raises(bj.BrigError):
        bj.plan(1 << 20, 1 << 20, partition_fill=101)


def test_reference_file_formats_round_trip(bj, tmp_path):
    """brig_join_read_relation reads the reference's input layout (key block, then the value block
    with --read_val 1; synthesised row + base values without it) and brig_join_write_pairs writes the
    pairs in the same headerless int32 block layout; host code only, no GPU."""
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 2**32, 1000, dtype=np.uint64).astype(np.uint32)
    vals = rng.integers(0, 2**32, 1000, dtype=np.uint64).astype(np.uint32)
    f = str(tmp_path / "R.bin")
    np.concatenate([keys, vals]).tofile(f)
    k, v = bj.read_relation(f, 1000, read_val=True)
    assert np.array_equal(k, keys) and np.array_equal(v, vals)
    k, v = bj.read_relation(f, 1000, read_val=False, val_base=100000001)
    assert np.array_equal(k, keys) and np.array_equal(v, np.arange(1000, dtype=np.uint32) + 100000001)
    with pytest.raises(bj.BrigError):
        bj.read_relation(f, 1500, read_val=True)  # 3000 words asked of a 2000-word file
    out = str(tmp_path / "pairs.bin")
    bj.write_pairs(out, vals[:10], keys[:10], key=keys[5:15])
    assert np.array_equal(np.fromfile(out, np.uint32), np.concatenate([keys[5:15], vals[:10], keys[:10]]))
    bj.write_pairs(out, vals[:0], keys[:0])
    assert np.fromfile(out, np.uint32).size == 0


def test_golden_fixtures_read_as_the_reference_reads_them(bj):
    import json
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    for case in json.load(open(os.path.join(golden, "manifest.json"))):
        path = os.path.join(golden, case["r_file"])
        k, v = bj.read_relation(path, case["R"], read_val=False, val_base=1)
        assert np.array_equal(k, np.fromfile(path, np.uint32)[:case["R"]])
        assert v[0] == 1 and v[-1] == case["R"]
