"""Parity of the CUDA join path with the CPU oracle: exact match count and identical sorted
multiset of (r_val, s_val) pairs, on seeded inputs, through the C ABI."""
import numpy as np
import pytest

from gpu_helpers import assert_same_pairs, run_device

pytestmark = pytest.mark.gpu


def _parity(bj, oracle, torch, rk, rv, sk, sv, cap=None, **cfg):
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    st, r, s, _ = run_device(bj, torch, rk, rv, sk, sv, cap=cap if cap is not None else max(len(exp_r), 1), **cfg)
    assert st.count == len(exp_r)
    assert_same_pairs(oracle, r, s, exp_r, exp_s)
    return st


@pytest.mark.parametrize("bloom", [0, 1])
@pytest.mark.parametrize("n", [1000, 100_000, 1 << 20])
def test_uniform_hash(bj, oracle, torch_cuda, n, bloom):
    rk, rv, sk, sv = bj.gen_host(7 + n, n, n, 0.1)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=bloom)
    assert st.count == n // 10
    if bloom:
        assert st.count <= st.s_survivors < n


# Scatter forms. The engine picks, per scatter launch, the write pass (more than 1024 bins), the
# bulk-store form (1024-thread CTAs, 12288-tuple tiles) or its small form (two 512-thread CTAs per
# SM, 6144-tuple tiles) from the bin count and the mean slice length: small below 64K tuples per
# slice, or below 256K with at most 128 bins; S's level-2 survivors of a level-2 filter always small.
# Small joins take the small form everywhere; these cases reach the large form at 2^24 tuples with
# one level-1 slice per SM (slices of 113,664 tuples):
#   l1_large: 512 level-1 bins -> large level-1 scatters (level 2: 16 bins, short slices -> small);
#   l2_large: 16 x 512 -> small level-1 scatters, large level-2 scatters (slices of about 204K).
@pytest.mark.parametrize("case", [
    dict(partition_size=512),
    dict(partition_size=512, use_bloom=1, bloom_probe_level=1),
    dict(partition_mode=1, partition_size=500, second_partition_size=9),
    dict(partition_size=16, second_partition_size=512),
    dict(partition_size=16, second_partition_size=512, use_bloom=1, bloom_probe_level=2),
    dict(partition_mode=1, partition_size=16, second_partition_size=509),
], ids=["l1_large", "l1_large_bloom1", "l1_large_modulo", "l2_large", "l2_large_bloom2", "l2_large_modulo"])
def test_large_scatter_form_16M(bj, oracle, torch_cuda, case):
    n = 1 << 24
    rk, rv, sk, sv = bj.gen_host(5, n, n, 0.1)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, slices_per_sm=1, **case)
    assert st.count == n // 10
    assert st.partition_size == case["partition_size"]


@pytest.mark.parametrize("level", [1, 2])
@pytest.mark.parametrize("mode,p1,p2", [(0, 16, 16), (0, 64, 64), (1, 100, 7), (1, 512, 67), (0, 4, 64)])
def test_bloom_probe_levels(bj, oracle, torch_cuda, level, mode, p1, p2):
    """The filter probed in S's first partition pass or fused into its second pass (fan-out 4 gives
    level-1 partitions of 100K keys, whose filter segments span about 125 KB)."""
    rk, rv, sk, sv = bj.gen_host(31 + level, 400_000, 600_000, 0.05)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=1, bloom_probe_level=level,
                 partition_mode=mode, partition_size=p1, second_partition_size=p2)
    assert st.count == 30_000 and st.count <= st.s_survivors < 600_000 // 4


@pytest.mark.parametrize("bpk,k", [(8.0, 0), (14.0, 0), (10.0, 1), (10.0, 4), (16.0, 16)])
@pytest.mark.parametrize("level", [1, 2])
def test_bloom_pattern_tables_any_k(bj, oracle, torch_cuda, bpk, k, level):
    """The filter's masks come from pattern tables filled for the join's k (ceil(k/2) bits in one
    word of the pair, floor(k/2) in the other) for every k, not only k = 7: exact pairs, and the
    survivors stay a small superset of the matches."""
    rk, rv, sk, sv = bj.gen_host(61 + level, 400_000, 600_000, 0.05)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=1, bloom_bits_per_key=bpk,
                 bloom_num_hashes=k, bloom_probe_level=level, partition_size=16, second_partition_size=16)
    assert st.count == 30_000
    assert st.bloom_num_hashes == (k or round(bpk * 0.6931471805599453))
    assert st.count <= st.s_survivors < 600_000 // 4


@pytest.mark.parametrize("p1,p2", [(16, 16), (64, 8), (1, 1), (4096, 1), (2, 1024)])
def test_two_level_hash_fanouts(bj, oracle, torch_cuda, p1, p2):
    rk, rv, sk, sv = bj.gen_host(11, 300_000, 200_000, 0.3)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, partition_size=p1, second_partition_size=p2)
    assert (st.partition_size, st.second_partition_size) == (p1, p2)


@pytest.mark.parametrize("p1,p2", [(512, 0), (512, 67), (100, 3), (7, 1)])
@pytest.mark.parametrize("bloom", [0, 1])
def test_modulo_mode(bj, oracle, torch_cuda, p1, p2, bloom):
    rk, rv, sk, sv = bj.gen_host(13, 200_000, 250_000, 0.1)
    _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, partition_mode=bj.PART_MODULO, partition_size=p1,
            second_partition_size=p2, use_bloom=bloom)


@pytest.mark.parametrize("table", [256, 1024, 4096])
def test_duplicates_and_split_path(bj, oracle, torch_cuda, table):
    rng = np.random.default_rng(table)
    rk = rng.integers(0, 300, 20_000, dtype=np.uint32)     # heavy duplicates in R
    sk = rng.integers(0, 600, 5_000, dtype=np.uint32)
    rv = np.arange(len(rk), dtype=np.uint32)
    sv = np.arange(len(sk), dtype=np.uint32) + 7
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, table_capacity=table, partition_size=2,
                 second_partition_size=1)
    if table == 256:
        assert st.split_tasks > 0


def test_single_hot_key(bj, oracle, torch_cuda):
    rk = np.full(3000, 0xDEADBEEF, np.uint32)
    sk = np.concatenate([np.full(700, 0xDEADBEEF, np.uint32), np.arange(100, dtype=np.uint32)])
    rv = np.arange(len(rk), dtype=np.uint32)
    sv = np.arange(len(sk), dtype=np.uint32)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, table_capacity=256)
    assert st.count == 3000 * 700 and st.split_tasks > 0


@pytest.mark.parametrize("bloom", [0, 1])
def test_edge_keys_full_domain(bj, oracle, torch_cuda, bloom):
    edge = np.array([0, 1, 0x7FFFFFFF, 0x80000000, 0x80000001, 0xFFFFFFFE, 0xFFFFFFFF], np.uint32)
    rng = np.random.default_rng(5)
    rk = np.concatenate([edge, edge, rng.integers(0, 2**32, 5000, dtype=np.uint64).astype(np.uint32)])
    sk = np.concatenate([edge, rng.permutation(rk)[:3000], rng.integers(0, 2**32, 3000, dtype=np.uint64).astype(np.uint32)])
    rv = rng.integers(0, 2**32, len(rk), dtype=np.uint64).astype(np.uint32)
    sv = rng.integers(0, 2**32, len(sk), dtype=np.uint64).astype(np.uint32)
    _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=bloom)


@pytest.mark.parametrize("nr,ns", [(0, 100), (100, 0), (0, 0), (1, 1)])
def test_empty_and_tiny(bj, oracle, torch_cuda, nr, ns):
    rk = np.arange(nr, dtype=np.uint32)
    sk = np.arange(ns, dtype=np.uint32)
    st = _parity(bj, oracle, torch_cuda, rk, rk.copy(), sk, sk.copy(), use_bloom=1)
    assert st.count == min(nr, ns)


def test_ragged_unaligned_inputs(bj, oracle, torch_cuda):
    rk, rv, sk, sv = bj.gen_host(21, 99_999, 77_777, 0.5)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    st, r, s, _ = run_device(bj, torch_cuda, rk, rv, sk, sv, cap=len(exp_r), offset=1, use_bloom=1)
    assert st.count == len(exp_r)
    assert_same_pairs(oracle, r, s, exp_r, exp_s)


@pytest.mark.parametrize("offsets", [(1, 3, 2, 0), (3, 1, 0, 2), (2, 2, 3, 1)])
@pytest.mark.parametrize("mode", [0, 1])
def test_differently_misaligned_key_and_value_arrays(bj, oracle, torch_cuda, offsets, mode):
    # keys and values misaligned by different amounts, over many scatter tiles per slice
    rk, rv, sk, sv = bj.gen_host(31, 700_001, 900_003, 0.2)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    st, r, s, _ = run_device(bj, torch_cuda, rk, rv, sk, sv, cap=len(exp_r), offset=offsets,
                             partition_mode=mode, use_bloom=mode)
    assert st.count == len(exp_r)
    assert_same_pairs(oracle, r, s, exp_r, exp_s)


def test_capacity_overflow_counts_exactly(bj, oracle, torch_cuda):
    rk, rv, sk, sv = bj.gen_host(3, 50_000, 50_000, 0.4)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    cap = len(exp_r) // 3
    st, r, s, _ = run_device(bj, torch_cuda, rk, rv, sk, sv, cap=cap)
    assert st.count == len(exp_r) and st.overflow == 1 and st.written == cap and len(r) == cap
    exp = set(zip(exp_r.tolist(), exp_s.tolist()))
    got = list(zip(r.tolist(), s.tolist()))
    assert len(set(got)) == cap and all(p in exp for p in got)


def test_emit_key(bj, oracle, torch_cuda):
    rk, rv, sk, sv = bj.gen_host(4, 30_000, 40_000, 0.2)
    st, r, s, k = run_device(bj, torch_cuda, rk, rv, sk, sv, emit_key=True)
    assert np.array_equal(k, rk[r]) and np.array_equal(k, sk[s])


def test_zipf_skewed_probe_side(bj, oracle, torch_cuda):
    rk, rv, sk, sv = bj.gen_host(99, 200_000, 800_000, 0.1, zipf_s=1.0)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=1, s_chunk=4096)
    assert st.count == 80_000


@pytest.mark.parametrize("build_side", ["r", "s"])
def test_long_and_short_buckets_in_one_warp(bj, oracle, torch_cuda, build_side):
    """Build chunks holding a few keys repeated hundreds of times among unique keys: warps whose
    candidates mix long and short buckets take the load-balanced bucket walk."""
    rng = np.random.default_rng(5)
    uniq = rng.permutation(np.arange(1, 200_001, dtype=np.uint32))
    hot = np.repeat(np.array([7, 1_000_003, 0x80000000, 0xFFFFFFFF], np.uint32), [900, 300, 40, 9])
    small = np.concatenate([uniq[:30_000], hot])
    big = np.concatenate([uniq[10_000:150_000], np.array([7, 0x80000000, 0xFFFFFFFF, 5], np.uint32)])
    small = small[rng.permutation(len(small))]
    big = big[rng.permutation(len(big))]
    rk, sk = (small, big) if build_side == "r" else (big, small)
    rv = np.arange(len(rk), dtype=np.uint32)
    sv = np.arange(len(sk), dtype=np.uint32) + 3
    for bloom in (0, 1):
        _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=bloom, table_capacity=1024, emit_key=True)


def test_handle_reuse_and_graph_replay(bj, oracle, torch_cuda):
    with bj.Join(use_bloom=1, use_cuda_graph=1) as j:
        for seed in (1, 2, 3):
            rk, rv, sk, sv = bj.gen_host(seed, 120_000, 90_000, 0.25)
            exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
            st, r, s, _ = run_device(bj, torch_cuda, rk, rv, sk, sv, cap=len(exp_r) + 10, handle=j)
            assert st.count == len(exp_r)
            assert_same_pairs(oracle, r, s, exp_r, exp_s)


def test_run_host_entry_point(bj, oracle):
    rk, rv, sk, sv = bj.gen_host(8, 70_000, 60_000, 0.3)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    with bj.Join(use_bloom=1) as j:
        cnt, r, s = j.run_host(rk, rv, sk, sv, capacity=len(exp_r))
    assert cnt == len(exp_r)
    assert_same_pairs(oracle, r, s, exp_r, exp_s)


@pytest.mark.parametrize("pinned", [False, True])
def test_run_host_overlapped_copies(bj, oracle, torch_cuda, pinned):
    """Host inputs of at least 2^23 tuples: S is copied on a second stream while R's passes run,
    and S's passes wait for the copy (pageable arrays copy synchronously, pinned ones overlap)."""
    rk, rv, sk, sv = bj.gen_host(77, 4_500_000, 4_000_000, 0.2)
    if pinned:
        arrs = []
        for a in (rk, rv, sk, sv):
            t = torch_cuda.empty(len(a), dtype=torch_cuda.int32, pin_memory=True)
            t.numpy()[:] = a.view(np.int32)
            arrs.append(t.numpy().view(np.uint32))
        rk, rv, sk, sv = arrs
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    with bj.Join(use_bloom=1) as j:
        for _ in range(2):  # the second run reuses the handle's buffers, stream and events
            cnt, r, s = j.run_host(rk, rv, sk, sv, capacity=len(exp_r))
            assert cnt == len(exp_r) == 800_000
            assert_same_pairs(oracle, r, s, exp_r, exp_s)


@pytest.mark.parametrize("chunks,bloom,zipf", [(2, 1, 0.0), (3, 0, 0.0), (4, 1, 1.0), (7, 1, 0.0)])
def test_run_host_s_chunks(bj, oracle, torch_cuda, chunks, bloom, zipf):
    """S copied and joined in chunks against R partitioned and filtered once (the reference's
    s_chunks loop): the same pairs as the one-piece join, with a smaller last chunk (|S| is not a
    multiple of the chunk count), and again on the same handle."""
    rk, rv, sk, sv = bj.gen_host(55 + chunks, 300_000, 1_000_003, 0.3, zipf_s=zipf)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    with bj.Join(use_bloom=bloom, s_chunks=chunks) as j:
        for _ in range(2):
            cnt, r, s = j.run_host(rk, rv, sk, sv, capacity=len(exp_r))
            assert cnt == len(exp_r)
            assert_same_pairs(oracle, r, s, exp_r, exp_s)
        st = j.stats()
        assert st.count == len(exp_r) and st.overflow == 0
        assert st.count <= st.s_survivors <= len(sk)


def test_run_host_s_chunks_keys_and_overflow(bj, oracle, torch_cuda):
    rk, rv, sk, sv = bj.gen_host(91, 200_000, 600_000, 0.4)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    with bj.Join(use_bloom=1, s_chunks=5) as j:
        cnt, r, s, k = j.run_host(rk, rv, sk, sv, capacity=len(exp_r), emit_key=True)
        assert cnt == len(exp_r)
        assert np.array_equal(k, rk[r]) and np.array_equal(k, sk[s])
        # pairs past the capacity are counted but not written, across chunk boundaries
        cap = len(exp_r) // 3
        cnt, r, s = j.run_host(rk, rv, sk, sv, capacity=cap, allow_overflow=True)
        assert cnt == len(exp_r) and len(r) == cap and j.last_status == bj.BRIG_E_OVERFLOW
        exp = set(zip(exp_r.tolist(), exp_s.tolist()))
        assert len(set(zip(r.tolist(), s.tolist()))) == cap and all(p in exp for p in zip(r.tolist(), s.tolist()))


def test_device_generator_matches_host(bj, torch_cuda):
    n_r, n_s = 300_001, 500_003
    h = bj.gen_host(1234, n_r, n_s, 0.37)
    d = [torch_cuda.empty(n, dtype=torch_cuda.int32, device="cuda") for n in (n_r, n_r, n_s, n_s)]
    bj.gen_device(1234, n_r, n_s, 0.37, 0.0, *d)
    torch_cuda.cuda.synchronize()
    for a, b in zip(h, d):
        assert np.array_equal(a, b.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("preset", ["reference_fanout_512", "planner"])
def test_config0_16M_x_16M(bj, oracle, torch_cuda, preset):
    """The plain single join at its stated size: |R| = |S| = 2^24, 10% of S matching, Bloom filter on
    (10 bits/key, k = 7). `reference_fanout_512` is the reference's README preset --partition_size
    512, i.e. first-level fan-out 512 by key % 512 (second level auto: 67); `planner` is the engine's
    own choice. Exact count and identical sorted pair multiset against the oracle."""
    n = 1 << 24
    rk, rv, sk, sv = bj.gen_host(42, n, n, 0.1)
    cfg = dict(use_bloom=1, bloom_bits_per_key=10.0, bloom_num_hashes=7)
    if preset == "reference_fanout_512":
        cfg.update(partition_mode=bj.PART_MODULO, partition_size=512)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, **cfg)
    assert st.count == 1_677_721 and st.bloom_num_hashes == 7
    assert st.count <= st.s_survivors < n // 4
    if preset == "reference_fanout_512":
        assert (st.partition_size, st.second_partition_size) == (512, 67)


def test_bounded_waits_report_internal_error_and_stay_exact(bj, oracle, torch_cuda):
    """wait_poll_limit = -1 gives every bounded wait of the kernels (the bulk-copy mbarriers of the
    scatters) no polls: each one counts a device-side error at once and then waits
    for its copy with the default bound. The run must end (no hang), report BRIG_E_INTERNAL, publish
    -1 as the device count, keep its pairs exact, and leave the context usable for the next run."""
    rk, rv, sk, sv = bj.gen_host(77, 300_000, 400_000, 0.2)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    cap = len(exp_r) + 16
    d = [torch_cuda.from_numpy(a.view(np.int32)).cuda() for a in (rk, rv, sk, sv)]
    out_r = torch_cuda.empty(cap, dtype=torch_cuda.int32, device="cuda")
    out_s = torch_cuda.empty(cap, dtype=torch_cuda.int32, device="cuda")
    d_count = torch_cuda.zeros(1, dtype=torch_cuda.int64, device="cuda")
    with bj.Join(use_bloom=1, partition_size=16, second_partition_size=8, wait_poll_limit=-1) as j:
        j.run(d[0], d[1], len(rk), d[2], d[3], len(sk), out_r, out_s, cap, d_count=d_count)
        with pytest.raises(bj.BrigError) as e:
            j.stats()
        assert e.value.status == bj.BRIG_E_INTERNAL
        assert int(d_count.item()) == -1
    n = len(exp_r)
    assert_same_pairs(oracle, out_r[:n].cpu().numpy().view(np.uint32), out_s[:n].cpu().numpy().view(np.uint32),
                      exp_r, exp_s)
    st = _parity(bj, oracle, torch_cuda, rk, rv, sk, sv, use_bloom=1, partition_size=16, second_partition_size=8)
    assert st.count == n


def test_gather_rate_helper(bj, torch_cuda):
    """brig_join_gather_rate (the benchmark's ceiling for the level-2 Bloom probe's filter reads)
    enqueues one kernel of the requested size and rejects tables that are not a power of two."""
    table = torch_cuda.arange(1 << 18, dtype=torch_cuda.int32, device="cuda")
    sink = torch_cuda.zeros(1, dtype=torch_cuda.int32, device="cuda")
    n0 = bj.kernel_launches()
    issued = bj.gather_rate(table, 1 << 24, sink)
    torch_cuda.cuda.synchronize()
    assert bj.kernel_launches() - n0 == 1
    assert (1 << 23) < issued <= (1 << 24)
    with pytest.raises(bj.BrigError):
        bj.gather_rate(table[:1000], 1 << 20, sink)


def test_adaptive_bloom_switches_off_and_retests(bj, oracle, torch_cuda):
    """use_bloom = BLOOM_ADAPTIVE: a run whose filter lets more than 30% of S through turns the filter
    off for the handle's next single joins, every 16th of which tests it again; once a test run
    sees few survivors the filter stays on. Every run is exact."""
    hi = bj.gen_host(71, 200_000, 300_000, 0.6)   # 60% of S matches: the filter does not pay
    lo = bj.gen_host(72, 200_000, 300_000, 0.05)  # 5% matches: it does
    exp = {id(x): oracle.pairs(*x) for x in (hi, lo)}
    with bj.Join(use_bloom=bj.BLOOM_ADAPTIVE) as j:
        def run(data):
            st, r, s, _ = run_device(bj, torch_cuda, *data, cap=len(data[2]), handle=j)
            er, es = exp[id(data)]
            assert st.count == len(er)
            assert_same_pairs(oracle, r, s, er, es)
            return st.bloom_num_hashes > 0, st.s_survivors
        on, surv = run(hi)  # first run filtered: its survivors (> 30%) come back behind it
        assert on and surv > 0.3 * len(hi[2])
        states = [run(hi)[0] for _ in range(16)]  # runs 2..17: off, except the 16th (a re-test)
        assert states == [False] * 15 + [True]
        states = [run(lo)[0] for _ in range(16)]  # runs 18..33: off until the re-test at 33
        assert states == [False] * 15 + [True]
        assert run(lo)[0] and run(lo)[0]  # the re-test saw 5% survivors: the filter stays on
