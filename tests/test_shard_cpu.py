"""The sharded join's host side on the CPU: key ownership, filter sizing, and the exchanges of
brig_join.shard run by thread ranks and by two gloo ranks, with a host stand-in for the device
steps (owners restated on the host, an exact 'filter', joins by the oracle). Every pair of the
union of the ranks' results must be the oracle's, each exactly once."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from shard_helpers import Hub, HostShardOps, ThreadComm, mix32_np, owners_np, run_ranks, spread

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def shard(bj):
    import brig_join.shard as sh
    return sh


def union(results):
    return (np.concatenate([r.r_val.numpy().view(np.uint32) for r in results]),
            np.concatenate([r.s_val.numpy().view(np.uint32) for r in results]))


def test_owner_matches_host_restatement(shard):
    rng = np.random.default_rng(1)
    keys = np.concatenate([[0, 1, 0x7FFFFFFF, 0x80000000, 0xFFFFFFFF], rng.integers(0, 2**32, 3000)]).astype(np.uint32)
    for nr in (1, 2, 3, 8, 64):
        got = np.array([shard.owner(int(k), nr) for k in keys])
        assert np.array_equal(got, owners_np(keys, nr)), nr
        assert got.min() >= 0 and got.max() < nr
    with pytest.raises(ValueError):
        shard.owner(5, 0)
    with pytest.raises(ValueError):
        shard.owner(5, 65)


def test_owners_are_even_and_independent_of_the_partition_bits(oracle):
    """Each owner gets about 1/nranks of the keys, and one owner's keys still fill every level-1
    partition (the top 9 bits of mix32) evenly, as the local join's planner expects."""
    rk, _, _, _ = oracle.gen(3, 400_000, 1, 0.0, want_vals=False)
    own = owners_np(rk, 8)
    share = np.bincount(own, minlength=8) / len(rk)
    assert np.all(np.abs(share - 0.125) < 0.005), share
    p1 = (mix32_np(rk[own == 0]) >> np.uint64(23)).astype(np.int64)
    per = np.bincount(p1, minlength=512)
    chi2 = float(((per - per.mean()) ** 2 / per.mean()).sum())
    assert per.min() > 0 and chi2 < 511 + 6 * 32, chi2  # uniform: 511 +- 32 (511 degrees of freedom)


def test_filter_words(shard):
    assert shard.filter_words(0, 10.0) == 8
    assert shard.filter_words(1000, 10.0) == 320  # 10000 bits: 40 blocks of 256
    assert shard.filter_words(1, 0.5) == 8
    with pytest.raises(ValueError):
        shard.filter_words(10, 0.0)
    with pytest.raises(ValueError):
        shard.filter_words(-1, 10.0)
    with pytest.raises(ValueError):
        shard.filter_words(1 << 40, 10.0)  # 2^32 words or more


@pytest.mark.parametrize("bits", [0.0, 10.0])
@pytest.mark.parametrize("hot", [0.0, 0.3])
def test_thread_ranks_give_the_oracle_pairs(shard, oracle, bits, hot):
    size = 3
    (rk, rv, sk, sv), parts = spread(oracle, 11, 30_000, 60_000, size, match=0.3, hot=hot)
    hub = Hub(size)

    def rank(r):
        job = shard.ShardedJoin(ThreadComm(hub, r), HostShardOps(oracle), bits_per_key=bits, sample=4096)
        return job.run(*(torch.from_numpy(a.view(np.int32).copy()) for a in parts[r]))

    res = run_ranks(hub, rank)
    got_r, got_s = union(res)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    assert len(got_r) == len(exp_r) and all(x.total == len(exp_r) for x in res)
    a, b = oracle.sort_pairs(got_r, got_s), oracle.sort_pairs(exp_r, exp_s)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    hk = [x.heavy_keys for x in res]
    assert all(np.array_equal(h, hk[0]) for h in hk)  # every rank takes the same heavy keys
    if hot:
        assert int(rk[7]) in hk[0].tolist()
        assert sum(x.stats["s_heavy_kept"] for x in res) >= int(0.3 * len(sk))
    else:
        assert len(hk[0]) == 0
    if bits:  # the prefilter drops S tuples that match nothing; the heavy ones skip it
        assert sum(x.stats["s_survivors"] for x in res) < len(sk)


def test_a_rank_without_tuples(shard, oracle):
    """One rank holds no R and no S tuple, another no R: they still take part in every exchange and
    the union of the results is the oracle's."""
    size = 3
    (rk, rv, sk, sv), parts = spread(oracle, 13, 9000, 20000, size, match=0.4, hot=0.2)
    e = np.zeros(0, dtype=np.uint32)
    parts = [parts[0], (e, e, e, e), (e, e, np.concatenate([parts[1][2], parts[2][2]]),
                                      np.concatenate([parts[1][3], parts[2][3]]))]
    rk, rv = parts[0][0], parts[0][1]
    hub = Hub(size)

    def rank(r):
        job = shard.ShardedJoin(ThreadComm(hub, r), HostShardOps(oracle), sample=4096)
        return job.run(*(torch.from_numpy(a.view(np.int32).copy()) for a in parts[r]))

    res = run_ranks(hub, rank)
    got_r, got_s = union(res)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    assert all(x.total == len(exp_r) for x in res)
    a, b = oracle.sort_pairs(got_r, got_s), oracle.sort_pairs(exp_r, exp_s)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_heavy_keys_take_the_heaviest_up_to_the_cap(shard, oracle):
    """Five hot keys of different weights and a cap of two: every rank picks the same two, the
    heaviest ones."""
    size = 3
    rng = np.random.default_rng(3)
    (rk, rv, sk, sv), parts = spread(oracle, 17, 5000, 60_000, size, match=0.1)
    sk = sk.copy()
    hot = rk[10:15]
    rows = rng.permutation(len(sk))
    start = 0
    for key, share in zip(hot, (0.20, 0.16, 0.12, 0.08, 0.04)):
        n = int(share * len(sk))
        sk[rows[start:start + n]] = key
        start += n
    cut = [(len(sk) * r // size, len(sk) * (r + 1) // size) for r in range(size)]
    parts = [(parts[r][0], parts[r][1], sk[a:b], sv[a:b]) for r, (a, b) in enumerate(cut)]
    hub = Hub(size)

    def rank(r):
        job = shard.ShardedJoin(ThreadComm(hub, r), HostShardOps(oracle), bits_per_key=0.0, max_heavy=2,
                                sample=8192)
        return job.heavy_keys(torch.from_numpy(parts[r][2].view(np.int32).copy()))

    got = run_ranks(hub, rank)
    assert all(np.array_equal(g, got[0]) for g in got)
    assert got[0].tolist() == sorted(int(k) for k in hot[:2])


def test_exchanges_of_nothing(shard):
    """Every rank sends and gathers empty blocks: the exchanges return empty tensors and sizes."""
    size = 2
    hub = Hub(size)

    def rank(r):
        c = ThreadComm(hub, r)
        y, rc = c.all_to_all_v(torch.zeros(0, dtype=torch.int32), [0, 0])
        g, sizes = c.all_gather_v(torch.zeros(0, dtype=torch.int32))
        return y.numel(), rc, g.numel(), sizes, c.all_reduce_sum(0, "cpu")

    assert run_ranks(hub, rank) == [(0, [0, 0], 0, [0, 0], 0)] * size


def test_sharded_join_arguments(shard, oracle):
    class Many:
        rank, size = 0, 65

    with pytest.raises(ValueError):
        shard.ShardedJoin(Many(), HostShardOps(oracle))
    with pytest.raises(ValueError):
        shard.ShardedJoin(ThreadComm(Hub(1), 0), HostShardOps(oracle), max_heavy=shard.MAX_HEAVY + 1)
    with pytest.raises(TypeError):
        shard.ShardedJoin(ThreadComm(Hub(1), 0), HostShardOps(oracle)).run(
            *(torch.zeros(3, dtype=torch.int64) for _ in range(4)))


def test_heavy_keys_keep_a_hot_key_off_its_owner(shard, oracle):
    """A key held by 40% of S: with the heavy-key handling every rank receives about its fair
    share; without it the hot key's owner receives its whole share of S."""
    size = 4
    _, parts = spread(oracle, 5, 20_000, 80_000, size, match=0.1, hot=0.4)

    def received(heavy_share):
        hub = Hub(size)

        def rank(r):
            job = shard.ShardedJoin(ThreadComm(hub, r), HostShardOps(oracle), bits_per_key=0.0,
                                    heavy_share=heavy_share, sample=8192)
            x = job.run(*(torch.from_numpy(a.view(np.int32).copy()) for a in parts[r]))
            return x.stats["s_received"] + x.stats["s_heavy_kept"]

        return np.array(run_ranks(hub, rank))

    with_heavy, without = received(0.1), received(0.0)
    assert with_heavy.max() < 1.15 * with_heavy.mean()
    assert without.max() > 1.8 * without.mean()


def test_a_failing_rank_stops_the_others(shard, oracle):
    """A rank that raises before an exchange breaks the rendezvous; the others end with an error
    instead of waiting."""
    size = 3
    _, parts = spread(oracle, 2, 3000, 3000, size)
    hub = Hub(size)

    class Boom(HostShardOps):
        def bloom_build(self, key, bits_per_key, num_hashes):
            raise RuntimeError("rank 1 fails")

    def rank(r):
        ops = Boom(oracle) if r == 1 else HostShardOps(oracle)
        return shard.ShardedJoin(ThreadComm(hub, r), ops).run(
            *(torch.from_numpy(a.view(np.int32).copy()) for a in parts[r]))

    with pytest.raises(RuntimeError, match="rank 1 fails"):
        run_ranks(hub, rank)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out_dir, hot):
    import datetime
    import torch.distributed as dist
    sys.path[:0] = [HERE, ROOT, os.path.join(ROOT, "brig-join_b200")]
    import brig_join.shard as sh
    from oracle import oracle as o
    from shard_helpers import HostShardOps as Ops, spread as spr
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        _, parts = spr(o, 21, 20_000, 50_000, world, match=0.25, hot=hot)
        job = sh.ShardedJoin(sh.TorchComm(), Ops(o), bits_per_key=10.0, sample=4096)
        x = job.run(*(torch.from_numpy(a.view(np.int32).copy()) for a in parts[rank]))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), r=x.r_val.numpy(), s=x.s_val.numpy(), total=x.total,
                 heavy=x.heavy_keys)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("hot", [0.0, 0.3])
def test_two_gloo_ranks_give_the_oracle_pairs(oracle, tmp_path, hot):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, str(tmp_path), hot)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    outs = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    got_r = np.concatenate([d["r"] for d in outs]).view(np.uint32)
    got_s = np.concatenate([d["s"] for d in outs]).view(np.uint32)
    (rk, rv, sk, sv), _ = spread(oracle, 21, 20_000, 50_000, world, match=0.25, hot=hot)
    exp_r, exp_s = oracle.pairs(rk, rv, sk, sv)
    assert all(int(d["total"]) == len(exp_r) for d in outs)
    a, b = oracle.sort_pairs(got_r, got_s), oracle.sort_pairs(exp_r, exp_s)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(outs[0]["heavy"], outs[1]["heavy"])
    assert (int(rk[7]) in outs[0]["heavy"].tolist()) == (hot > 0)
