"""Sharded joins across GPUs: one process per GPU, the exchanges over torch.distributed (NCCL).

The reference's multi-PE join sends R and the Bloom-prefiltered S to the PE that owns each
first-level partition (src/r_shuffle.cu:33-191), merges the PEs' filters with an OR all-reduce
(src/bf_allreduce.cu:236-284), rebalances S' and replicates hot R partitions on skewed inputs
(src/s_redistribute.cu:26-152, src/r_replicate.cu:13-100), then joins locally. Here the device work
is the engine's, through the C ABI (brig_shard_* and brig_join_run, include/brig_join.h), and this
module moves the grouped tuples and the filters between ranks. Per rank, in the same collective
order on every rank whatever its data:

  1. heavy keys: each rank samples its S keys; the samples' most frequent keys are gathered, and a
     key whose estimated share of all of S exceeds ``heavy_share / nranks`` is heavy (the same
     sorted list on every rank);
  2. R is grouped by owner (brig_shard_owner) plus a heavy bin; bin r goes to rank r (all-to-all),
     the heavy bin to every rank (all-gather);
  3. each rank builds its owner's filter over the R tuples it received; the filters are gathered
     (they cover disjoint keys: no OR reduction);
  4. S is prefiltered against its owner's filter and grouped in one pass; bin r goes to rank r, the
     heavy bin stays;
  5. local joins: the owned R with the received S, the gathered heavy R with the kept heavy S.
Every matching pair comes out on exactly one rank. Keys and values travel as int32 tensors holding
the uint32 bit patterns.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import BRIG_OK, Join, ShardSpec, _ptr, check, lib

MAX_RANKS = 64
MAX_HEAVY = 1024


def owner(key: int, nranks: int) -> int:
    """Rank that owns `key` among `nranks` ranks."""
    o = lib().brig_shard_owner(key & 0xFFFFFFFF, nranks)
    if o < 0:
        raise ValueError(f"nranks {nranks} outside 1..{MAX_RANKS}")
    return o


def filter_words(n_keys: int, bits_per_key: float) -> int:
    """32-bit words of an owner's filter over n_keys keys."""
    w = lib().brig_shard_filter_words(n_keys, bits_per_key)
    if w < 0:
        raise ValueError(f"no filter for {n_keys} keys at {bits_per_key} bits per key")
    return w


def _i32(t: torch.Tensor) -> torch.Tensor:
    if t.dtype == torch.uint32:
        t = t.view(torch.int32)
    if t.dtype != torch.int32:
        raise TypeError(f"keys and values are 32-bit tensors, not {t.dtype}")
    return t.contiguous()


class TorchComm:
    """The exchanges over a torch.distributed process group (NCCL for CUDA tensors, gloo for CPU)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def all_to_all_v(self, x: torch.Tensor, counts: list[int]) -> tuple[torch.Tensor, list[int]]:
        """x holds one block per rank back to back (counts[r] elements for rank r); returns the
        blocks the ranks sent this rank, in rank order, and their sizes."""
        d = self.dist
        c = torch.tensor(counts, dtype=torch.int64, device=x.device)
        rc = torch.empty_like(c)
        d.all_to_all_single(rc, c, group=self.group)
        rcl = rc.tolist()
        y = torch.empty(sum(rcl), dtype=x.dtype, device=x.device)
        d.all_to_all_single(y, x[: sum(counts)], output_split_sizes=rcl, input_split_sizes=list(counts),
                            group=self.group)
        return y, rcl

    def all_gather_v(self, x: torch.Tensor) -> tuple[torch.Tensor, list[int]]:
        """Every rank's x, concatenated in rank order, and their sizes."""
        d = self.dist
        n = torch.tensor([x.numel()], dtype=torch.int64, device=x.device)
        ns = [torch.empty_like(n) for _ in range(self.size)]
        d.all_gather(ns, n, group=self.group)
        sizes = torch.cat(ns).tolist()
        m = max(1, max(sizes))
        pad = torch.zeros(m, dtype=x.dtype, device=x.device)
        pad[: x.numel()] = x
        parts = [torch.empty_like(pad) for _ in range(self.size)]
        d.all_gather(parts, pad, group=self.group)
        return torch.cat([p[:s] for p, s in zip(parts, sizes)]), sizes

    def all_reduce_sum(self, v: int, device) -> int:
        t = torch.tensor([v], dtype=torch.int64, device=device)
        self.dist.all_reduce(t, group=self.group)
        return int(t.item())


class CudaShardOps:
    """The device steps of a rank: the engine's shard kernels and joins on the current CUDA stream."""

    def __init__(self, **join_kw):
        self.join_handle = Join(**join_kw)
        self._lost = []  # each scatter's count of tuples that found their bin full, read by lost()

    @staticmethod
    def _stream():
        return torch.cuda.current_stream().cuda_stream

    def split(self, nranks: int, key, val, heavy=None, filt=None, filter_loc=None, num_hashes=0, cache=None):
        """Groups (key, val) into owner bins (and a heavy bin when `heavy` holds keys); with a filter
        only tuples that pass their owner's filter are kept. Returns (keys, values, bin counts).
        cache: keep each tuple's bin between the count and the scatter (default: with a filter, where
        it saves the second filter read)."""
        key, val = _i32(key), _i32(val)
        dev = key.device
        nh = 0 if heavy is None else heavy.numel()
        use_cache = (filt is not None) if cache is None else cache
        bins = torch.empty(max(key.numel(), 1), dtype=torch.uint8, device=dev) if use_cache else None
        sp = ShardSpec(nranks, num_hashes if filt is not None else 0, _ptr(filt), _ptr(filter_loc),
                       _ptr(heavy) if nh else None, nh, 0, _ptr(bins))
        nb = nranks + (1 if nh else 0)
        counts = torch.empty(nb, dtype=torch.int64, device=dev)
        st = self._stream()
        check(lib().brig_shard_count(C.byref(sp), _ptr(key), key.numel(), _ptr(counts), st), "brig_shard_count")
        cl = counts.tolist()
        total = sum(cl)
        ok = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
        ov = torch.empty_like(ok)
        scratch = torch.empty(2 * nb + 2, dtype=torch.int64, device=dev)
        check(lib().brig_shard_scatter(C.byref(sp), _ptr(key), _ptr(val), key.numel(), _ptr(counts), _ptr(scratch),
                                       _ptr(ok), _ptr(ov), st), "brig_shard_scatter")
        self._lost.append(scratch[2 * nb + 1:])
        return ok[:total], ov[:total], cl

    def lost(self) -> int:
        """Tuples that found their bin full in the scatters since the last call (one read for all)."""
        if not self._lost:
            return 0
        n = int(torch.cat(self._lost).sum().item())
        self._lost = []
        return n

    def bloom_build(self, key, bits_per_key: float, num_hashes: int) -> torch.Tensor:
        key = _i32(key)
        w = filter_words(key.numel(), bits_per_key)
        words = torch.empty(w, dtype=torch.int32, device=key.device)
        check(lib().brig_shard_bloom_build(_ptr(key), key.numel(), _ptr(words), w, num_hashes, self._stream()),
              "brig_shard_bloom_build")
        return words

    def join(self, rk, rv, sk, sv):
        """Local join; returns (r_vals, s_vals) of every pair."""
        rk, rv, sk, sv = _i32(rk), _i32(rv), _i32(sk), _i32(sv)
        dev = rk.device
        cap = max(sk.numel(), 1)
        for _ in range(2):
            out_r = torch.empty(cap, dtype=torch.int32, device=dev)
            out_s = torch.empty(cap, dtype=torch.int32, device=dev)
            self.join_handle.run(rk, rv, rk.numel(), sk, sv, sk.numel(), out_r, out_s, cap, stream=self._stream())
            st = self.join_handle.stats(allow_overflow=True)
            if self.join_handle.last_status == BRIG_OK:
                return out_r[: st.count], out_s[: st.count]
            cap = st.count  # BRIG_E_OVERFLOW: the count is exact, so the second run fits
        raise RuntimeError("local join overflowed twice")

    def to_device(self, a: np.ndarray, like: torch.Tensor) -> torch.Tensor:
        return torch.from_numpy(a).to(like.device)


@dataclass
class ShardResult:
    r_val: torch.Tensor        # this rank's pairs
    s_val: torch.Tensor
    count: int                 # pairs on this rank
    total: int                 # pairs on all ranks
    heavy_keys: np.ndarray     # the heavy keys (uint32, sorted; the same on every rank)
    stats: dict = field(default_factory=dict)


class ShardedJoin:
    """A join of relations spread over the ranks of `comm`, each rank holding some tuples of R and S.

    bits_per_key = 0 turns the prefilter off; heavy_share = 0 turns the heavy-key handling off.
    Every rank runs the same collectives in the same order. A scatter that found a bin full on any
    rank makes every rank raise after the last collective. A rank that fails in between leaves the
    others waiting in their next collective until the process group's timeout, so give the group a
    short timeout."""

    def __init__(self, comm, ops=None, bits_per_key: float = 10.0, num_hashes: int = 7, heavy_share: float = 0.1,
                 sample: int = 65536, max_heavy: int = 256, seed: int = 0, **join_kw):
        if comm.size > MAX_RANKS:
            raise ValueError(f"at most {MAX_RANKS} ranks")
        if max_heavy > MAX_HEAVY:
            raise ValueError(f"at most {MAX_HEAVY} heavy keys")
        self.comm = comm
        self.ops = ops if ops is not None else CudaShardOps(**join_kw)
        self.bits_per_key = bits_per_key
        self.num_hashes = num_hashes
        self.heavy_share = heavy_share
        self.sample = sample
        self.max_heavy = max_heavy
        self.seed = seed

    def heavy_keys(self, s_key: torch.Tensor) -> np.ndarray:
        """The heavy keys, from a sample of every rank's S (collective: every rank calls it)."""
        comm = self.comm
        if comm.size == 1:  # one rank: every tuple stays, there is nothing to balance
            return np.zeros(0, dtype=np.uint32)
        s_key = _i32(s_key)
        n = s_key.numel()
        m = min(n, self.sample) if self.heavy_share > 0 else 0
        keys = torch.zeros(0, dtype=torch.int32, device=s_key.device)
        cnts = torch.zeros(0, dtype=torch.int32, device=s_key.device)
        if m > 0:
            g = torch.Generator(device=s_key.device)
            g.manual_seed(self.seed * 1000003 + comm.rank)
            idx = torch.randint(0, n, (m,), device=s_key.device, generator=g)
            uniq, cnt = torch.unique(s_key[idx], return_counts=True)
            top = torch.topk(cnt, min(self.max_heavy, uniq.numel()))
            keys, cnts = uniq[top.indices], top.values.to(torch.int32)
        meta = torch.tensor([n, m], dtype=torch.int64, device=s_key.device)
        gk, sizes = comm.all_gather_v(keys)
        gc, _ = comm.all_gather_v(cnts)
        gm, _ = comm.all_gather_v(meta)
        gk = gk.cpu().numpy().view(np.uint32)
        gc = gc.cpu().numpy().astype(np.float64)
        gm = gm.cpu().numpy().reshape(-1, 2)
        total_s = float(gm[:, 0].sum())
        if total_s == 0 or self.heavy_share <= 0:
            return np.zeros(0, dtype=np.uint32)
        est, off = {}, 0
        for r, sz in enumerate(sizes):
            n_r, m_r = gm[r]
            for k, c in zip(gk[off: off + sz], gc[off: off + sz]):
                est[int(k)] = est.get(int(k), 0.0) + c * n_r / max(m_r, 1)
            off += sz
        bar = self.heavy_share * total_s / comm.size
        heavy = sorted(k for k, e in est.items() if e > bar and e >= 8)
        heavy = sorted(sorted(heavy, key=lambda k: -est[k])[: self.max_heavy])
        return np.array(heavy, dtype=np.uint32)

    def run(self, r_key, r_val, s_key, s_val) -> ShardResult:
        comm, ops = self.comm, self.ops
        ws = comm.size
        r_key, r_val, s_key, s_val = _i32(r_key), _i32(r_val), _i32(s_key), _i32(s_val)
        heavy = self.heavy_keys(s_key)
        heavy_t = ops.to_device(heavy.view(np.int32), r_key) if heavy.size else None
        # 2. R to its owners; the heavy bin to every rank
        rk, rv, rc = ops.split(ws, r_key, r_val, heavy=heavy_t)
        own = sum(rc[:ws])
        r_own_k, _ = comm.all_to_all_v(rk[:own], rc[:ws])
        r_own_v, _ = comm.all_to_all_v(rv[:own], rc[:ws])
        if heavy_t is not None:
            r_hvy_k, _ = comm.all_gather_v(rk[own:])
            r_hvy_v, _ = comm.all_gather_v(rv[own:])
        # 3. the owners' filters, gathered
        filt = loc = None
        if self.bits_per_key > 0:
            words = ops.bloom_build(r_own_k, self.bits_per_key, self.num_hashes)
            filt, sizes = comm.all_gather_v(words)
            offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
            loc = ops.to_device(np.stack([offs, np.asarray(sizes, dtype=np.int64)], axis=1).reshape(-1), r_key)
        # 4. S prefiltered and sent to its owners; the heavy bin stays
        sk, sv, sc = ops.split(ws, s_key, s_val, heavy=heavy_t, filt=filt, filter_loc=loc,
                               num_hashes=self.num_hashes)
        s_own = sum(sc[:ws])
        s_own_k, _ = comm.all_to_all_v(sk[:s_own], sc[:ws])
        s_own_v, _ = comm.all_to_all_v(sv[:s_own], sc[:ws])
        # 5. local joins
        a_r, a_s = ops.join(r_own_k, r_own_v, s_own_k, s_own_v)
        parts_r, parts_s = [a_r], [a_s]
        if heavy_t is not None:
            b_r, b_s = ops.join(r_hvy_k, r_hvy_v, sk[s_own:], sv[s_own:])
            parts_r.append(b_r)
            parts_s.append(b_s)
        out_r, out_s = torch.cat(parts_r), torch.cat(parts_s)
        count = out_r.numel()
        total = comm.all_reduce_sum(count, r_key.device)
        # every rank learns of a failed scatter on any rank and raises, after the same collectives
        lost = comm.all_reduce_sum(ops.lost() if hasattr(ops, "lost") else 0, r_key.device)
        if lost:
            raise RuntimeError(f"brig_shard_scatter: {lost} tuples found their bin full")
        stats = {"r_owned": r_own_k.numel(), "s_received": s_own_k.numel(), "s_survivors": sum(sc),
                 "s_heavy_kept": sum(sc[ws:]), "r_heavy": (r_hvy_k.numel() if heavy_t is not None else 0)}
        return ShardResult(out_r, out_s, count, total, heavy, stats)
