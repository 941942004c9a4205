"""Test infrastructure for the sharded join (brig_join.shard): ranks as threads of one process, a host
stand-in for the device steps (CPU tests), and inputs spread over ranks."""
import threading

import numpy as np
import torch

OWNER_SEED = 0x6A09E667


def mix32_np(x):
    """The engine's 32-bit mix (MurmurHash3's finaliser) over a uint32 array."""
    x = np.array(x, dtype=np.uint64)  # a copy: the steps below work in place
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x85EBCA6B)) & np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(13)
    x = (x * np.uint64(0xC2B2AE35)) & np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(16)
    return x


def owners_np(keys, nranks):
    """Owner rank of every key, restated on the host: fastrange32(mix32(key ^ seed), nranks)."""
    k = np.asarray(keys, dtype=np.uint64) ^ np.uint64(OWNER_SEED)
    return ((mix32_np(k) * np.uint64(nranks)) >> np.uint64(32)).astype(np.int64)


class Hub:
    """The rendezvous of `size` thread ranks: every exchange posts one object per rank and returns
    all of them, in rank order, to every rank."""

    def __init__(self, size):
        self.size = size
        self.slots = [None] * size
        self.barrier = threading.Barrier(size, timeout=300)

    def exchange(self, rank, obj):
        self.slots[rank] = obj
        self.barrier.wait()
        got = list(self.slots)
        self.barrier.wait()
        return got


class ThreadComm:
    """brig_join.shard's exchange interface for ranks that are threads of one process."""

    def __init__(self, hub, rank):
        self.hub, self.rank, self.size = hub, rank, hub.size

    def all_to_all_v(self, x, counts):
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        blocks = [x[offs[r]:offs[r + 1]] for r in range(self.size)]
        got = self.hub.exchange(self.rank, blocks)
        mine = [got[r][self.rank] for r in range(self.size)]
        return torch.cat(mine), [int(b.numel()) for b in mine]

    def all_gather_v(self, x):
        got = self.hub.exchange(self.rank, x)
        return torch.cat(got), [int(t.numel()) for t in got]

    def all_reduce_sum(self, v, device):
        return int(sum(self.hub.exchange(self.rank, v)))


def run_ranks(hub, fn):
    """Runs fn(rank) on one thread per rank of `hub`; returns the results in rank order. A rank that
    fails breaks the hub's barrier, so the others stop too, and the first failure is re-raised."""
    out, errs = [None] * hub.size, []

    def body(r):
        try:
            out[r] = fn(r)
        except BaseException as e:  # noqa: BLE001 - re-raised below
            errs.append(e)
            hub.barrier.abort()

    ts = [threading.Thread(target=body, args=(r,)) for r in range(hub.size)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    if errs:
        raise next((e for e in errs if not isinstance(e, threading.BrokenBarrierError)), errs[0])
    return out


class HostShardOps:
    """A host stand-in for CudaShardOps on CPU tensors: owners from owners_np, an owner's 'filter'
    that lists the keys it owns (padded to whole blocks of 8 words), joins by the oracle."""

    def __init__(self, oracle):
        self.oracle = oracle

    def split(self, nranks, key, val, heavy=None, filt=None, filter_loc=None, num_hashes=0):
        k = key.numpy().view(np.uint32)
        v = val.numpy().view(np.uint32)
        bins = owners_np(k, nranks)
        nb = nranks
        if heavy is not None and heavy.numel():
            bins[np.isin(k, heavy.numpy().view(np.uint32))] = nranks
            nb += 1
        keep = np.ones(len(k), dtype=bool)
        if filt is not None:
            f = filt.numpy().view(np.uint32)
            loc = filter_loc.numpy().reshape(-1, 2)
            for o in range(nranks):
                sel = bins == o
                keep[sel] = np.isin(k[sel], f[loc[o, 0]:loc[o, 0] + loc[o, 1]]) if loc[o, 1] >= 8 else False
        kb, kk, kv = bins[keep], k[keep], v[keep]
        order = np.argsort(kb, kind="stable")
        counts = np.bincount(kb, minlength=nb)[:nb]
        return (torch.from_numpy(kk[order].view(np.int32).copy()), torch.from_numpy(kv[order].view(np.int32).copy()),
                [int(c) for c in counts])

    def bloom_build(self, key, bits_per_key, num_hashes):
        keys = np.unique(key.numpy().view(np.uint32))
        pad = (-len(keys)) % 8 if len(keys) else 8
        words = np.concatenate([keys, np.zeros(pad, dtype=np.uint32)])
        return torch.from_numpy(words.view(np.int32).copy())

    def join(self, rk, rv, sk, sv):
        a, b = self.oracle.pairs(rk.numpy().view(np.uint32), rv.numpy().view(np.uint32),
                                 sk.numpy().view(np.uint32), sv.numpy().view(np.uint32))
        return torch.from_numpy(a.view(np.int32).copy()), torch.from_numpy(b.view(np.int32).copy())

    def to_device(self, a, like):
        return torch.from_numpy(np.ascontiguousarray(a))


def spread(oracle, seed, n_r, n_s, size, match=0.2, hot=0.0):
    """One global pair of relations (oracle.gen, R keys distinct), its rows dealt to `size` ranks in
    contiguous slices; with hot > 0 that share of S rows takes one R key (a skewed S). Returns the
    global arrays and the per-rank slices [(rk, rv, sk, sv), ...]."""
    rk, rv, sk, sv = oracle.gen(seed, n_r, n_s, match)
    if hot > 0:
        rng = np.random.default_rng(seed)
        rows = rng.choice(n_s, int(hot * n_s), replace=False)
        sk = sk.copy()
        sk[rows] = rk[7]
    cut = lambda n, r: (n * r // size, n * (r + 1) // size)  # noqa: E731
    parts = []
    for r in range(size):
        a, b = cut(n_r, r)
        c, d = cut(n_s, r)
        parts.append((rk[a:b], rv[a:b], sk[c:d], sv[c:d]))
    return (rk, rv, sk, sv), parts
