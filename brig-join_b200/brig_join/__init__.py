"""Python binding of the B200 equi-join engine (ctypes over include/brig_join.h).

The engine itself is C++/CUDA in ``libbrigjoin.so``; this module only marshals arguments so the
tests and the benchmark can call the C ABI. Device arrays are passed as raw addresses (for example
``torch.Tensor.data_ptr()``), host arrays as numpy arrays. Loading fails loudly when the shared
library is missing: there is no Python or CPU fallback for the join.

The handle mirrors the reference's entry points: ``Join.run`` is the one-PE join path of
``gpu_main`` (src/hash_kernel.cu:103-1131) over device-resident inputs, ``Join.run_host`` its
H2D-inclusive "Total" form (src/hash_kernel.cu:637-641), ``Join.stats`` the PE0 summary
(src/hash_kernel.cu:1142-1156).
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libbrigjoin.so")
HEADERS = [os.path.join(REPO_ROOT, "include", "brig_join.h")]

BRIG_OK = 0
BRIG_E_INVALID = 1
BRIG_E_NOMEM = 2
BRIG_E_CUDA = 3
BRIG_E_OVERFLOW = 4
BRIG_E_UNSUPPORTED = 5
BRIG_E_TIMEOUT = 6
BRIG_E_INTERNAL = 7
BRIG_E_REJECTED = 8
BRIG_E_NOT_READY = 9
STATUS_NAMES = {
    0: "BRIG_OK", 1: "BRIG_E_INVALID", 2: "BRIG_E_NOMEM", 3: "BRIG_E_CUDA", 4: "BRIG_E_OVERFLOW",
    5: "BRIG_E_UNSUPPORTED", 6: "BRIG_E_TIMEOUT", 7: "BRIG_E_INTERNAL", 8: "BRIG_E_REJECTED",
    9: "BRIG_E_NOT_READY",
}
PART_HASH = 0
PART_MODULO = 1
BLOOM_ADAPTIVE = 2  # use_bloom: the filter, switched off while it lets more than 30% of S through
ABI_VERSION = 1
NUM_STAGES = 13
NOALLOC_MAX_TUPLES = 262144

_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)


class Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("partition_mode", C.c_int32),
        ("partition_size", C.c_int32),
        ("second_partition_size", C.c_int32),
        ("use_bloom", C.c_int32),
        ("bloom_num_hashes", C.c_int32),
        ("bloom_bits_per_key", C.c_double),
        ("bloom_num_bits", C.c_int64),
        ("table_capacity", C.c_int32),
        ("s_chunk", C.c_int32),
        ("emit_key", C.c_int32),
        ("device", C.c_int32),
        ("use_cuda_graph", C.c_int32),
        ("profile_stages", C.c_int32),
        ("bloom_probe_level", C.c_int32),
        ("max_level1_bits", C.c_int32),
        ("s_chunks", C.c_int32),
        ("wait_poll_limit", C.c_int32),
        ("partition_fill", C.c_int32),
        ("slices_per_sm", C.c_int32),
    ]


class Output(C.Structure):
    _fields_ = [
        ("r_val", C.c_void_p),
        ("s_val", C.c_void_p),
        ("key", C.c_void_p),
        ("capacity", C.c_int64),
        ("d_count", C.c_void_p),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("count", C.c_int64),
        ("written", C.c_int64),
        ("s_survivors", C.c_int64),
        ("tasks", C.c_int64),
        ("split_tasks", C.c_int64),
        ("overflow", C.c_int32),
        ("partition_size", C.c_int32),
        ("second_partition_size", C.c_int32),
        ("bloom_num_hashes", C.c_int32),
        ("bloom_num_bits", C.c_int64),
        ("workspace_bytes", C.c_int64),
    ]


class BatchItem(C.Structure):
    _fields_ = [
        ("r_key", C.c_void_p), ("r_val", C.c_void_p), ("n_r", C.c_int64),
        ("s_key", C.c_void_p), ("s_val", C.c_void_p), ("n_s", C.c_int64),
        ("out", Output),
    ]


class ServeConfig(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_int64),
        ("max_wave", C.c_int32),
        ("streams", C.c_int32),
        ("max_queue", C.c_int32),
        ("max_wave_mtuples", C.c_int32),
        ("large_mtuples", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


class ServeRequest(C.Structure):
    _fields_ = [
        ("r_key", C.c_void_p), ("r_val", C.c_void_p), ("n_r", C.c_int64),
        ("s_key", C.c_void_p), ("s_val", C.c_void_p), ("n_s", C.c_int64),
        ("inputs_on_device", C.c_int32),
        ("reserved0", C.c_int32),
        ("out_r_val", C.c_void_p),
        ("out_s_val", C.c_void_p),
        ("capacity", C.c_int64),
    ]


class ServeResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("wave", C.c_int32),
        ("count", C.c_int64),
        ("submit_to_done_ms", C.c_double),
        ("queue_ms", C.c_double),
        ("setup_ms", C.c_double),
        ("join_ms", C.c_double),
    ]


class ShardSpec(C.Structure):
    _fields_ = [("nranks", C.c_int32), ("bloom_num_hashes", C.c_int32), ("filter", C.c_void_p),
                ("filter_loc", C.c_void_p), ("heavy", C.c_void_p), ("n_heavy", C.c_int32),
                ("reserved", C.c_int32), ("bin_cache", C.c_void_p)]


class BrigError(RuntimeError):
    def __init__(self, status: int, msg: str, where: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")


_lib = None


def lib() -> C.CDLL:
    """Loads libbrigjoin.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C brig-join_b200` "
                           "(there is no fallback implementation)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.brig_join_config_init.argtypes = [C.POINTER(Config)]
    L.brig_join_config_init.restype = None
    L.brig_join_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.brig_join_destroy.argtypes = [vp]
    L.brig_join_run.argtypes = [vp, vp, vp, C.c_int64, vp, vp, C.c_int64, C.POINTER(Output), vp]
    L.brig_join_run_host.argtypes = [vp, vp, vp, C.c_int64, vp, vp, C.c_int64, vp, vp, vp,
                                     C.c_int64, _i64p, vp]
    L.brig_join_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.brig_join_plan.argtypes = [C.POINTER(Config), C.c_int64, C.c_int64, C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32), _i64p]
    L.brig_join_run_batch.argtypes = [vp, C.POINTER(BatchItem), C.c_int32, vp]
    L.brig_join_batch_counts.argtypes = [vp, _i64p, C.c_int32]
    L.brig_join_autotune.argtypes = [vp, C.POINTER(BatchItem), C.c_int32, vp, C.POINTER(Config)]
    L.brig_join_autotune_candidates.argtypes = [C.POINTER(Config), C.POINTER(Config), C.c_int32, C.POINTER(C.c_int32)]
    L.brig_gen_device.argtypes = [C.c_uint64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                  vp, vp, vp, vp, vp]
    L.brig_gen_host.argtypes = [C.c_uint64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                vp, vp, vp, vp]
    L.brig_join_stage_name.argtypes = [C.c_int32]
    L.brig_join_stage_name.restype = C.c_char_p
    L.brig_join_stage_times.argtypes = [vp, C.POINTER(C.c_double), C.c_int32]
    L.brig_join_run_noalloc.argtypes = [C.POINTER(Config), vp, vp, C.c_int64, vp, vp, C.c_int64,
                                        C.POINTER(Output), vp]
    L.brig_join_last_error.argtypes = []
    L.brig_join_last_error.restype = C.c_char_p
    L.brig_join_kernel_launches.argtypes = []
    L.brig_join_kernel_launches.restype = C.c_int64
    L.brig_join_gather_rate.argtypes = [vp, C.c_int64, C.c_int64, vp, _i64p, vp]
    L.brig_join_read_relation.argtypes = [C.c_char_p, C.c_int64, C.c_int32, C.c_uint32, vp, vp]
    L.brig_join_write_pairs.argtypes = [C.c_char_p, vp, vp, vp, C.c_int64]
    L.brig_shard_owner.argtypes = [C.c_uint32, C.c_int32]
    L.brig_shard_owner.restype = C.c_int32
    L.brig_shard_filter_words.argtypes = [C.c_int64, C.c_double]
    L.brig_shard_filter_words.restype = C.c_int64
    L.brig_shard_count.argtypes = [C.POINTER(ShardSpec), vp, C.c_int64, vp, vp]
    L.brig_shard_scatter.argtypes = [C.POINTER(ShardSpec), vp, vp, C.c_int64, vp, vp, vp, vp, vp]
    L.brig_shard_bloom_build.argtypes = [vp, C.c_int64, vp, C.c_int64, C.c_int32, vp]
    if hasattr(L, "brig_serve_create"):
        L.brig_serve_create.argtypes = [C.POINTER(Config), C.POINTER(ServeConfig), C.POINTER(vp)]
        L.brig_serve_submit.argtypes = [vp, C.POINTER(ServeRequest), _i64p]
        L.brig_serve_poll.argtypes = [vp, C.c_int64, C.c_int32, C.POINTER(ServeResult)]
        L.brig_serve_destroy.argtypes = [vp]
    _lib = L
    return L


def last_error() -> str:
    return lib().brig_join_last_error().decode()


def check(status: int, where: str, ok=(BRIG_OK,)) -> int:
    if status not in ok:
        raise BrigError(status, last_error(), where)
    return status


def header_functions() -> list[str]:
    """Names of every function declared in include/*.h (for export checks)."""
    names = []
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(brig_\w+)\s*\(", txt, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def make_config(**kw) -> Config:
    cfg = Config()
    lib().brig_join_config_init(C.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


def autotune_candidates(**kw) -> list:
    """The configurations brig_join_autotune may try from the configuration kw."""
    base = make_config(**kw)
    n = C.c_int32()
    check(lib().brig_join_autotune_candidates(C.byref(base), None, 0, C.byref(n)), "autotune_candidates")
    out = (Config * n.value)()
    check(lib().brig_join_autotune_candidates(C.byref(base), out, n.value, C.byref(n)), "autotune_candidates")
    return list(out)


def config_dict(c: Config) -> dict:
    """The fields of a Config as a dict (keyword arguments of make_config / Join)."""
    return {name: getattr(c, name) for name, _ in Config._fields_ if name != "abi_version"}


def plan(n_r: int, n_s: int, **kw):
    """(P1, P2, workspace bytes) the planner picks for a join of this shape."""
    cfg = make_config(**kw)
    p1, p2, ws = C.c_int32(), C.c_int32(), C.c_int64()
    check(lib().brig_join_plan(C.byref(cfg), n_r, n_s, C.byref(p1), C.byref(p2), C.byref(ws)), "plan")
    return p1.value, p2.value, ws.value


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(type(x))


class Join:
    """A join handle (brig_join_create / brig_join_destroy)."""

    def __init__(self, **kw):
        self.cfg = make_config(**kw)
        h = C.c_void_p()
        check(lib().brig_join_create(C.byref(self.cfg), C.byref(h)), "brig_join_create")
        self.h = h

    def close(self):
        if self.h:
            lib().brig_join_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, r_key, r_val, n_r, s_key, s_val, n_s, out_r, out_s, capacity, out_key=None,
            d_count=None, stream=None):
        """Device-array join (asynchronous on `stream`)."""
        out = Output(_ptr(out_r), _ptr(out_s), _ptr(out_key), capacity, _ptr(d_count))
        check(lib().brig_join_run(self.h, _ptr(r_key), _ptr(r_val), n_r, _ptr(s_key), _ptr(s_val), n_s,
                                  C.byref(out), _ptr(stream)), "brig_join_run")

    def stats(self, allow_overflow=False) -> Stats:
        st = Stats()
        ok = (BRIG_OK, BRIG_E_OVERFLOW) if allow_overflow else (BRIG_OK,)
        self.last_status = check(lib().brig_join_get_stats(self.h, C.byref(st)), "brig_join_get_stats", ok)
        return st

    def stage_times(self) -> dict:
        """{stage name: device milliseconds} of the last run (needs profile_stages=1)."""
        ms = (C.c_double * NUM_STAGES)()
        check(lib().brig_join_stage_times(self.h, ms, NUM_STAGES), "brig_join_stage_times")
        return {lib().brig_join_stage_name(i).decode(): ms[i] for i in range(NUM_STAGES)}

    def run_host(self, r_key: np.ndarray, r_val: np.ndarray, s_key: np.ndarray, s_val: np.ndarray,
                 capacity: int | None = None, emit_key=False, out=None, allow_overflow=False, stream=None):
        """Host-array join; returns (count, r_vals, s_vals[, keys]) trimmed to min(count, capacity)."""
        n_r, n_s = len(r_key), len(s_key)
        if capacity is None:
            capacity = max(n_s, 1)
        if out is None:
            out = (np.empty(capacity, np.uint32), np.empty(capacity, np.uint32),
                   np.empty(capacity, np.uint32) if emit_key else None)
        cnt = C.c_int64()
        ok = (BRIG_OK, BRIG_E_OVERFLOW) if allow_overflow else (BRIG_OK,)
        self.last_status = check(lib().brig_join_run_host(self.h, _ptr(r_key), _ptr(r_val), n_r, _ptr(s_key), _ptr(s_val), n_s,
                                       _ptr(out[0]), _ptr(out[1]), _ptr(out[2]), capacity, C.byref(cnt),
                                       _ptr(stream)), "brig_join_run_host", ok)
        n = min(cnt.value, capacity)
        res = (cnt.value, out[0][:n], out[1][:n])
        if emit_key:
            res = res + (out[2][:n],)
        return res

    def run_batch(self, items: list[dict], stream=None):
        check(lib().brig_join_run_batch(self.h, self._items(items), len(items), _ptr(stream)),
              "brig_join_run_batch")

    @staticmethod
    def _items(items):
        arr = (BatchItem * len(items))()
        for i, it in enumerate(items):
            arr[i] = BatchItem(_ptr(it["r_key"]), _ptr(it["r_val"]), it["n_r"], _ptr(it["s_key"]),
                               _ptr(it["s_val"]), it["n_s"],
                               Output(_ptr(it["out_r"]), _ptr(it["out_s"]), _ptr(it.get("out_key")),
                                      it["capacity"], _ptr(it.get("d_count"))))
        return arr

    def autotune(self, items: list[dict], stream=None) -> dict:
        """Times candidate configurations on this batch; keeps and returns the fastest."""
        chosen = Config()
        check(lib().brig_join_autotune(self.h, self._items(items), len(items), _ptr(stream), C.byref(chosen)),
              "brig_join_autotune")
        return {"table_capacity": chosen.table_capacity, "max_level1_bits": chosen.max_level1_bits,
                "use_bloom": chosen.use_bloom,
                "bloom_bits_per_key": chosen.bloom_bits_per_key if chosen.use_bloom else 0.0,
                "bloom_num_hashes": chosen.bloom_num_hashes if chosen.use_bloom else 0,
                "bloom_probe_level": chosen.bloom_probe_level if chosen.use_bloom else 0,
                "partition_fill": chosen.partition_fill, "slices_per_sm": chosen.slices_per_sm}

    def batch_counts(self, n: int, allow_overflow=False) -> np.ndarray:
        c = np.zeros(n, np.int64)
        ok = (BRIG_OK, BRIG_E_OVERFLOW) if allow_overflow else (BRIG_OK,)
        check(lib().brig_join_batch_counts(self.h, c.ctypes.data_as(_i64p), n), "brig_join_batch_counts", ok)
        return c


class Server:
    """Served joins (brig_serve_*): submit host-array requests, poll tickets."""

    def __init__(self, hbm_budget_bytes=0, max_wave=0, streams=0, max_queue=0, max_wave_mtuples=0,
                 large_mtuples=0, **join_cfg):
        self.cfg = make_config(**join_cfg)
        self.scfg = ServeConfig(hbm_budget_bytes, max_wave, streams, max_queue, max_wave_mtuples, large_mtuples)
        h = C.c_void_p()
        check(lib().brig_serve_create(C.byref(self.cfg), C.byref(self.scfg), C.byref(h)), "brig_serve_create")
        self.h = h
        self._keep = {}

    def submit(self, r_key, r_val, s_key, s_val, capacity=0, out=None, on_device=False) -> int:
        """Queues a join; host arrays (numpy) unless on_device. Returns the ticket."""
        if out is None and not on_device:
            cap = capacity if capacity > 0 else max(len(s_key), 1)
            out = (np.empty(cap, np.uint32), np.empty(cap, np.uint32))
        n_r = r_key.numel() if hasattr(r_key, "numel") else len(r_key)
        n_s = s_key.numel() if hasattr(s_key, "numel") else len(s_key)
        req = ServeRequest(_ptr(r_key), _ptr(r_val), n_r, _ptr(s_key), _ptr(s_val), n_s, 1 if on_device else 0, 0,
                           _ptr(out[0]) if out else None, _ptr(out[1]) if out else None, capacity)
        t = C.c_int64()
        check(lib().brig_serve_submit(self.h, C.byref(req), C.byref(t)), "brig_serve_submit")
        self._keep[t.value] = (r_key, r_val, s_key, s_val, out)
        return t.value

    def poll(self, ticket: int, timeout_ms: int = -1):
        """(result, r_vals, s_vals) once the ticket is done; raises BrigError(BRIG_E_NOT_READY) on timeout."""
        res = ServeResult()
        check(lib().brig_serve_poll(self.h, ticket, timeout_ms, C.byref(res)), "brig_serve_poll")
        keep = self._keep.pop(ticket)
        out = keep[4]
        n = min(res.count, len(out[0])) if out else 0
        return res, (out[0][:n] if out else None), (out[1][:n] if out else None)

    def close(self):
        if self.h:
            lib().brig_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def gen_host(seed: int, n_r: int, n_s: int, match_frac: float = 0.1, zipf_s: float = 0.0):
    """Synthetic inputs on the host: (r_key, r_val, s_key, s_val) uint32 arrays."""
    rk = np.empty(n_r, np.uint32)
    rv = np.empty(n_r, np.uint32)
    sk = np.empty(n_s, np.uint32)
    sv = np.empty(n_s, np.uint32)
    check(lib().brig_gen_host(seed, n_r, n_s, match_frac, zipf_s, _ptr(rk), _ptr(rv), _ptr(sk), _ptr(sv)),
          "brig_gen_host")
    return rk, rv, sk, sv


def gen_device(seed: int, n_r: int, n_s: int, match_frac, zipf_s, r_key, r_val, s_key, s_val, stream=None):
    check(lib().brig_gen_device(seed, n_r, n_s, match_frac, zipf_s, _ptr(r_key), _ptr(r_val), _ptr(s_key),
                                _ptr(s_val), _ptr(stream)), "brig_gen_device")


def kernel_launches() -> int:
    return int(lib().brig_join_kernel_launches())


def read_relation(path: str, n: int, read_val: bool = False, val_base: int = 1):
    """One relation in the reference's input layout: (keys, values) as uint32 arrays; without a value
    block the values are val_base + row (the reference uses 1 for R, 100000001 for S)."""
    import numpy as np
    k = np.empty(n, np.uint32)
    v = np.empty(n, np.uint32)
    check(lib().brig_join_read_relation(os.fsencode(path), n, 1 if read_val else 0, val_base,
                                        k.ctypes.data, v.ctypes.data), "brig_join_read_relation")
    return k, v


def write_pairs(path: str, r_val, s_val, key=None) -> None:
    """Writes pairs in the reference's headerless int32 block layout (keys, R values, S values)."""
    import numpy as np
    r = np.ascontiguousarray(r_val, np.uint32)
    s = np.ascontiguousarray(s_val, np.uint32)
    k = None if key is None else np.ascontiguousarray(key, np.uint32)
    if len(r) != len(s) or (k is not None and len(k) != len(r)):
        raise ValueError("pair arrays differ in length")
    check(lib().brig_join_write_pairs(os.fsencode(path), None if k is None else k.ctypes.data, r.ctypes.data,
                                      s.ctypes.data, len(r)), "brig_join_write_pairs")


def gather_rate(table, loads: int, sink, stream=None) -> int:
    """Enqueues the random-read kernel over the device tensor `table` (a power-of-two byte size);
    returns the number of 8-byte reads it performs. Time it with events around the call."""
    issued = C.c_int64()
    check(lib().brig_join_gather_rate(_ptr(table), table.numel() * table.element_size(), loads, _ptr(sink),
                                      C.byref(issued), _ptr(stream)), "brig_join_gather_rate")
    return int(issued.value)
