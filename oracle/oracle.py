"""ctypes loader for the CPU oracle (liboracle.so) and the reference's own CPU join
(_ref/libref_sanity.so, built from the reference's src/sanity_check.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg as the checker. The engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_sanity.so")
REF_GEN = os.path.join(HERE, "_ref", "gen_dataset")

_o = None
_r = None
vp = C.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _o
    if _o is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_count.argtypes = [vp, C.c_int64, vp, C.c_int64]
        L.oracle_count.restype = C.c_int64
        L.oracle_pairs.argtypes = [vp, vp, C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_int64]
        L.oracle_pairs.restype = C.c_int64
        L.oracle_sortmerge_pairs.argtypes = [vp, vp, C.c_int64, vp, vp, C.c_int64, vp, vp, C.c_int64]
        L.oracle_sortmerge_pairs.restype = C.c_int64
        L.oracle_sort_pairs.argtypes = [vp, vp, C.c_int64]
        L.oracle_sort_pairs.restype = C.c_int
        L.oracle_pairs_digest.argtypes = [vp, vp, C.c_int64]
        L.oracle_pairs_digest.restype = C.c_uint64
        L.oracle_gen.argtypes = [C.c_uint64, C.c_int64, C.c_int64, C.c_double, vp, vp, vp, vp]
        L.oracle_gen.restype = C.c_int
        _o = L
    return _o


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def count(rk, sk) -> int:
    rk, sk = _u32(rk), _u32(sk)
    return int(lib().oracle_count(rk.ctypes.data, len(rk), sk.ctypes.data, len(sk)))


def pairs(rk, rv, sk, sv, with_key=False):
    """All key-equal pairs as (r_vals, s_vals[, keys]), in S order."""
    rk, rv, sk, sv = _u32(rk), _u32(rv), _u32(sk), _u32(sv)
    n = int(lib().oracle_pairs(rk.ctypes.data, rv.ctypes.data, len(rk), sk.ctypes.data, sv.ctypes.data, len(sk),
                               None, None, None, 0))
    if n < 0:
        raise MemoryError("oracle_pairs")
    a = np.empty(n, np.uint32)
    b = np.empty(n, np.uint32)
    k = np.empty(n, np.uint32) if with_key else None
    lib().oracle_pairs(rk.ctypes.data, rv.ctypes.data, len(rk), sk.ctypes.data, sv.ctypes.data, len(sk),
                       a.ctypes.data, b.ctypes.data, k.ctypes.data if with_key else None, n)
    return (a, b, k) if with_key else (a, b)


def sortmerge_pairs(rk, rv, sk, sv):
    rk, rv, sk, sv = _u32(rk), _u32(rv), _u32(sk), _u32(sv)
    n = int(lib().oracle_sortmerge_pairs(rk.ctypes.data, rv.ctypes.data, len(rk), sk.ctypes.data, sv.ctypes.data,
                                         len(sk), None, None, 0))
    if n < 0:
        raise MemoryError("oracle_sortmerge_pairs")
    a = np.empty(n, np.uint32)
    b = np.empty(n, np.uint32)
    lib().oracle_sortmerge_pairs(rk.ctypes.data, rv.ctypes.data, len(rk), sk.ctypes.data, sv.ctypes.data, len(sk),
                                 a.ctypes.data, b.ctypes.data, n)
    return a, b


def sort_pairs(a, b):
    """Returns copies of (a, b) sorted lexicographically."""
    a, b = np.array(a, dtype=np.uint32, copy=True), np.array(b, dtype=np.uint32, copy=True)
    if lib().oracle_sort_pairs(a.ctypes.data, b.ctypes.data, len(a)) != 0:
        raise MemoryError("oracle_sort_pairs")
    return a, b


def digest(a, b) -> int:
    a, b = _u32(a), _u32(b)
    return int(lib().oracle_pairs_digest(a.ctypes.data, b.ctypes.data, len(a)))


def gen(seed, n_r, n_s, match_frac=0.1, want_vals=True):
    """The benchmark's synthetic inputs (uniform matches) computed on the host by gen.c:
    (r_key, r_val, s_key, s_val) as uint32 arrays (values None when want_vals is False)."""
    rk = np.empty(n_r, np.uint32)
    sk = np.empty(n_s, np.uint32)
    rv = np.empty(n_r, np.uint32) if want_vals else None
    sv = np.empty(n_s, np.uint32) if want_vals else None
    p = lambda a: a.ctypes.data if a is not None else None
    if lib().oracle_gen(seed, n_r, n_s, match_frac, p(rk), p(rv), p(sk), p(sv)) != 0:
        raise ValueError("oracle_gen: bad arguments")
    return rk, rv, sk, sv


# ---- the reference's own CPU join ---------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _r
    if _r is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(REF_LIB + " (build with `make -C oracle ref` where the reference is present)")
        L = C.CDLL(REF_LIB)
        L.ref_sanity_count.argtypes = [vp, C.c_longlong, vp, C.c_longlong, C.POINTER(C.c_double)]
        L.ref_sanity_count.restype = C.c_longlong
        L.ref_omp_max_threads.argtypes = []
        L.ref_omp_max_threads.restype = C.c_int
        _r = L
    return _r


def ref_count(rk, sk):
    """(count, seconds) from the reference's run_sanity_check on int32 views of the keys."""
    rk = np.ascontiguousarray(rk).view(np.int32)
    sk = np.ascontiguousarray(sk).view(np.int32)
    sec = C.c_double()
    n = ref_lib().ref_sanity_count(rk.ctypes.data, len(rk), sk.ctypes.data, len(sk), C.byref(sec))
    return int(n), sec.value


def ref_threads() -> int:
    return int(ref_lib().ref_omp_max_threads())
