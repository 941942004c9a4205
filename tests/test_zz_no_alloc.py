"""The allocation-free entry point (brig_join_run_noalloc) gives the same pairs and count as the
allocating entry point (brig_join_run), on two calls in a row that reuse its static scratch.

It serves callers that cannot allocate device memory when they join (a host framework that owns
all device memory through its own pool, or a latency-critical caller that cannot afford the
synchronisation of cudaMalloc/cudaFree). The file is named so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import assert_same_pairs, dev, run_device

pytestmark = pytest.mark.gpu


def _run_noalloc(bj, torch, rk, rv, sk, sv, cap, expect=None, **cfg):
    c = bj.make_config(**cfg)
    d = [dev(torch, a) for a in (rk, rv, sk, sv)]
    out_r = torch.empty(cap, dtype=torch.int32, device="cuda")
    out_s = torch.empty(cap, dtype=torch.int32, device="cuda")
    d_count = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    o = bj.Output(out_r.data_ptr(), out_s.data_ptr(), None, cap, d_count.data_ptr())
    st = bj.lib().brig_join_run_noalloc(C.byref(c), d[0].data_ptr(), d[1].data_ptr(), len(rk),
                                        d[2].data_ptr(), d[3].data_ptr(), len(sk), C.byref(o), None)
    assert st == bj.BRIG_OK, bj.last_error()
    torch.cuda.synchronize()
    n = int(d_count.item())
    m = min(max(n, 0), cap)
    return n, out_r[:m].cpu().numpy().view(np.uint32), out_s[:m].cpu().numpy().view(np.uint32)


def test_noalloc_matches_allocating_entry_point_on_two_calls(bj, oracle, torch_cuda):
    cases = [  # (n_r, n_s, match fraction, config); the second call has a different layout
        (200_000, 250_000, 0.3, dict(use_bloom=1)),
        (120_000, bj.NOALLOC_MAX_TUPLES, 0.6, dict(partition_mode=bj.PART_MODULO, partition_size=512)),
    ]
    for i, (nr, ns, frac, cfg) in enumerate(cases):
        rk, rv, sk, sv = bj.gen_host(900 + i, nr, ns, frac)
        st, r_ref, s_ref, _ = run_device(bj, torch_cuda, rk, rv, sk, sv, cap=ns, **cfg)
        n, r, s = _run_noalloc(bj, torch_cuda, rk, rv, sk, sv, ns, **cfg)
        assert n == st.count == int(frac * ns)
        assert_same_pairs(oracle, r, s, r_ref, s_ref)
        assert_same_pairs(oracle, r, s, *oracle.pairs(rk, rv, sk, sv))


def test_noalloc_reports_device_errors_through_the_count(bj, oracle, torch_cuda):
    """With no handle to report BRIG_E_INTERNAL through, a device-side failure reaches the caller as
    -1 in d_count: every bounded wait is made to give up at once (wait_poll_limit = -1), then a
    default call on the same scratch gives the exact count again."""
    rk, rv, sk, sv = bj.gen_host(950, 100_000, 150_000, 0.2)
    n, _, _ = _run_noalloc(bj, torch_cuda, rk, rv, sk, sv, 150_000, use_bloom=1, wait_poll_limit=-1)
    assert n == -1
    n, r, s = _run_noalloc(bj, torch_cuda, rk, rv, sk, sv, 150_000, use_bloom=1)
    assert n == 30_000
    assert_same_pairs(oracle, r, s, *oracle.pairs(rk, rv, sk, sv))


def test_noalloc_rejects_sizes_beyond_its_limit(bj, torch_cuda):
    c = bj.make_config()
    buf = torch_cuda.zeros(16, dtype=torch_cuda.int32, device="cuda")
    cnt = torch_cuda.zeros(1, dtype=torch_cuda.int64, device="cuda")
    o = bj.Output(buf.data_ptr(), buf.data_ptr(), None, 16, cnt.data_ptr())
    p = buf.data_ptr()
    st = bj.lib().brig_join_run_noalloc(C.byref(c), p, p, bj.NOALLOC_MAX_TUPLES + 1, p, p, 10, C.byref(o), None)
    assert st == bj.BRIG_E_UNSUPPORTED and "BRIG_NOALLOC_MAX_TUPLES" in bj.last_error()
