"""GPU-side helpers for the parity tests: move numpy inputs to the device with torch (plumbing
only), call the engine through the C ABI, bring the pairs back and compare with the oracle."""
import numpy as np


def dev(torch, a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if len(a) == 0:
        return torch.empty(1, dtype=torch.int32, device="cuda")
    return torch.from_numpy(a.view(np.int32)).to("cuda")


def run_device(bj, torch, rk, rv, sk, sv, cap=None, emit_key=False, handle=None, offset=0, **cfg):
    """Joins numpy inputs on the GPU; returns (stats, r_vals, s_vals, keys-or-None).

    `offset` > 0 places each input `offset` elements into its buffer, so the kernels see
    addresses that are not 16-byte aligned; a 4-tuple gives each of (r_key, r_val, s_key, s_val)
    its own offset."""
    if cap is None:
        cap = max(len(sk), 1)
    offs = tuple(offset) if isinstance(offset, (tuple, list)) else (offset,) * 4
    ins = []
    for a, off in zip((rk, rv, sk, sv), offs):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        buf = torch.zeros(len(a) + off + 1, dtype=torch.int32, device="cuda")
        if len(a):
            buf[off:off + len(a)] = torch.from_numpy(a.view(np.int32)).to("cuda")
        ins.append(buf)
    ptr = [t.data_ptr() + 4 * off for t, off in zip(ins, offs)]
    out_r = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    out_s = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    out_k = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda") if emit_key else None
    d_count = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    own = handle is None
    j = handle if handle is not None else bj.Join(**cfg)
    try:
        j.run(ptr[0], ptr[1], len(rk), ptr[2], ptr[3], len(sk), out_r, out_s, cap, out_key=out_k,
              d_count=d_count)
        st = j.stats(allow_overflow=True)
    finally:
        if own:
            j.close()
    torch.cuda.synchronize()
    assert int(d_count.item()) == st.count, "device count differs from stats count"
    n = min(st.count, cap)
    r = out_r[:n].cpu().numpy().view(np.uint32).copy()
    s = out_s[:n].cpu().numpy().view(np.uint32).copy()
    k = out_k[:n].cpu().numpy().view(np.uint32).copy() if emit_key else None
    return st, r, s, k


def assert_same_pairs(oracle, got_r, got_s, exp_r, exp_s):
    assert len(got_r) == len(exp_r), f"pair count {len(got_r)} != oracle {len(exp_r)}"
    a = oracle.sort_pairs(got_r, got_s)
    b = oracle.sort_pairs(exp_r, exp_s)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), "pair multiset differs from oracle"
