"""Served joins: continuous batching under an HBM budget returns exactly the oracle result for every
request, and a request's result is the same alone and in a mix of concurrent requests."""
import threading
import time

import numpy as np
import pytest

from gpu_helpers import assert_same_pairs

pytestmark = pytest.mark.gpu


def _req(bj, seed, nr, ratio, frac):
    return bj.gen_host(seed, nr, nr * ratio, frac)


def test_every_request_matches_oracle(bj, oracle, torch_cuda):
    rng = np.random.default_rng(1)
    reqs = [_req(bj, 1000 + i, int(rng.integers(1, 200_000)), int(rng.choice([1, 4, 16])),
                 float(rng.choice([0.01, 0.1, 0.5]))) for i in range(40)]
    with bj.Server(hbm_budget_bytes=2 << 30, max_wave=8, streams=2, use_bloom=1) as srv:
        tickets = [srv.submit(*r) for r in reqs]
        waves = set()
        for t, r in zip(tickets, reqs):
            res, a, b = srv.poll(t)
            assert res.status == bj.BRIG_OK
            er, es = oracle.pairs(*r)
            assert res.count == len(er)
            assert_same_pairs(oracle, a, b, er, es)
            waves.add(res.wave)
    assert len(waves) > 1


def test_same_result_alone_and_in_mix(bj, oracle, torch_cuda):
    x = _req(bj, 77, 150_000, 4, 0.5)
    er, es = oracle.pairs(*x)
    with bj.Server(hbm_budget_bytes=4 << 30, max_wave=16, streams=3, use_bloom=1) as srv:
        res, a, b = srv.poll(srv.submit(*x))
        assert res.count == len(er)
        assert_same_pairs(oracle, a, b, er, es)
        # the same request again, arriving while a stream of other requests is being served
        others = [_req(bj, 200 + i, 50_000 + 7000 * i, 4, 0.1) for i in range(24)]
        stop = threading.Event()
        tix = []

        def feeder():
            for r in others:
                tix.append((srv.submit(*r), r))
                time.sleep(0.002)
        th = threading.Thread(target=feeder)
        th.start()
        time.sleep(0.01)
        t = srv.submit(*x)
        th.join()
        res2, a2, b2 = srv.poll(t)
        assert res2.count == len(er)
        assert_same_pairs(oracle, a2, b2, er, es)
        for tk, r in tix:
            resk, ak, bk = srv.poll(tk)
            ork, osk = oracle.pairs(*r)
            assert resk.count == len(ork)
            assert_same_pairs(oracle, ak, bk, ork, osk)


def test_wave_tuple_cap_runs_large_requests_alone(bj, oracle, torch_cuda):
    # With a 1M-tuple cap per wave, requests above 1M tuples each run as a wave of their own, while
    # the small ones may share waves; every result is still exact.
    small = [_req(bj, 300 + i, 20_000, 4, 0.1) for i in range(8)]
    large = [_req(bj, 400 + i, 400_000, 4, 0.1) for i in range(3)]
    reqs = small[:4] + large + small[4:]
    with bj.Server(hbm_budget_bytes=4 << 30, max_wave=16, streams=1, max_wave_mtuples=1) as srv:
        tickets = [srv.submit(*r) for r in reqs]
        results = [srv.poll(t) for t in tickets]
    waves = {}
    for (res, a, b), r in zip(results, reqs):
        assert res.status == bj.BRIG_OK
        er, es = oracle.pairs(*r)
        assert res.count == len(er)
        assert_same_pairs(oracle, a, b, er, es)
        waves.setdefault(res.wave, []).append(len(r[0]) + len(r[2]))
    for sizes in waves.values():
        assert sum(sizes) <= 1_000_000 or len(sizes) == 1, waves


def test_admission_rejects_oversized_and_drains_under_tight_budget(bj, oracle, torch_cuda):
    big = _req(bj, 5, 2_000_000, 1, 0.1)
    small = [_req(bj, 50 + i, 100_000, 4, 0.1) for i in range(6)]
    with bj.Server(hbm_budget_bytes=64 << 20, max_wave=4, streams=2) as srv:
        with pytest.raises(bj.BrigError) as e:
            srv.submit(*big)
        assert e.value.status == bj.BRIG_E_REJECTED
        tix = [srv.submit(*r) for r in small]
        for t, r in zip(tix, small):
            res, a, b = srv.poll(t)
            assert res.status == bj.BRIG_OK and res.count == 40_000


def test_poll_timeout_and_unknown_ticket(bj, torch_cuda):
    with bj.Server(hbm_budget_bytes=1 << 30) as srv:
        with pytest.raises(bj.BrigError) as e:
            srv.poll(12345, 0)
        assert e.value.status == bj.BRIG_E_INVALID
        t = srv.submit(*_req(bj, 3, 10_000, 1, 0.1))
        res, _, _ = srv.poll(t, 10_000)
        assert res.status == bj.BRIG_OK


def test_large_requests_run_one_at_a_time_and_small_ones_pass_them(bj, oracle, torch_cuda):
    """Requests above large_mtuples run one at a time on the first stream: no two of them are on the
    GPU together (each starts after the previous one's join has finished), while the small requests
    submitted behind them start without waiting for them; every result is exact."""
    reqs = []
    for i in range(9):
        big = i % 3 == 0
        nr, ns = (400_000, 900_000) if big else (20_000, 30_000)
        reqs.append((big, bj.gen_host(800 + i, nr, ns, 0.2)))
    exps = [oracle.pairs(*r) for _, r in reqs]
    with bj.Server(hbm_budget_bytes=8 << 30, max_wave=4, streams=3, large_mtuples=1) as srv:
        tickets = [srv.submit(*r, capacity=len(e[0]) + 8) for (_, r), e in zip(reqs, exps)]
        results = [srv.poll(t) for t in tickets]
    spans = []
    for (big, r), (er, es), (res, a, b) in zip(reqs, exps, results):
        assert res.status == bj.BRIG_OK and res.count == len(er)
        assert_same_pairs(oracle, a, b, er, es)
        if big:
            spans.append((res.queue_ms, res.queue_ms + res.setup_ms + res.join_ms))
    spans.sort()
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 0.05, spans  # the next large request started after the previous one's join
    smalls = [res.queue_ms for (big, _), (res, _, _) in zip(reqs, results) if not big]
    assert min(smalls) < spans[-1][0], (smalls, spans)  # some small request did not wait for the last large one
