"""Scheduler of the evolution server on its host-only backend (fake_device):
admission by footprint, continuous batching, failure paths.  No GPU."""
import threading
import time

import numpy as np
import pytest


@pytest.fixture()
def jw():
    import jimwlk
    return jimwlk


def bytes_of(N):
    return N * N * (144 + 32 + 192)


def test_fake_server_completes_everything(jw):
    srv = jw.Server(fake_device=True, max_bytes=64 << 20, fake_ns_per_site_step=0.5)
    rids = [srv.submit(N, steps, seed=i) for i, (N, steps) in enumerate([(64, 40), (128, 10), (32, 100), (256, 5)])]
    for rid, (N, steps) in zip(rids, [(64, 40), (128, 10), (32, 100), (256, 5)]):
        st, res, sb, rb = srv.wait(rid, timeout=30)
        assert st == jw.OK and res.N == N and res.steps == steps and len(sb) == N // 2 + 1
        assert res.t_submit <= res.t_admit <= res.t_done
    s = srv.stats()
    assert s.completed == 4 and s.failed == 0 and s.queued == 0
    assert s.site_steps == sum(N * N * k for N, k in [(64, 40), (128, 10), (32, 100), (256, 5)])
    # per-size totals: every size served, site-steps split exactly, no device
    # time on the host-only backend
    sizes = srv.size_stats()
    assert sorted(sizes) == [32, 64, 128, 256]
    for N, k in [(64, 40), (128, 10), (32, 100), (256, 5)]:
        assert sizes[N]["site_steps"] == N * N * k and sizes[N]["ticks"] >= 1
        assert sizes[N]["step_ms"] == 0.0 and sizes[N]["mv_ms"] == 0.0
    srv.close()


def test_admission_by_footprint(jw):
    """Only two 256^2 events fit; six requests all finish, never more than two resident."""
    budget = 2 * bytes_of(256) + bytes_of(256) // 2
    srv = jw.Server(fake_device=True, max_bytes=budget, fake_ns_per_site_step=2.0, max_steps_per_tick=4)
    rids = [srv.submit(256, 20, seed=i) for i in range(6)]
    results = [srv.wait(r, timeout=60) for r in rids]
    assert all(st == jw.OK for st, *_ in results)
    assert srv.stats().max_active == 2
    # later requests waited in the queue: admissions are spread out
    admits = sorted(res.t_admit for _, res, _, _ in results)
    assert admits[-1] > admits[0]
    srv.close()


def test_small_requests_pass_a_blocked_large_one(jw):
    """First fit: a 1024^2 request that does not fit yet does not block 32^2 ones."""
    budget = bytes_of(1024) + bytes_of(32) * 4
    srv = jw.Server(fake_device=True, max_bytes=budget, fake_ns_per_site_step=1.0, max_steps_per_tick=2)
    big1 = srv.submit(1024, 300, seed=1)
    time.sleep(0.05)
    big2 = srv.submit(1024, 30, seed=2)  # must wait for big1
    small = [srv.submit(32, 4, seed=10 + i) for i in range(3)]
    t_small = max(srv.wait(r, timeout=60)[1].t_done for r in small)
    res2 = srv.wait(big2, timeout=60)[1]
    srv.wait(big1, timeout=60)
    assert t_small < res2.t_admit  # the small ones ran while big2 was still queued
    srv.close()


def test_requests_join_while_others_run(jw):
    srv = jw.Server(fake_device=True, max_bytes=256 << 20, fake_ns_per_site_step=5.0, max_steps_per_tick=1)
    first = srv.submit(128, 200, seed=1)
    time.sleep(0.02)
    late = srv.submit(64, 3, seed=2)
    st, res_late, _, _ = srv.wait(late, timeout=30)
    st1, res_first, _, _ = srv.wait(first, timeout=30)
    assert st == st1 == jw.OK
    assert res_late.t_done < res_first.t_done  # admitted and finished while the first still ran
    srv.close()


def test_rejections_and_timeouts(jw):
    srv = jw.Server(fake_device=True, max_bytes=bytes_of(512), fake_ns_per_site_step=20.0)
    assert srv.try_submit(N=24, steps=1)[0] == jw.EUNSUPPORTED           # not a power of two
    assert srv.try_submit(N=4096, steps=1)[0] == jw.EUNSUPPORTED         # beyond 2048
    assert srv.try_submit(N=1024, steps=1)[0] == jw.ENOMEM               # larger than the whole budget
    assert srv.try_submit(N=64, steps=-1)[0] == jw.EINVAL                # poisoned parameters
    assert srv.try_submit(N=64, steps=1, kernel=jw.LINEAR_KERNEL)[0] == jw.EUNSUPPORTED
    assert srv.try_submit(N=64, steps=1, coupling=jw.HATTA_COUPLING_CONSTANT)[0] == jw.EUNSUPPORTED
    rid = srv.submit(512, 1000, seed=3)
    st, _ = srv.try_wait(rid, 0.01)
    assert st == jw.ETIMEOUT
    assert srv.try_wait(987654, 0.01)[0] == jw.ENOTFOUND
    srv.close()  # drops the running request cleanly


def test_concurrent_submitters(jw):
    srv = jw.Server(fake_device=True, max_bytes=128 << 20, fake_ns_per_site_step=0.2)
    out, lock = [], threading.Lock()

    def client(k):
        for i in range(5):
            rid = srv.submit(64, 5 + i, seed=100 * k + i)
            st, res, sb, _ = srv.wait(rid, timeout=30)
            with lock:
                out.append((st, res.steps))

    th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    [t.start() for t in th]
    [t.join() for t in th]
    assert len(out) == 20 and all(st == jw.OK for st, _ in out)
    assert srv.stats().completed == 20
    srv.close()


@pytest.mark.parametrize("tick_sites", [0, 3 * 64 * 64])
def test_shortest_remaining_work_first(jw, tick_sites):
    """A long request (512^2 x 100 steps) and three short ones (64^2 x 200).
    Every resident request at every tick (tick_sites = 0): the long one needs
    13 ticks of 8 steps and the short ones 25, so the long one finishes first.
    With tick_sites = 3 * 64^2 the short ones (less remaining work) take the
    ticks until they are done, and the long one finishes last."""
    srv = jw.Server(fake_device=True, max_bytes=1 << 30, fake_ns_per_site_step=20.0, max_steps_per_tick=8,
                    tick_sites=tick_sites)
    long_ = srv.submit(512, 100, seed=1)
    short = [srv.submit(64, 200, seed=2 + i) for i in range(3)]
    t_long = srv.wait(long_, timeout=60)[1].t_done
    t_short = [srv.wait(r, timeout=60)[1].t_done for r in short]
    if tick_sites:
        assert max(t_short) < t_long
    else:
        assert t_long < min(t_short)
    assert srv.stats().completed == 4
    srv.close()
