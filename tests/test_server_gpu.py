"""The evolution server on the GPU: every request's result is the same when it
runs alone and when it runs mixed with others (continuous batching), the
mixed-precision S(r) matches the FP64 oracle, and footprint admission works."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIX = [dict(N=32, steps=12, seed=5, coupling=3), dict(N=64, steps=7, seed=6, coupling=1),
       dict(N=32, steps=20, seed=7, coupling=0), dict(N=128, steps=5, seed=8, coupling=3),
       dict(N=16, steps=30, seed=9, coupling=3), dict(N=64, steps=16, seed=10, coupling=0)]


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def run(jw, reqs, **opt):
    srv = jw.Server(**opt)
    rids = [srv.submit(r["N"], r["steps"], ny_slices=6, step=0.0004, coupling=r["coupling"], seed=r["seed"])
            for r in reqs]
    out = [srv.wait(rid, timeout=300) for rid in rids]
    st = srv.stats()
    srv.close()
    return out, st


@pytest.mark.parametrize("tick_sites", [0, 2 * 64 * 64])
@pytest.mark.parametrize("precision", [1, 0])
def test_each_result_same_alone_and_in_mix(jw, precision, tick_sites):
    """Also with the least-remaining-work-first ticks (tick_sites), which step
    different subsets of the resident requests at each tick."""
    mixed, st = run(jw, MIX, precision=precision, max_steps_per_tick=4, tick_sites=tick_sites)
    assert st.completed == len(MIX) and st.max_active >= 2
    for r, (status, res, sb, rb) in zip(MIX, mixed):
        assert status == jw.OK
        (s1, res1, sb1, rb1), = run(jw, [r], precision=precision, max_steps_per_tick=3)[0]
        assert s1 == jw.OK
        assert np.array_equal(sb, sb1), r           # bitwise: events never interact
        assert res.Qs == res1.Qs


def test_served_sr_matches_fp64_oracle(jw, oracle):
    N, steps, seed = 32, 20, 77
    (status, res, sb, rb), = run(jw, [dict(N=N, steps=steps, seed=seed, coupling=3)], precision=1)[0]
    assert status == jw.OK
    V = oracle.evolve_momentum(oracle.initial_condition(N, 0.5 * N, 0.04, 6, seed), steps, 0, 0.0004, 3, 1, seed)
    corr, _, _ = oracle.measure(V)
    _, Sb, Rb, _, qs = oracle.dipole(corr)
    assert np.abs(sb - Sb).max() < 1e-5
    assert np.abs(rb - Rb).max() < 1e-12
    if qs > 0:
        assert abs(res.Qs - qs) / qs < 1e-4


def test_admission_under_a_tight_budget(jw):
    per = 256 * 256 * (144 + 32 + 192)
    reqs = [dict(N=256, steps=6, seed=30 + i, coupling=3) for i in range(5)]
    out, st = run(jw, reqs, precision=1, max_bytes=int(2.5 * per))  # two fit, three do not
    assert all(o[0] == jw.OK for o in out)
    assert st.max_active <= 2
