"""GPU tests of the batched engine (jw_engine_*): FP64 parity with the
reference's golden vectors, mixed-precision error against the FP64 oracle,
batch independence (each event alone == in a mixed batch) and error paths."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUPLING = {"FIXED": 3, "NOISE_COUPLING_CONSTANT": 1, "SQRT_COUPLING_CONSTANT": 0}
TOL_V64 = 1e-12      # FP64 engine, V element-wise
TOL_V32 = 2e-5       # mixed engine, V element-wise after the golden runs
TOL_SR = 1e-5        # mixed engine, dipole S(r) absolute


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def event_from(eng, fx):
    return eng.add_event(int(fx["N"]), ny_slices=int(fx["slices"]), mu=float(fx["mu"]), mass=float(fx["mass"]),
                         step=float(fx["step"]), coupling=COUPLING[str(fx["coupling"])], seed=int(fx["seed"]))


@pytest.mark.parametrize("name", ["evolve_noise_N16", "evolve_sqrt_N16", "evolve_fixed_N32", "c1_N64"])
def test_fp64_engine_matches_reference(jw, gold, name):
    fx = gold(name)
    eng = jw.Engine(precision=jw.PRECISION_FP64)
    eid = event_from(eng, fx)
    eng.init_mv([eid])
    assert np.abs(eng.get_V(eid) - fx["V_mv"]).max() < TOL_V64
    eng.step([eid], int(fx["steps"]))
    assert eng.steps_taken(eid) == int(fx["steps"])
    assert np.abs(eng.get_V(eid) - fx["V_final"]).max() < TOL_V64
    eng.measure([eid])
    s, e, n = eng.correlator(eid)
    assert n == 1
    assert np.abs(s - fx["sum"]).max() < 1e-11 * np.abs(fx["sum"]).max()
    assert np.abs(e - fx["err"]).max() < 1e-11 * np.abs(fx["err"]).max()
    assert eng.sync() == jw.OK


@pytest.mark.parametrize("name", ["evolve_fixed_N32", "c1_N64", "evolve_sqrt_N16"])
def test_mixed_engine_error_vs_fp64(jw, gold, oracle, name):
    fx = gold(name)
    eng = jw.Engine(precision=jw.PRECISION_MIXED)
    eid = event_from(eng, fx)
    eng.init_mv([eid])
    eng.step([eid], int(fx["steps"]))
    V = eng.get_V(eid)
    assert np.abs(V - fx["V_final"]).max() < TOL_V32
    M = V.reshape(-1, 3, 3)
    assert np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - np.eye(3)).max() < 1e-12
    eng.measure([eid])
    s, _, _ = eng.correlator(eid)
    _, Sb, _, _, qs = oracle.dipole(s)
    _, Sb_ref, _, _, qs_ref = oracle.dipole(fx["corr"])
    assert np.abs(Sb - Sb_ref).max() < TOL_SR
    if qs_ref > 0:
        assert abs(qs - qs_ref) / qs_ref < 1e-4


def test_each_event_same_alone_and_in_batch(jw):
    """Events of different sizes and couplings stepped together give bitwise the
    same V as each stepped alone."""
    specs = [dict(N=32, seed=11, coupling=3), dict(N=64, seed=12, coupling=1), dict(N=32, seed=13, coupling=0),
             dict(N=16, seed=14, coupling=3)]
    for prec in (jw.PRECISION_MIXED, jw.PRECISION_FP64):
        alone = []
        for sp in specs:
            eng = jw.Engine(precision=prec)
            eid = eng.add_event(sp["N"], ny_slices=8, step=0.0004, coupling=sp["coupling"], seed=sp["seed"])
            eng.init_mv([eid])
            eng.step([eid], 7)
            alone.append(eng.get_V(eid))
            eng.close()
        eng = jw.Engine(precision=prec)
        ids = [eng.add_event(sp["N"], ny_slices=8, step=0.0004, coupling=sp["coupling"], seed=sp["seed"])
               for sp in specs]
        eng.init_mv(ids)
        eng.step(ids[:2], 3)
        eng.step(ids[2:], 5)
        eng.step(ids[2:], 2)
        eng.step(ids[:2], 4)
        for eid, want in zip(ids, alone):
            assert np.array_equal(eng.get_V(eid), want)
        assert eng.sync() == jw.OK


def test_set_get_roundtrip_and_steps(jw, oracle):
    eng = jw.Engine(precision=jw.PRECISION_FP64)
    eid = eng.add_event(16, ny_slices=4, step=0.0004, coupling=3, seed=5)
    V0 = oracle.initial_condition(16, 8.0, 0.04, 4, 99)
    eng.set_V(eid, V0)
    assert np.array_equal(eng.get_V(eid), V0)
    eng.step([eid], 6)
    want = oracle.evolve_momentum(V0, 6, 0, 0.0004, 3, 1, 5)
    assert np.abs(eng.get_V(eid) - want).max() < TOL_V64
    eng.step([eid], 1)
    want = oracle.evolve_momentum(want, 1, 6, 0.0004, 3, 1, 5)
    assert np.abs(eng.get_V(eid) - want).max() < TOL_V64


def test_reunitarize_keeps_su3(jw):
    eng = jw.Engine(precision=jw.PRECISION_MIXED, reunitarize=True)
    eid = eng.add_event(64, ny_slices=10, step=0.01, coupling=0, seed=3)
    eng.init_mv([eid])
    eng.step([eid], 50)
    M = eng.get_V(eid).reshape(-1, 3, 3)
    assert np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(M) - 1).max() < 1e-13


def test_engine_errors(jw):
    eng = jw.Engine(precision=jw.PRECISION_MIXED, max_bytes=64 << 20)
    st, _ = eng.try_add_event(N=24)
    assert st == jw.EUNSUPPORTED
    st, _ = eng.try_add_event(N=64, kernel=jw.LINEAR_KERNEL)
    assert st == jw.EUNSUPPORTED
    st, _ = eng.try_add_event(N=64, coupling=jw.HATTA_COUPLING_CONSTANT)
    assert st == jw.EUNSUPPORTED
    st, _ = eng.try_add_event(N=2048)  # over the 64 MB budget
    assert st == jw.ENOMEM
    eid = eng.add_event(64)
    with pytest.raises(jw.JimwlkError):
        eng.step([eid, eid], 1)
    with pytest.raises(jw.JimwlkError):
        eng.step([12345], 1)
    eng.remove_event(eid)
    with pytest.raises(jw.JimwlkError):
        eng.step([eid], 1)
