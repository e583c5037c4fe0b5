"""GPU tests of the engine's ensemble measurement (jw_engine_measure_ensemble,
jw_engine_step_measure_ensemble): the statistics reduction of
main_optimized.cpp:317-336 over events, checked against the reference's own
per-event values, against the engine's per-event measurements, and the one-call
step + measurement against the two calls it replaces."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUPLING = {"FIXED": 3, "NOISE_COUPLING_CONSTANT": 1, "SQRT_COUPLING_CONSTANT": 0}


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def event_from(eng, fx):
    return eng.add_event(int(fx["N"]), ny_slices=int(fx["slices"]), mu=float(fx["mu"]), mass=float(fx["mass"]),
                         step=float(fx["step"]), coupling=COUPLING[str(fx["coupling"])], seed=int(fx["seed"]))


def test_fp64_ensemble_matches_reference(jw, gold):
    """Two 16^2 events (NOISE and SQRT coupling): the ensemble sums are the
    sums of the reference's per-event reduce outputs (field.h:1521-1536)."""
    fxs = [gold("evolve_noise_N16"), gold("evolve_sqrt_N16")]
    assert int(fxs[0]["steps"]) == int(fxs[1]["steps"])
    eng = jw.Engine(precision=jw.PRECISION_FP64)
    ids = [event_from(eng, fx) for fx in fxs]
    eng.init_mv(ids)
    eng.step(ids, int(fxs[0]["steps"]))
    s, e = eng.measure_ensemble(ids)
    ref_s = fxs[0]["sum"] + fxs[1]["sum"]
    ref_e = fxs[0]["err"] + fxs[1]["err"]
    assert np.abs(s - ref_s).max() < 1e-11 * np.abs(ref_s).max()
    assert np.abs(e - ref_e).max() < 1e-11 * np.abs(ref_e).max()
    assert np.all(s.imag == 0) and np.all(e.imag == 0)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_ensemble_is_sum_of_event_measurements(jw, precision):
    """sum = sum over events of the symmetrised correlator, err = sum of its
    square: the per-event accumulators after one measurement hold exactly those."""
    prec = jw.PRECISION_MIXED if precision == "mixed" else jw.PRECISION_FP64
    eng = jw.Engine(precision=prec, max_batch=2)
    ids = [eng.add_event(64, ny_slices=4, mu=32.0, mass=0.04, step=1e-3, coupling=jw.FIXED_COUPLING_CONSTANT,
                         seed=100 + i) for i in range(5)]
    eng.init_mv(ids)
    eng.step(ids, 3)
    s, e = eng.measure_ensemble(ids)
    eng.measure(ids)
    ps = np.zeros_like(s)
    pe = np.zeros_like(e)
    for i in ids:
        a, b, n = eng.correlator(i)
        assert n == 1
        ps += a
        pe += b
    assert np.abs(s - ps).max() <= 1e-13 * np.abs(ps).max()
    assert np.abs(e - pe).max() <= 1e-13 * np.abs(pe).max()


@pytest.mark.parametrize("precision,N,events,max_batch", [
    ("mixed", 64, 5, 2),      # fused, three launch groups
    ("mixed", 512, 3, 0),     # fused
    ("mixed", 1024, 2, 0),    # fused
    ("mixed", 2048, 1, 0),    # fused, one CTA per SM; pass 1 as a two-CTA cluster
    ("fp64", 64, 3, 0),       # FP64 engine: step, then the FP64 measurement
])
def test_step_measure_ensemble_same_as_two_calls(jw, precision, N, events, max_batch):
    """One call (step + ensemble measurement) gives bit for bit what the two
    calls give, on two calls in a row, into pageable and page-locked arrays."""
    import torch
    prec = jw.PRECISION_MIXED if precision == "mixed" else jw.PRECISION_FP64

    def make():
        eng = jw.Engine(precision=prec, max_batch=max_batch)
        ids = [eng.add_event(N, ny_slices=2, mu=0.5 * N, mass=0.04, step=1e-3,
                             coupling=jw.FIXED_COUPLING_CONSTANT, seed=7 + i) for i in range(events)]
        eng.init_mv(ids)
        return eng, ids

    a, ida = make()
    b, idb = make()
    pin_s = torch.empty((N, N), dtype=torch.complex128, pin_memory=True).numpy()
    pin_e = torch.empty((N, N), dtype=torch.complex128, pin_memory=True).numpy()
    for k, nsteps in enumerate((2, 1)):
        a.step(ida, nsteps)
        sa, ea = a.measure_ensemble(ida)
        if k == 0:
            sb, eb = b.step_measure_ensemble(idb, nsteps)
        else:
            sb, eb = b.step_measure_ensemble(idb, nsteps, pin_s, pin_e)
        assert a.sync() == jw.OK and b.sync() == jw.OK
        assert np.array_equal(sa, sb) and np.array_equal(ea, eb)
        assert np.abs(sa).max() > 0
    for i, j in zip(ida, idb):
        assert np.array_equal(a.get_V(i), b.get_V(j))
        assert a.steps_taken(i) == b.steps_taken(j) == 3
    a.close()
    b.close()
