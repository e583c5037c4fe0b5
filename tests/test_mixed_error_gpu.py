"""Mixed-precision error at the sizes and step counts the throughput is quoted
on, against the FP64 engine (itself pinned to the reference's V at 1e-12 by
test_engine_gpu.py and test_dropin_gpu.py).

* 4 events x 512^2, MV with Ny = 50, g^2 mu a = 0.5, m a = 0.02, 1000 steps,
  running (SQRT) coupling with step = ds/pi^2 and fixed coupling with
  step = alpha_s ds/pi^2 (alpha_s = 0.15, ds = 1e-4): the batched workload.
* one event per N in {128, 256, 1024} at 2000 steps, the longest run of the
  uneven batch, couplings mixed.
* one 2048^2 event with Ny = 100, g^2 mu a = 0.8, 2000 steps: the largest
  request of the serving mix.

Bars (the mixed form's stated tolerances): max |dS(r)| <= 1e-5 per event and
for the ensemble mean, |dQ_s|/Q_s <= 1e-4, unitarity drift of the mixed V
(reunitarised every step) <= 1e-13."""
import math

import pytest

pytestmark = pytest.mark.gpu

DS, ALPHA_S, MASS = 1e-4, 0.15, 0.04
TOL_SR = 1e-5
TOL_QS = 1e-4
TOL_DRIFT = 1e-13


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def spec(jw, N, steps, seed, coupling="sqrt", ny=50, g2mu=0.5):
    c = jw.SQRT_COUPLING_CONSTANT if coupling == "sqrt" else jw.FIXED_COUPLING_CONSTANT
    step = DS / math.pi ** 2 if coupling == "sqrt" else ALPHA_S * DS / math.pi ** 2
    return dict(N=N, ny_slices=ny, mu=g2mu * N, mass=MASS, step=step, coupling=c, seed=seed, steps=steps)


def check(res):
    assert res["status"] == (0, 0)
    for e in res["per_event"]:
        assert e["dS_max"] <= TOL_SR, e
        assert e["Qs_rel_err"] <= TOL_QS, e
        assert e["drift_mixed"] <= TOL_DRIFT, e
    for n, e in res["ensembles"].items():
        assert e["dS_max"] <= TOL_SR, (n, e)
        assert e["Qs_rel_err"] <= TOL_QS, (n, e)


@pytest.mark.parametrize("coupling", ["sqrt", "fixed"])
def test_mixed_error_512_batch_1000_steps(jw, coupling):
    from jimwlk.precision import compare_mixed_fp64
    res = compare_mixed_fp64(jw, [spec(jw, 512, 1000, 7000 + i, coupling) for i in range(4)])
    check(res)
    print(coupling, {k: res[k] for k in ("dS_max", "Qs_rel_err_max", "drift_mixed_max", "drift_fp64_max")})


def test_mixed_error_uneven_sizes_2000_steps(jw):
    from jimwlk.precision import compare_mixed_fp64
    specs = [spec(jw, 128, 2000, 81, "fixed"), spec(jw, 256, 2000, 82, "sqrt"), spec(jw, 1024, 2000, 83, "fixed")]
    check(compare_mixed_fp64(jw, specs))


def test_mixed_error_largest_served_request(jw):
    from jimwlk.precision import compare_mixed_fp64
    check(compare_mixed_fp64(jw, [spec(jw, 2048, 2000, 91, "fixed", ny=100, g2mu=0.8)]))
