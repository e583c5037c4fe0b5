"""Checkpoints (no reference counterpart): an engine event saved mid-run and
loaded into a fresh engine continues bit for bit (V, noise index,
accumulators), for a momentum-space and a position-space Hatta event; a
device field survives a save/load round trip and refuses a file of another
size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("kind", ["momentum", "hatta"])
def test_event_resumes_bit_for_bit(jw, tmp_path, precision, kind):
    prec = jw.PRECISION_MIXED if precision == "mixed" else jw.PRECISION_FP64
    kw = dict(ny_slices=8, mu=32.0, mass=0.04, step=1.5e-6, seed=77)
    if kind == "momentum":
        kw.update(coupling=jw.FIXED_COUPLING_CONSTANT)
    else:
        kw.update(coupling=jw.HATTA_COUPLING_CONSTANT, position_space=True, rr=9, step0=40)
    a = jw.Engine(precision=prec)
    ea = a.add_event(64, **kw)
    a.init_mv([ea])
    a.step([ea], 5)
    a.measure([ea])
    path = str(tmp_path / "event.jwck")
    a.save_event(ea, path)
    a.step([ea], 5)
    a.measure([ea])
    Va, (sa, erra, na), steps_a = a.get_V(ea), a.correlator(ea), a.steps_taken(ea)

    b = jw.Engine(precision=prec)
    eb = b.load_event(path)
    assert b.steps_taken(eb) == steps_a - 5
    b.step([eb], 5)
    b.measure([eb])
    Vb, (sb, errb, nb), steps_b = b.get_V(eb), b.correlator(eb), b.steps_taken(eb)
    assert steps_b == steps_a and nb == na == 2
    assert np.array_equal(Va, Vb)
    assert np.array_equal(sa, sb) and np.array_equal(erra, errb)
    assert a.sync() == jw.OK and b.sync() == jw.OK


def test_field_roundtrip(jw, tmp_path):
    ctx = jw.Context(jw.config_defaults(Nx=32, Ny=32))
    rng = np.random.default_rng(3)
    a = rng.standard_normal((32, 32, 9)) + 1j * rng.standard_normal((32, 32, 9))
    f = ctx.field().set(a)
    path = str(tmp_path / "V.jwf")
    f.save(path)
    g = ctx.field().load(path)
    assert np.array_equal(g.get(), a)
    other = jw.Context(jw.config_defaults(Nx=16, Ny=16))
    with pytest.raises(jw.JimwlkError):
        other.field().load(path)
    with pytest.raises(jw.JimwlkError):
        ctx.field(1).load(path)
