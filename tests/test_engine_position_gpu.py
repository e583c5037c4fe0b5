"""GPU tests of position-space events in the batched engine: FP64 parity with
the reference's position fixtures (SQRT coupling, SIN kernel), FIXED and
HATTA couplings against the oracle's direct sum, mixed-precision error, the
noise offset step0, batches of Hatta branches (one rr per event) and the
single-site correlator read-back."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SQRT, NOISE, HATTA, FIXED = 0, 1, 2, 3
TOL_V64 = 1e-12
TOL_V32 = 2e-5


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def pos_event(eng, N, seed, coupling, rr=0, step=0.0004, slices=6, step0=0, kernel=1):
    return eng.add_event(N, ny_slices=slices, mu=0.5 * N, mass=0.04, step=step, coupling=coupling, seed=seed,
                         position_space=True, rr=rr, step0=step0, kernel=kernel)


def test_fp64_position_engine_matches_reference(jw, gold):
    fx = gold("position_sqrt_sin_N16")
    eng = jw.Engine(precision=jw.PRECISION_FP64)
    eid = eng.add_event(16, ny_slices=int(fx["slices"]), mu=float(fx["mu"]), mass=float(fx["mass"]),
                        step=float(fx["step"]), coupling=SQRT, seed=int(fx["seed"]), position_space=True)
    eng.init_mv([eid])
    assert np.abs(eng.get_V(eid) - fx["V_mv"]).max() < TOL_V64
    eng.step([eid], int(fx["steps"]))
    assert np.abs(eng.get_V(eid) - fx["V_final"]).max() < TOL_V64
    assert eng.sync() == jw.OK


@pytest.mark.parametrize("coupling,rr", [(SQRT, 0), (HATTA, 40)])
def test_fp64_position_engine_matches_call_for_call_at_256(jw, coupling, rr):
    """At C2's lattice size (256^2), where the CPU oracle cannot run, the FP64
    position engine against the call-for-call position path (jw_evolve_position,
    prepare_A_and_B + update_uf in the reference's call order), which the
    reference's own fixtures pin at 16^2: the same MV initial condition and
    steps give the same V to 1e-12."""
    N, seed, steps, step = 256, 29, 4, 0.0004
    eng = jw.Engine(precision=jw.PRECISION_FP64)
    eid = pos_event(eng, N, seed, coupling, rr=rr, step=step, slices=2)
    eng.init_mv([eid])
    V0 = eng.get_V(eid)
    eng.step([eid], steps)
    got = eng.get_V(eid)
    assert eng.sync() == jw.OK
    eng.close()
    ctx = jw.Context(jw.config_defaults(Nx=N, Ny=N, seed=seed, mu=0.5 * N, mass=0.04, elementaryWilsonLines=2,
                                        step=step, CouplingChoice=coupling, KernelChoice=jw.SIN_KERNEL))
    V = ctx.field()
    V.set(V0)
    ctx.evolve_position(V, 0, steps, rr=rr)
    want = V.get()
    assert ctx.sync() == jw.OK
    ctx.close()
    assert np.abs(want - V0).max() > 1e-6  # the steps moved V
    assert np.abs(got - want).max() < TOL_V64


@pytest.mark.parametrize("coupling,rr", [(FIXED, 0), (HATTA, 5), (HATTA, 0), (SQRT, 0)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_position_engine_matches_oracle(jw, oracle, coupling, rr, precision):
    N, seed, steps, step = 32, 17, 6, 0.0004
    eng = jw.Engine(precision=jw.PRECISION_FP64 if precision == "fp64" else jw.PRECISION_MIXED)
    eid = pos_event(eng, N, seed, coupling, rr=rr, step=step, step0=3)
    eng.init_mv([eid])
    V0 = eng.get_V(eid)
    eng.step([eid], steps)
    assert eng.steps_taken(eid) == 3 + steps
    want = oracle.evolve_position(V0, steps, 3, step, coupling, 1, rr, None, seed)
    tol = TOL_V64 if precision == "fp64" else TOL_V32
    assert np.abs(eng.get_V(eid) - want).max() < tol
    assert eng.sync() == jw.OK


@pytest.mark.parametrize("coupling,rr", [(SQRT, 0), (HATTA, 5), (FIXED, 0)])
@pytest.mark.parametrize("precision,N", [("fp64", 32), ("mixed", 32), ("mixed", 64)])
def test_linear_kernel_position_engine_matches_oracle(jw, oracle, coupling, rr, precision, N):
    """The LINEAR position kernel (positions.h:105-150 with the unwrapped
    distance) in the engine: its DFT has a real part (k_i(d) is not odd at
    d_i = -N/2), carried in the event's real-part tables, against the oracle's
    direct sum (field.h:2368-2519).  At 64^2 the mixed engine's column pass is
    the persistent TMA form."""
    seed, steps, step = 19, 5, 0.0004
    eng = jw.Engine(precision=jw.PRECISION_FP64 if precision == "fp64" else jw.PRECISION_MIXED)
    eid = pos_event(eng, N, seed, coupling, rr=rr, step=step, step0=2, kernel=0)
    eng.init_mv([eid])
    V0 = eng.get_V(eid)
    eng.step([eid], steps)
    want = oracle.evolve_position(V0, steps, 2, step, coupling, 0, rr, None, seed)
    tol = TOL_V64 if precision == "fp64" else TOL_V32
    assert np.abs(eng.get_V(eid) - want).max() < tol
    assert eng.sync() == jw.OK


def test_hatta_branches_batched(jw, oracle):
    """The Hatta loop's branches (main_optimized.cpp:200-216): one event per
    (ix, iy), each with its own rr and noise offset, stepped in one batch, then
    measured and read back at its own (ix, iy) -- against each branch alone."""
    N, seed, steps = 16, 23, 4
    branches = []
    for ix in range(N):
        for iy in range(ix - 1, ix + 2):
            if 0 <= iy < N:
                dix = ix - N if ix >= N // 2 else ix
                diy = iy - N if iy >= N // 2 else iy
                branches.append((ix, iy, dix * dix + diy * diy))
    eng = jw.Engine(precision=jw.PRECISION_FP64)
    base = pos_event(eng, N, seed, HATTA, rr=0)
    eng.init_mv([base])
    V0 = eng.get_V(base)
    ids = []
    for b, (ix, iy, rr) in enumerate(branches):
        eid = pos_event(eng, N, seed, HATTA, rr=rr, step0=b * steps)
        eng.copy_V(eid, base)
        ids.append(eid)
    eng.step(ids, steps)
    eng.measure(ids)
    s, e = eng.correlator_at(ids, [b[0] for b in branches], [b[1] for b in branches])
    for k in (0, len(branches) // 2, len(branches) - 1):
        ix, iy, rr = branches[k]
        want = oracle.evolve_position(V0, steps, k * steps, 0.0004, HATTA, 1, rr, None, seed)
        assert np.abs(eng.get_V(ids[k]) - want).max() < TOL_V64
        full, full_err, _ = eng.correlator(ids[k])
        assert s[k] == full[ix, iy].real and e[k] == full_err[ix, iy].real
        c, _, _ = oracle.measure(want)
        assert abs(s[k] - c[ix, iy].real) <= 1e-12 * abs(c).max()
    eng.reset_correlators(ids)
    s, e = eng.correlator_at(ids, [b[0] for b in branches], [b[1] for b in branches])
    assert not s.any() and not e.any()


def test_position_engine_rejects_what_it_cannot_do(jw):
    eng = jw.Engine(precision=jw.PRECISION_MIXED)
    st, _ = eng.try_add_event(N=16, coupling=NOISE, position_space=True)   # needs the Cholesky factor
    assert st == jw.EUNSUPPORTED
    st, _ = eng.try_add_event(N=16, coupling=SQRT, kernel=0)               # LINEAR kernel in momentum space
    assert st == jw.EUNSUPPORTED
    st, _ = eng.try_add_event(N=16, coupling=HATTA)                        # HATTA in momentum space
    assert st == jw.EUNSUPPORTED
