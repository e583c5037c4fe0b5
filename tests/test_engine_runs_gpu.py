"""GPU tests of the engine's multi-step runs.  A call of K mixed-precision steps
runs pass 1, then K - 1 times (pass 2, pass 3 fused with the next pass 1), then
pass 2 and pass 3; K calls of one step never use the fused kernel.  Both must
give bit-identical lattices, as must any split of the steps into calls, the
timed run, and chunked launch groups."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def make(jw, N, events, precision, max_batch=0):
    eng = jw.Engine(precision=precision, max_batch=max_batch)
    ids = [eng.add_event(N, ny_slices=2, mu=0.5 * N, mass=0.04, step=2e-3, coupling=jw.FIXED_COUPLING_CONSTANT,
                         seed=11 + i) for i in range(events)]
    eng.init_mv(ids)
    return eng, ids


@pytest.mark.parametrize("precision,N,events", [
    ("mixed", 64, 3),      # fused pass 3 + 1
    ("mixed", 512, 2),     # fused, two CTAs per SM
    ("mixed", 1024, 1),    # fused, two-CTA clusters
    ("mixed", 2048, 1),    # fused, four-CTA clusters against the two-CTA pass 1 and pass 3
    ("fp64", 64, 2),       # FP64 engine: per-step graph replay
])
def test_split_of_steps_into_calls_is_bitwise_invariant(jw, precision, N, events):
    prec = jw.PRECISION_MIXED if precision == "mixed" else jw.PRECISION_FP64
    splits = {"one call": [7], "single steps": [1] * 7, "3 + 4": [3, 4], "2 + 5": [2, 5]}
    finals = {}
    for name, parts in splits.items():
        eng, ids = make(jw, N, events, prec)
        for k in parts:
            eng.step(ids, k)
        assert eng.sync() == jw.OK
        finals[name] = [eng.get_V(i) for i in ids]
        assert all(eng.steps_taken(i) == 7 for i in ids)
        eng.close()
    # the same 7 steps through the timed run
    eng, ids = make(jw, N, events, prec)
    kernels, total = eng.step_timed(ids, 7)
    assert eng.sync() == jw.OK and total > 0
    finals["timed"] = [eng.get_V(i) for i in ids]
    eng.close()
    ref = finals["one call"]
    assert np.abs(ref[0]).max() > 0
    for name, vs in finals.items():
        for a, b in zip(ref, vs):
            assert np.array_equal(a, b), name
    # launches of the timed run: mixed 1 + 7 + 1 + 6 (pass 1, pass 2, pass 3, pass 3+1)
    counts = {k: c for k, (_, c) in kernels.items()}
    if precision == "mixed":
        assert counts == {"pass1": 1, "pass2": 7, "pass3": 1, "pass31": 6}
    else:
        assert counts == {"pass1": 7, "pass2": 7, "pass3": 7, "pass31": 0}


def test_chunked_launch_groups_match_one_group(jw):
    """max_batch splits the events into launch groups that each run all their
    steps in turn; the lattices equal those of one launch group."""
    a, ida = make(jw, 128, 5, jw.PRECISION_MIXED)
    b, idb = make(jw, 128, 5, jw.PRECISION_MIXED, max_batch=2)
    a.step(ida, 6)
    b.step(idb, 6)
    assert a.sync() == jw.OK and b.sync() == jw.OK
    for i, j in zip(ida, idb):
        assert np.array_equal(a.get_V(i), b.get_V(j))
    a.close()
    b.close()


@pytest.mark.parametrize("N", [64, 512, 1024, 2048])
def test_autotuner_choice_does_not_change_results(jw, N):
    """The autotuner picks a valid column-tile width on the first run of a size,
    and every width gives the same lattice bit for bit."""
    events = {64: 3, 512: 2, 1024: 1, 2048: 1}[N]
    tma = 16 + (8 if N <= 512 else 4)  # the persistent form with tensor-memory-accelerator tile moves
    eng, ids = make(jw, N, events, jw.PRECISION_MIXED)
    eng.step(ids, 4)
    ref = [eng.get_V(i) for i in ids]
    eng.close()
    tuned = jw.Engine(precision=jw.PRECISION_MIXED, autotune=True)
    tids = [tuned.add_event(N, ny_slices=2, mu=0.5 * N, mass=0.04, step=2e-3, coupling=jw.FIXED_COUPLING_CONSTANT,
                            seed=11 + i) for i in range(events)]
    tuned.init_mv(tids)
    assert tuned.tuning(N) == 0
    tuned.step(tids, 4)
    assert tuned.sync() == jw.OK
    chosen = tuned.tuning(N)
    assert chosen in (1, 2, 4, 8, tma)
    for a, i in zip(ref, tids):
        assert np.array_equal(a, tuned.get_V(i))
    assert all(tuned.steps_taken(i) == 4 for i in tids)
    tuned.close()
    widths = [c for c in (1, 2, 4, 8) if c <= N and c * (N // 8) <= 1024 and
              2 * 16 * (N * c + (0 if c >= 8 else (N // 8) * c)) <= 227 * 1024]
    if 64 <= N <= 1024:
        widths.append(tma)
    assert chosen in widths
    for c in widths:
        eng, ids = make(jw, N, events, jw.PRECISION_MIXED)
        eng.set_tuning(N, c)
        eng.step(ids, 4)
        assert eng.sync() == jw.OK
        for a, i in zip(ref, ids):
            assert np.array_equal(a, eng.get_V(i)), c
        eng.close()
    eng, ids = make(jw, N, 1, jw.PRECISION_MIXED)
    with pytest.raises(RuntimeError):
        eng.set_tuning(N, 3)
    eng.close()


@pytest.mark.parametrize("N,events", [(64, 3), (256, 2), (512, 3), (1024, 1)])
def test_persistent_column_pass_is_bitwise_identical(jw, N, events):
    """The persistent column pass (tuning choice 24, or 20 with 4-column tiles at
    1024^2, or 16 for either: tensor-memory-accelerator tile loads and stores,
    per-pass twiddle table) gives the classic column pass's lattices bit for
    bit, over runs long enough for graph replay, with more work items than
    persistent CTAs."""
    eng, ids = make(jw, N, events, jw.PRECISION_MIXED)
    eng.set_tuning(N, 4 if N >= 1024 else 8)  # a classic width
    eng.step(ids, 6)
    ref = [eng.get_V(i) for i in ids]
    eng.close()
    for choice in (16, 24 if N <= 512 else 20):
        eng, ids = make(jw, N, events, jw.PRECISION_MIXED)
        eng.set_tuning(N, choice)
        eng.step(ids, 6)
        assert eng.sync() == jw.OK
        for a, i in zip(ref, ids):
            assert np.array_equal(a, eng.get_V(i)), choice
        eng.close()
    eng, ids = make(jw, 2048, 1, jw.PRECISION_MIXED)
    with pytest.raises(RuntimeError):  # not built at 2048^2
        eng.set_tuning(2048, 16)
    eng.close()


@pytest.mark.parametrize("N,events", [(128, 2), (256, 2), (1024, 1), (2048, 1)])
def test_radix_first_schedule(jw, N, events):
    """The column transforms' radix-first schedule (tuning choices + 32): bit-
    identical among its own tile widths, within FP32 rounding of the default
    schedule, offered to the autotuner only with autotune = 2, and a recorded
    choice replays its lattices bit for bit."""
    widths = [c for c in (1, 2, 4, 8) if c <= N and c * (N // 8) <= 1024 and
              2 * 16 * (N * c + (0 if c >= 8 else (N // 8) * c)) <= 227 * 1024]
    if 64 <= N <= 1024:
        widths.append(16 + (8 if N <= 512 else 4))
    eng, ids = make(jw, N, events, jw.PRECISION_MIXED)
    eng.step(ids, 4)
    ref0 = [eng.get_V(i) for i in ids]
    eng.close()
    ref1 = None
    for c in widths:
        eng, ids = make(jw, N, events, jw.PRECISION_MIXED)
        eng.set_tuning(N, c + 32)
        eng.step(ids, 4)
        assert eng.sync() == jw.OK
        got = [eng.get_V(i) for i in ids]
        eng.close()
        if ref1 is None:
            ref1 = got
            moved = max(float(np.abs(a - b).max()) for a, b in zip(got, ref0))
            # another rounding: within the mixed form's V tolerance (2e-5) of the default schedule
            assert 0.0 < moved < 2e-5, moved
        for a, b in zip(ref1, got):
            assert np.array_equal(a, b), c
    tuned = jw.Engine(precision=jw.PRECISION_MIXED, autotune=2)
    tids = [tuned.add_event(N, ny_slices=2, mu=0.5 * N, mass=0.04, step=2e-3, coupling=jw.FIXED_COUPLING_CONSTANT,
                            seed=11 + i) for i in range(events)]
    tuned.init_mv(tids)
    tuned.step(tids, 4)
    assert tuned.sync() == jw.OK
    chosen = tuned.tuning(N)
    assert chosen in widths + [c + 32 for c in widths]
    want = ref1 if chosen >= 32 else ref0
    for a, i in zip(want, tids):
        assert np.array_equal(a, tuned.get_V(i))
    tuned.close()
    eng, ids = make(jw, 512, 1, jw.PRECISION_MIXED)  # 512 = 8^3 has no radix-first schedule
    with pytest.raises(RuntimeError):
        eng.set_tuning(512, 8 + 32)
    eng.close()


@pytest.mark.parametrize("N", [64, 256])
def test_events_with_different_tables_share_a_launch(jw, N):
    """Events of one size with different kernel tables in one launch group --
    momentum-space couplings (one table per coupling) and position-space events
    (a table per event, HATTA with different rr, SIN and LINEAR kernels) -- give
    each event's lattice bit for bit as when it runs alone.  The persistent
    column pass keeps a tile's table values across the work items of one table
    only."""
    descs = [dict(coupling=jw.SQRT_COUPLING_CONSTANT), dict(coupling=jw.FIXED_COUPLING_CONSTANT),
             dict(coupling=jw.SQRT_COUPLING_CONSTANT), dict(coupling=jw.FIXED_COUPLING_CONSTANT),
             dict(coupling=jw.HATTA_COUPLING_CONSTANT, position_space=True, rr=3),
             dict(coupling=jw.HATTA_COUPLING_CONSTANT, position_space=True, rr=40),
             dict(coupling=jw.SQRT_COUPLING_CONSTANT, position_space=True, kernel=jw.LINEAR_KERNEL)]

    def add(eng, i, d):
        return eng.add_event(N, ny_slices=2, mu=0.5 * N, mass=0.04, step=4e-4, seed=31 + i, **d)

    eng = jw.Engine(precision=jw.PRECISION_MIXED)
    ids = [add(eng, i, d) for i, d in enumerate(descs)]
    eng.init_mv(ids)
    eng.step(ids, 5)
    assert eng.sync() == jw.OK
    together = [eng.get_V(i) for i in ids]
    eng.close()
    for i, d in enumerate(descs):
        one = jw.Engine(precision=jw.PRECISION_MIXED)
        eid = add(one, i, d)
        one.init_mv([eid])
        one.step([eid], 5)
        assert one.sync() == jw.OK
        assert np.array_equal(one.get_V(eid), together[i]), d
        one.close()
