"""GPU parity of position-space evolution (jw_prepare_A_and_B,
jw_set_correlations_for_coupling_constant, jw_cholesky_decompose,
jw_multiply_by_cholesky, jw_reduce_hatta, jw_evolve_position) against the
reference's golden vectors (tests/golden/position_*.npz, produced by the
reference's own prepare_A_and_B_local, gmatrix::decompose and
multiplyByCholesky) and against the oracle.  FP64 tolerances: 1e-13 relative
for single applications, 1e-12 absolute on V after an evolution."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUPLING = {"SQRT_COUPLING_CONSTANT": 0, "NOISE_COUPLING_CONSTANT": 1}
HATTA = 2
POSITION_FIXTURES = ["position_sqrt_sin_N16", "position_sqrt_linear_N8", "position_cholesky_N8",
                     "position_cholesky_N16", "position_sqrt_sin_N15", "position_cholesky_N10",
                     "position_cholesky_N12"]


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def ctx_for(jw, N, seed, step, coupling, kernel):
    return jw.Context(jw.config_defaults(Nx=N, Ny=N, seed=seed, step=step, EvolutionChoice=0,
                                         CouplingChoice=coupling, KernelChoice=kernel))


def fixture_ctx(jw, fx):
    kn = 1 if str(fx["kernel"]) == "SIN_KERNEL" else 0
    cp = COUPLING[str(fx["coupling"])]
    return ctx_for(jw, int(fx["N"]), int(fx["seed"]), float(fx["step"]), cp, kn), cp, kn


def correlation_matrix(corr):
    """S(i, j) = corr(|x_i - x_j|, |y_i - y_j|) (matrix.h:190-196)."""
    N = corr.shape[0]
    x = np.arange(N * N) // N
    y = np.arange(N * N) % N
    return corr[np.abs(x[:, None] - x[None, :]), np.abs(y[:, None] - y[None, :])]


@pytest.mark.parametrize("name", POSITION_FIXTURES)
def test_prepare_A_and_B_matches_reference(jw, gold, name):
    fx = gold(name)
    ctx, cp, kn = fixture_ctx(jw, fx)
    V = ctx.field().set(fx["V_mv"])
    xx, xy = ctx.field(), ctx.field()
    ctx.generate_gaussian(xx, xy, 0, False)
    if cp == 1:
        corr = ctx.field(1)
        ctx.set_correlations_for_coupling_constant(corr)
        ctx.execute2D(corr, 0)
        assert np.abs(corr.get()[..., 0] - fx["chol_corr"]).max() <= 1e-15
        L = ctx.cholesky(corr)
        if "chol_L" in fx:
            assert np.abs(L.get() - fx["chol_L"]).max() <= 1e-13
        ctx.multiply_by_cholesky(xx, L)
        ctx.multiply_by_cholesky(xy, L)
        assert np.abs(xx.get() - fx["xi_x_corr"]).max() <= 1e-13
    A, B = ctx.field(), ctx.field()
    ctx.prepare_A_and_B(A, B, xx, xy, V, 0, cp, kn)
    assert rel(A.get(), fx["A_pos"]) <= 1e-13
    assert rel(B.get(), fx["B_pos"]) <= 1e-13
    assert ctx.sync() == jw.OK


@pytest.mark.parametrize("name", POSITION_FIXTURES)
def test_evolve_position_matches_reference(jw, gold, name):
    fx = gold(name)
    ctx, cp, kn = fixture_ctx(jw, fx)
    V = ctx.field().set(fx["V_mv"])
    L = None
    if cp == 1:
        corr = ctx.field(1)
        ctx.set_correlations_for_coupling_constant(corr)
        ctx.execute2D(corr, 0)
        L = ctx.cholesky(corr)
    ctx.evolve_position(V, 0, int(fx["steps"]), 0, L)
    assert ctx.sync() == jw.OK
    assert np.abs(V.get() - fx["V_final"]).max() <= 1e-12
    Vk, c = ctx.field(), ctx.field(1)
    Vk.copy_from(V)
    ctx.execute2D(Vk, 1)
    ctx.trace(Vk, c)
    ctx.average_and_symmetrize(c)
    assert rel(c.get()[..., 0], fx["corr"]) <= 1e-12


def test_dipole_matches_oracle(jw, gold, oracle):
    """jw_dipole (S(r) bins, Q_s) of the measured correlator against the oracle's definition."""
    fx = gold("position_sqrt_sin_N16")
    ctx, cp, kn = fixture_ctx(jw, fx)
    c = ctx.field(1).set(fx["corr"][..., None])
    Sb, rb, cb, qs, Sxy = ctx.dipole(c, with_xy=True)
    So, Sbo, rbo, cbo, qso = oracle.dipole(fx["corr"])
    assert np.abs(Sxy - So).max() <= 1e-13 and np.abs(Sb - Sbo).max() <= 1e-13
    assert np.array_equal(cb, cbo) and np.abs(rb - rbo).max() <= 1e-13
    assert abs(qs - qso) <= 1e-12 * max(abs(qso), 1.0)


@pytest.mark.parametrize("N,kernel,rr", [(16, 1, 5), (16, 0, 2), (32, 1, 8)])
def test_hatta_matches_oracle(jw, oracle, N, kernel, rr):
    """HATTA coupling: the SQRT formula at min(r2, rr) (the reference's own
    value is uninitialised there), against the oracle's direct sum."""
    seed, step = 31, 0.0004
    ctx = ctx_for(jw, N, seed, step, HATTA, kernel)
    V0 = oracle.initial_condition(N, 0.5 * N, 0.04, 4, seed)
    V = ctx.field().set(V0)
    xx, xy = ctx.field(), ctx.field()
    ctx.generate_gaussian(xx, xy, 0, False)
    A, B = ctx.field(), ctx.field()
    ctx.prepare_A_and_B(A, B, xx, xy, V, rr, HATTA, kernel)
    Ao, Bo = oracle.prepare_A_and_B(xx.get(), xy.get(), V0, rr, HATTA, kernel)
    assert rel(A.get(), Ao) <= 1e-13 and rel(B.get(), Bo) <= 1e-13
    ctx.evolve_position(V, 0, 3, rr)
    assert ctx.sync() == jw.OK
    V1 = oracle.evolve_position(V0, 3, 0, step, HATTA, kernel, rr, None, seed)
    assert np.abs(V.get() - V1).max() <= 1e-12


@pytest.mark.parametrize("N", [32, 64, 10, 12, 24])
def test_cholesky_factor_reproduces_correlation(jw, N):
    """L L^T = S over several 128-row diagonal blocks, and L xi against numpy
    for a 9-component and a 1-component field.  At 10^2, 12^2 and 24^2 the
    order N^2 is padded to the blocking (112, 256, 640) with an identity block."""
    ctx = ctx_for(jw, N, 3, 0.0004, 1, 1)
    corr = ctx.field(1)
    ctx.set_correlations_for_coupling_constant(corr)
    ctx.execute2D(corr, 0)
    c = corr.get()[..., 0]
    L = ctx.cholesky(corr)
    Lh = L.get()
    S = correlation_matrix(c)
    assert np.abs(np.triu(Lh, 1)).max() == 0.0
    rng = np.random.default_rng(N)
    rows = np.sort(rng.choice(N * N, size=min(N * N, 256), replace=False))
    assert np.abs(Lh[rows] @ Lh.T - S[rows]).max() <= 1e-12 * np.abs(S).max()
    for t in (9, 1):
        a = rng.standard_normal((N, N, t)) + 1j * rng.standard_normal((N, N, t))
        f = ctx.field(t).set(a)
        ctx.multiply_by_cholesky(f, L)
        want = (Lh @ a.reshape(N * N, t)).reshape(N, N, t)
        assert rel(f.get(), want) <= 1e-13
    assert ctx.sync() == jw.OK


@pytest.mark.parametrize("N", [16, 32, 12, 24])
def test_cholesky_matches_oracle(jw, oracle, N):
    """The blocked factorisation (diagonal blocks, panel solves, tensor-core
    trailing updates: one panel at 16^2, eight at 32^2) against the oracle's
    column-by-column recurrence (matrix.h:151-200)."""
    ctx = ctx_for(jw, N, 3, 0.0004, 1, 1)
    corr = ctx.field(1)
    ctx.set_correlations_for_coupling_constant(corr)
    ctx.execute2D(corr, 0)
    Lo = oracle.cholesky(oracle.correlations(N))
    assert np.abs(ctx.cholesky(corr).get() - Lo).max() <= 1e-13


def test_reduce_hatta_touches_one_site(jw):
    N = 16
    ctx = ctx_for(jw, N, 3, 0.0004, HATTA, 1)
    rng = np.random.default_rng(7)
    c0 = rng.random((N, N, 1)) + 0.0j
    s0 = rng.standard_normal((N, N, 1)) + 1j * rng.standard_normal((N, N, 1))
    e0 = rng.standard_normal((N, N, 1)) + 1j * rng.standard_normal((N, N, 1))
    c, s, e = ctx.field(1).set(c0), ctx.field(1).set(s0), ctx.field(1).set(e0)
    ctx.reduce_hatta(c, s, e, 3, 4)
    ws, we = s0.copy(), e0.copy()
    ws[3, 4, 0] += c0[3, 4, 0]
    we[3, 4, 0] += c0[3, 4, 0].real ** 2
    assert np.array_equal(s.get(), ws) and np.array_equal(e.get(), we)


def test_position_arguments_are_checked(jw):
    ctx = ctx_for(jw, 16, 3, 0.0004, 1, 1)
    V, xx, xy, A = ctx.field(), ctx.field(), ctx.field(), ctx.field()
    with pytest.raises(jw.JimwlkError):
        ctx.prepare_A_and_B(A, A, xx, xy, V, 0, 0, 1)      # A and B alias
    with pytest.raises(jw.JimwlkError):
        ctx.evolve_position(V, 0, 1, 0, None)              # NOISE coupling needs the factor
