"""GPU parity of the call-for-call FP64 layer (jw_execute2D, jw_generate_gaussian,
jw_prepare_A_local, jw_uxiulocal, jw_update_uf, jw_set_mv_model,
jw_solve_poisson, jw_mul_exp, jw_trace, jw_average_and_symmetrize, jw_reduce,
jw_initial_condition, jw_evolve_momentum) against the reference's golden
vectors (tests/golden/, produced by the reference's own code) and against the
oracle.  Tolerances: FP64, element-wise absolute on O(1) fields."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_V = 1e-12       # V after a full evolution, element-wise
TOL_FN = 1e-13      # single function applications


@pytest.fixture(scope="module")
def jw():
    import jimwlk
    return jimwlk


def make_ctx(jw, N, seed=1, **kw):
    return jw.Context(jw.config_defaults(Nx=N, Ny=N, seed=seed, **kw))


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256, 512, 1024, 2048])
def test_execute2D_matches_dft(jw, N):
    ctx = make_ctx(jw, N)
    rng = np.random.default_rng(N)
    t = 9 if N <= 256 else 1
    a = rng.standard_normal((N, N, t)) + 1j * rng.standard_normal((N, N, t))
    f = ctx.field(t).set(a)
    ctx.execute2D(f, 1)
    fwd = f.get()
    assert rel(fwd, np.fft.fft2(a, axes=(0, 1)) / N) < 1e-14 * np.log2(N)
    ctx.execute2D(f, 0)
    assert np.abs(f.get() - a).max() < 1e-14 * np.log2(N) * 4
    assert ctx.sync() == jw.OK


@pytest.mark.parametrize("N", [2, 3, 12, 15, 24, 100, 384, 1000, 1536, 2047])
def test_execute2D_general_n_matches_dft(jw, N):
    """Sizes that are not powers of two: the chirp-z transform (power-of-two
    convolution length M >= 2N - 1) against numpy's DFT, forward and back."""
    ctx = make_ctx(jw, N)
    rng = np.random.default_rng(N)
    t = 9 if N <= 384 else 1
    a = rng.standard_normal((N, N, t)) + 1j * rng.standard_normal((N, N, t))
    f = ctx.field(t).set(a)
    ctx.execute2D(f, 1)
    M = 8
    while M < 2 * N - 1:
        M *= 2
    tol = 1e-14 * np.log2(M)
    assert rel(f.get(), np.fft.fft2(a, axes=(0, 1)) / N) < tol
    ctx.execute2D(f, 0)
    assert np.abs(f.get() - a).max() < 4 * tol
    assert ctx.sync() == jw.OK


def test_context_rejects_unsupported_sizes(jw):
    for N in (1, 2049, 4096):
        with pytest.raises(jw.JimwlkError):
            make_ctx(jw, N)
    with pytest.raises(jw.JimwlkError):
        jw.Context(jw.config_defaults(Nx=24, Ny=16))


@pytest.mark.parametrize("name", ["functions_N16", "functions_N24", "functions_N15"])
def test_functions_match_reference(jw, gold, name):
    """One call of each function against the reference; 24 and 15 are not
    powers of two, so their transforms take the chirp-z form."""
    fx = gold(name)
    N, seed = int(fx["N"]), int(fx["seed"])
    ctx = make_ctx(jw, N, seed=seed)
    f = ctx.field().set(fx["fft_in"])
    ctx.execute2D(f, 1)
    assert np.abs(f.get() - fx["fft_fwd"]).max() < TOL_FN
    f.set(fx["fft_in"])
    ctx.execute2D(f, 0)
    assert np.abs(f.get() - fx["fft_bwd"]).max() < TOL_FN
    xx, xy = ctx.field(), ctx.field()
    ctx.generate_gaussian(xx, xy, 0, False)
    assert np.abs(xx.get() - fx["xi_x"]).max() < 1e-14 and np.abs(xy.get() - fx["xi_y"]).max() < 1e-14
    ctx.generate_gaussian(xx, xy, 0, True)
    assert np.abs(xx.get() - fx["xi_x_nc"]).max() < 1e-14 and np.abs(xy.get() - fx["xi_y_nc"]).max() < 1e-14
    X, Y, A = ctx.field().set(fx["xi_x_k"]), ctx.field().set(fx["xi_y_k"]), ctx.field()
    for cp, cname in ((0, "sqrt"), (1, "noise")):
        for k, kname in ((0, "linear"), (1, "sin")):
            ctx.prepare_A_local(A, X, Y, cp, k)
            assert rel(A.get(), fx[f"A_{cname}_{kname}"]) < TOL_FN
    V = ctx.field().set(fx["V_mv"])
    ux, uy = ctx.field(), ctx.field()
    ctx.uxiulocal(ux, uy, V, ctx.field().set(fx["xi_x"]), ctx.field().set(fx["xi_y"]))
    assert np.abs(ux.get() - fx["ux"]).max() < TOL_FN and np.abs(uy.get() - fx["uy"]).max() < TOL_FN
    ctx.update_uf(V, ctx.field().set(fx["B_x"]), ctx.field().set(fx["A_x"]), float(fx["step"]))
    assert np.abs(V.get() - fx["V_upd"]).max() < TOL_FN
    # measurement chain of main_optimized.cpp:321-334
    Vk = ctx.field().set(fx["V_mv"])
    ctx.execute2D(Vk, 1)
    corr, s, e = ctx.field(1), ctx.field(1), ctx.field(1)
    ctx.trace(Vk, corr)
    ctx.average_and_symmetrize(corr)
    ctx.reduce(corr, s, e)
    assert rel(corr.get()[..., 0], fx["corr"]) < 1e-13
    assert rel(s.get()[..., 0], fx["sum"]) < 1e-13 and rel(e.get()[..., 0], fx["err"]) < 1e-12
    assert ctx.sync() == jw.OK


def test_initial_condition_matches_reference(jw, gold):
    fx = gold("functions_N16")
    N = int(fx["N"])
    ctx = make_ctx(jw, N, seed=int(fx["seed"]), mu=float(fx["mu"]), mass=float(fx["mass"]),
                   elementaryWilsonLines=int(fx["slices"]))
    V = ctx.field()
    ctx.initial_condition(V)
    assert np.abs(V.get() - fx["V_mv"]).max() < TOL_V
    assert ctx.sync() == jw.OK


COUPLING = {"FIXED": 3, "NOISE_COUPLING_CONSTANT": 1, "SQRT_COUPLING_CONSTANT": 0}


@pytest.mark.parametrize("name", ["evolve_noise_N16", "evolve_sqrt_N16", "evolve_linear_N16", "evolve_fixed_N32",
                                  "c1_N64", "evolve_sqrt_N24", "evolve_noise_N15"])
def test_evolution_matches_reference(jw, gold, name):
    """MV initial condition + Langevin steps + one measurement, V element-wise <= 1e-12."""
    fx = gold(name)
    N = int(fx["N"])
    ctx = make_ctx(jw, N, seed=int(fx["seed"]), mu=float(fx["mu"]), mass=float(fx["mass"]),
                   elementaryWilsonLines=int(fx["slices"]), step=float(fx["step"]),
                   CouplingChoice=COUPLING[str(fx["coupling"])],
                   KernelChoice=1 if str(fx["kernel"]) == "SIN_KERNEL" else 0)
    V = ctx.field()
    ctx.initial_condition(V)
    assert np.abs(V.get() - fx["V_mv"]).max() < TOL_V
    ctx.evolve_momentum(V, 0, int(fx["steps"]))
    Vf = V.get()
    assert np.abs(Vf - fx["V_final"]).max() < TOL_V
    ctx.execute2D(V, 1)
    corr, s, e = ctx.field(1), ctx.field(1), ctx.field(1)
    ctx.trace(V, corr)
    ctx.average_and_symmetrize(corr)
    ctx.reduce(corr, s, e)
    assert rel(corr.get()[..., 0], fx["corr"]) < 1e-11
    assert ctx.sync() == jw.OK


def test_evolution_larger_lattice_vs_oracle(jw, oracle):
    """128^2, SQRT running coupling, against the oracle (itself pinned to the reference)."""
    N, seed, steps, step = 128, 21, 4, 0.0004
    ctx = make_ctx(jw, N, seed=seed, mu=0.5 * N, mass=0.04, elementaryWilsonLines=8, step=step,
                   CouplingChoice=0)
    V = ctx.field()
    ctx.initial_condition(V)
    V0 = oracle.initial_condition(N, 0.5 * N, 0.04, 8, seed)
    assert np.abs(V.get() - V0) .max() < TOL_V
    ctx.evolve_momentum(V, 0, steps)
    V1 = oracle.evolve_momentum(V0, steps, 0, step, 0, 1, seed)
    assert np.abs(V.get() - V1).max() < TOL_V
    assert ctx.sync() == jw.OK


def test_unitarity_after_evolution(jw):
    N = 64
    ctx = make_ctx(jw, N, seed=4, mu=32.0, mass=0.04, elementaryWilsonLines=10, step=0.0004)
    V = ctx.field()
    ctx.initial_condition(V)
    ctx.evolve_momentum(V, 0, 20)
    M = V.get().reshape(-1, 3, 3)
    assert np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(M) - 1).max() < 1e-12


def test_bad_arguments_are_rejected(jw):
    ctx = make_ctx(jw, 16)
    a, b = ctx.field(), ctx.field(1)
    with pytest.raises(jw.JimwlkError):
        ctx.uxiulocal(a, a, a, a, a)
    with pytest.raises(jw.JimwlkError):
        ctx.trace(b, a)
    with pytest.raises(jw.JimwlkError):
        ctx.prepare_A_local(a, ctx.field(), ctx.field(), 2, 1)  # HATTA is undefined in momentum space
    with pytest.raises(jw.JimwlkError):
        make_ctx(jw, 4096)  # above the largest lattice
