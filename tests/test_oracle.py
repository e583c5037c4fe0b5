"""The oracle (oracle/jw_oracle.c) against the reference's golden vectors and
against the reference's own code where it is built here, plus the invariants
the reference's test drivers probe (tests/*.cpp of the reference)."""
import os

import numpy as np
import pytest

from jwref import Reference, config_text, f32, reference_available

FIXED_COUPLING = 3
COUPLING = {"FIXED": FIXED_COUPLING, "NOISE_COUPLING_CONSTANT": 1, "SQRT_COUPLING_CONSTANT": 0}


@pytest.mark.parametrize("name", ["evolve_noise_N16", "evolve_sqrt_N16", "evolve_linear_N16", "evolve_fixed_N32",
                                  "c1_N64", "evolve_sqrt_N24", "evolve_noise_N15"])
def test_oracle_matches_golden_evolution(oracle, gold, name):
    fx = gold(name)
    N, seed = int(fx["N"]), int(fx["seed"])
    V0 = oracle.initial_condition(N, float(fx["mu"]), float(fx["mass"]), int(fx["slices"]), seed)
    assert np.abs(V0 - fx["V_mv"]).max() <= 1e-13
    kn = 1 if str(fx["kernel"]) == "SIN_KERNEL" else 0
    V1 = oracle.evolve_momentum(V0, int(fx["steps"]), 0, float(fx["step"]), COUPLING[str(fx["coupling"])], kn, seed)
    assert np.abs(V1 - fx["V_final"]).max() <= 1e-13
    corr, s, e = oracle.measure(V1)
    assert np.abs(corr - fx["corr"]).max() <= 1e-13 * np.abs(fx["corr"]).max()
    assert np.abs(e - fx["err"]).max() <= 1e-13 * np.abs(fx["err"]).max()


@pytest.mark.parametrize("name", ["functions_N16", "functions_N24", "functions_N15"])
def test_oracle_matches_golden_functions(oracle, gold, name):
    """One application of each hot-path function; 24 and 15 are sizes that
    are not powers of two (the reference plans FFTW for any N)."""
    fx = gold(name)
    N, seed = int(fx["N"]), int(fx["seed"])
    assert np.abs(oracle.execute2D(fx["fft_in"], 1) - fx["fft_fwd"]).max() <= 1e-13
    assert np.abs(oracle.execute2D(fx["fft_in"], 0) - fx["fft_bwd"]).max() <= 1e-13
    z = oracle.langevin_normals(seed, 0, N)
    xx, xy = oracle.generate_gaussian(z, False)
    assert np.array_equal(xx, fx["xi_x"]) and np.array_equal(xy, fx["xi_y"])
    xx, xy = oracle.generate_gaussian(z, True)
    assert np.abs(xx - fx["xi_x_nc"]).max() <= 1e-15 and np.abs(xy - fx["xi_y_nc"]).max() <= 1e-15
    for cp, cname in ((0, "sqrt"), (1, "noise")):
        for k, kname in ((0, "linear"), (1, "sin")):
            a = oracle.prepare_A_local(fx["xi_x_k"], fx["xi_y_k"], cp, k)
            ref = fx[f"A_{cname}_{kname}"]
            assert np.abs(a - ref).max() <= 1e-13 * np.abs(ref).max()
    ux, uy = oracle.uxiulocal(fx["V_mv"], fx["xi_x"], fx["xi_y"])
    assert np.abs(ux - fx["ux"]).max() <= 1e-14 and np.abs(uy - fx["uy"]).max() <= 1e-14
    V = oracle.update_uf(fx["V_mv"], fx["B_x"], fx["A_x"], float(fx["step"]))
    assert np.abs(V - fx["V_upd"]).max() <= 1e-14


@pytest.mark.parametrize("name", ["position_sqrt_sin_N16", "position_sqrt_linear_N8", "position_cholesky_N8",
                                  "position_cholesky_N16", "position_sqrt_sin_N15", "position_cholesky_N10",
                                  "position_cholesky_N12"])
def test_oracle_matches_golden_position(oracle, gold, name):
    """Position-space evolution (main_optimized.cpp:271-304) with Cholesky-
    correlated noise for NOISE coupling (main_optimized.cpp:145-157)."""
    fx = gold(name)
    N, seed = int(fx["N"]), int(fx["seed"])
    cp = COUPLING[str(fx["coupling"])]
    kn = 1 if str(fx["kernel"]) == "SIN_KERNEL" else 0
    L = None
    z0 = oracle.langevin_normals(seed, 0, N)
    xx, xy = oracle.generate_gaussian(z0, False)
    if cp == 1:
        corr = oracle.correlations(N)
        assert np.abs(corr - fx["chol_corr"]).max() <= 1e-15
        L = oracle.cholesky(corr)
        if "chol_L" in fx:
            assert np.abs(L - fx["chol_L"]).max() <= 1e-13
        xx = oracle.multiply_by_cholesky(L, xx)
        assert np.abs(xx - fx["xi_x_corr"]).max() <= 1e-13
        xy = oracle.multiply_by_cholesky(L, xy)
    A, B = oracle.prepare_A_and_B(xx, xy, fx["V_mv"], 0, cp, kn)
    assert np.abs(A - fx["A_pos"]).max() <= 1e-13 * np.abs(fx["A_pos"]).max()
    assert np.abs(B - fx["B_pos"]).max() <= 1e-13 * np.abs(fx["B_pos"]).max()
    V1 = oracle.evolve_position(fx["V_mv"], int(fx["steps"]), 0, float(fx["step"]), cp, kn, 0, L, seed)
    assert np.abs(V1 - fx["V_final"]).max() <= 1e-13
    c, _, _ = oracle.measure(V1)
    assert np.abs(c - fx["corr"]).max() <= 1e-13 * np.abs(fx["corr"]).max()


def test_cholesky_reconstructs_correlation(oracle):
    """L L^T equals the site-site correlation matrix (main_optimized.cpp:145-157
    factorises it so that L xi has that covariance)."""
    N = 8
    corr = oracle.correlations(N)
    L = oracle.cholesky(corr)
    V = N * N
    S = np.empty((V, V), np.complex128)
    for i in range(V):
        for j in range(V):
            S[i, j] = corr[abs(i // N - j // N), abs(i % N - j % N)]
    assert np.abs(np.triu(L, 1)).max() == 0.0
    assert np.abs(L @ L.T - S).max() <= 1e-12 * np.abs(S).max()


@pytest.mark.skipif(not reference_available(8), reason="reference harness not built (needs the reference tree)")
def test_oracle_bitwise_vs_reference_N8(oracle):
    N, seed = 8, 5
    r = Reference(N, config_text(mu=4.0, mass=0.04, wilson_lines=4, step=0.0004,
                                 coupling="SQRT_COUPLING_CONSTANT"))
    c = r.config()
    V0 = oracle.initial_condition(N, c["mu"], c["mass"], 4, seed)
    Vr = r.initial_condition(np.concatenate([oracle.mv_normals(seed, s, N).ravel() for s in range(4)]))
    assert np.array_equal(V0, Vr)
    V1 = oracle.evolve_momentum(V0, 5, 0, c["step"], 0, 1, seed)
    V1r = r.evolve_momentum(Vr, np.concatenate([oracle.langevin_normals(seed, s, N).ravel() for s in range(5)]), 5)
    assert np.array_equal(V1, V1r)


def test_config_parse_is_float_rounded():
    """config.h:84-93 parses mu, mass and step through float."""
    assert f32(0.04) != 0.04 and abs(f32(0.04) - 0.04) < 1e-9


# ---- invariants of the reference's own test drivers ----

def test_fft_delta_and_roundtrip(oracle):
    """tests/test_fftw_execute.cpp:59-72: a delta transforms to 1/sqrt(V)."""
    N = 16
    f = np.zeros((N, N, 1), np.complex128)
    f[0, 0, 0] = 1.0
    g = oracle.execute2D(f, 0)
    assert np.allclose(g, 1.0 / N, atol=1e-16, rtol=0)
    rng = np.random.default_rng(3)
    h = rng.standard_normal((N, N, 9)) + 1j * rng.standard_normal((N, N, 9))
    assert np.abs(oracle.execute2D(oracle.execute2D(h, 1), 0) - h).max() < 1e-14


def test_fft_parseval(oracle):
    """tests/test_fftw_execute_random_std.cpp:76-96: the unitary FFT preserves the norm."""
    rng = np.random.default_rng(4)
    h = rng.standard_normal((32, 32, 1)) + 1j * rng.standard_normal((32, 32, 1))
    assert abs(np.sum(np.abs(oracle.execute2D(h, 1)) ** 2) / np.sum(np.abs(h) ** 2) - 1) < 1e-13


def test_noise_statistics(oracle):
    """tests/test_noise_vectors.cpp:106-137: unit-variance, uncorrelated components."""
    z = np.concatenate([oracle.langevin_normals(9, s, 32).reshape(-1, 16) for s in range(8)])
    assert abs(z.mean()) < 0.01
    assert np.allclose(z.var(axis=0), 1.0, atol=0.03)
    c = np.corrcoef(z.T)
    assert np.abs(c - np.eye(16)).max() < 0.03


def test_exponential_is_unitary(oracle):
    """tests/test_hermitian.cpp:101-150: exp(i H) is unitary with det 1 for traceless H."""
    rng = np.random.default_rng(5)
    for scale in (1e-3, 0.3, 3.0, 30.0):
        n = rng.standard_normal((64, 8)) * scale
        xi, _ = oracle.generate_gaussian(np.repeat(n, 2, axis=1).reshape(8, 8, 16), False)
        m, st = oracle.su3_exponentiate(xi.reshape(-1, 9), 1.0)
        M = m.reshape(-1, 3, 3)
        assert np.all(st == 0)
        assert np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - np.eye(3)).max() < 1e-12
        assert np.abs(np.linalg.det(M) - 1).max() < 1e-11


def test_degenerate_matrix_takes_ql_route(oracle):
    """zheevh3 falls back to QL when eigenvalues are degenerate (su3_matrix.h:318-319)."""
    A = np.diag([1.0, 1.0, -2.0]).astype(np.complex128)
    Q, w, s = oracle.zheevh3(A)
    assert s == 0
    assert np.allclose(sorted(w), [-2, 1, 1], atol=1e-14)
    assert np.abs(Q @ np.diag(w) @ Q.conj().T - A).max() < 1e-14


def test_symmetrize_constant_field(oracle):
    """tests/test_symmetrize_average.cpp:98-136: a constant correlator is unchanged."""
    N = 8
    V = np.zeros((N, N, 9), np.complex128)
    V[..., 0] = V[..., 4] = V[..., 8] = 1.0
    corr, s, e = oracle.measure(V)
    # V = 1 transforms to N at k = 0 only: C(0) = 3 N^2 / N^4
    assert abs(corr[0, 0] - 3.0 / N ** 2) < 1e-15 and np.abs(corr.ravel()[1:]).max() < 1e-15
    assert abs(e[0, 0] - (3.0 / N ** 2) ** 2) < 1e-18


def test_dipole_of_unit_field(oracle):
    """S(r) = 1 everywhere for V = 1; no saturation scale."""
    N = 16
    V = np.zeros((N, N, 9), np.complex128)
    V[..., 0] = V[..., 4] = V[..., 8] = 1.0
    corr, _, _ = oracle.measure(V)
    Sxy, Sb, rb, cb, qs = oracle.dipole(corr)
    assert np.allclose(Sxy, 1.0, atol=1e-13) and qs == 0.0
