"""Generates the golden vectors in tests/golden/ from the reference's own code.

Run in a container that has the reference tree (for oracle/_ref/libref_<N>.so,
built by `make -C oracle ref`):

    python tests/golden/make_golden.py [fixture names]   # all fixtures when none is named

Every output array below is produced by the reference's functions (field.h,
su3_matrix.h, zheevh3, mpi_fftw_class.h with the project FFT shim) fed with the
engine's Philox noise stream (the oracle's host copy of it, oracle/jw_oracle.c),
so that the GPU tests can check the CUDA library against the reference on a
machine without the reference tree.  The script also checks the oracle against
the same outputs and refuses to write fixtures if they disagree.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from jwref import Oracle, Reference, config_text, f32  # noqa: E402

FIXED = 3  # fixed coupling: plain generate_gaussian + NOISE kernel factor 1


def fixture_functions(o: Oracle, N: int, seed: int) -> dict:
    """One application of each hot-path function at lattice N."""
    cfg = dict(mu=0.5 * N, mass=0.04, wilson_lines=6, step=0.0004, coupling="NOISE_COUPLING_CONSTANT")
    r = Reference(N, config_text(**cfg))
    c = r.config()
    rng = np.random.default_rng(seed)
    out = {"N": N, "seed": seed, "mu": c["mu"], "mass": c["mass"], "step": c["step"], "slices": 6}
    f = rng.standard_normal((N, N, 9)) + 1j * rng.standard_normal((N, N, 9))
    out["fft_in"] = f
    out["fft_fwd"] = r.execute2D(f, 1)
    out["fft_bwd"] = r.execute2D(f, 0)
    z = o.langevin_normals(seed, 0, N)
    out["xi_x"], out["xi_y"] = r.generate_gaussian(z, False)
    out["xi_x_nc"], out["xi_y_nc"] = r.generate_gaussian(z, True)
    X = r.execute2D(out["xi_x"], 1)
    Y = r.execute2D(out["xi_y"], 1)
    out["xi_x_k"], out["xi_y_k"] = X, Y
    for cp, cname in ((0, "sqrt"), (1, "noise")):
        for k, kname in ((0, "linear"), (1, "sin")):
            out[f"A_{cname}_{kname}"] = r.prepare_A_local(X, Y, cp, k)
    V = r.initial_condition(np.concatenate([o.mv_normals(seed, s, N).ravel() for s in range(6)]))
    out["V_mv"] = V
    ux, uy = r.uxiulocal(V, out["xi_x"], out["xi_y"])
    out["ux"], out["uy"] = ux, uy
    A = r.execute2D(out["A_noise_sin"], 0)
    B = r.execute2D(r.prepare_A_local(r.execute2D(ux, 1), r.execute2D(uy, 1), 1, 1), 0)
    out["A_x"], out["B_x"] = A, B
    out["V_upd"] = r.update_uf(V, B, A, c["step"])
    corr, s, e = r.measure(V)
    out["corr"], out["sum"], out["err"] = corr, s, e
    return out


def fixture_evolution(o: Oracle, N: int, seed: int, coupling: str, steps: int, step: float, slices: int,
                      mu: float, mass: float, kernel: str = "SIN_KERNEL") -> dict:
    """MV initial condition then `steps` Langevin steps and one measurement."""
    cfg_coupling = "NOISE_COUPLING_CONSTANT" if coupling == "FIXED" else coupling
    r = Reference(N, config_text(mu=mu, mass=mass, wilson_lines=slices, step=step, coupling=cfg_coupling,
                                 kernel=kernel))
    c = r.config()
    V0 = r.initial_condition(np.concatenate([o.mv_normals(seed, s, N).ravel() for s in range(slices)]))
    zs = np.concatenate([o.langevin_normals(seed, s, N).ravel() for s in range(steps)])
    if coupling == "FIXED":
        V1 = r.evolve_momentum_fixed(V0, zs, steps)
    else:
        V1 = r.evolve_momentum(V0, zs, steps)
    corr, s, e = r.measure(V1)
    return {"N": N, "seed": seed, "mu": c["mu"], "mass": c["mass"], "step": c["step"], "slices": slices,
            "steps": steps, "coupling": coupling, "kernel": kernel, "V_mv": V0, "V_final": V1, "corr": corr,
            "sum": s, "err": e}


def fixture_position(o: Oracle, N: int, seed: int, coupling: str, kernel: str, steps: int, slices: int) -> dict:
    """Position-space evolution (main_optimized.cpp:271-304): MV initial
    condition, `steps` steps with prepare_A_and_B_local and, for NOISE
    coupling, Cholesky-correlated noise (main_optimized.cpp:145-157)."""
    r = Reference(N, config_text(mu=0.5 * N, mass=0.04, wilson_lines=slices, step=0.0004,
                                 evolution="POSITION_EVOLUTION", coupling=coupling, kernel=kernel))
    c = r.config()
    V0 = r.initial_condition(np.concatenate([o.mv_normals(seed, s, N).ravel() for s in range(slices)]))
    out = {"N": N, "seed": seed, "mu": c["mu"], "mass": c["mass"], "step": c["step"], "slices": slices,
           "steps": steps, "coupling": coupling, "kernel": kernel, "V_mv": V0}
    z0 = o.langevin_normals(seed, 0, N)
    xx, xy = o.generate_gaussian(z0, False)
    cp = 1 if coupling == "NOISE_COUPLING_CONSTANT" else 0
    kn = 1 if kernel == "SIN_KERNEL" else 0
    if cp == 1:
        L, corr = r.cholesky_setup()
        out["chol_corr"] = corr
        if N <= 8:
            out["chol_L"] = L
        out["xi_x_corr"] = r.multiply_by_cholesky(xx)
        xx_c, xy_c = out["xi_x_corr"], r.multiply_by_cholesky(xy)
    else:
        xx_c, xy_c = xx, xy
    out["A_pos"], out["B_pos"] = r.prepare_A_and_B(xx_c, xy_c, V0, 0, cp, kn)
    zs = np.concatenate([o.langevin_normals(seed, s, N).ravel() for s in range(steps)])
    V1 = r.evolve_position(V0, zs, steps)
    out["V_final"] = V1
    out["corr"], out["sum"], out["err"] = r.measure(V1)
    return out


DRIVER_RUNS = {
    # name: (N, seed, config fields)
    "driver_sqrt_sin_N16": (16, 41, dict(stat=2, mu=8.0, mass=0.04, wilson_lines=6, langevin_steps=12,
                                         measurements=4, step=0.0004, evolution="MOMENTUM_EVOLUTION",
                                         coupling="SQRT_COUPLING_CONSTANT", kernel="SIN_KERNEL")),
    "driver_noise_sin_N16": (16, 42, dict(stat=1, mu=8.0, mass=0.04, wilson_lines=6, langevin_steps=8,
                                          measurements=2, step=0.0004, evolution="MOMENTUM_EVOLUTION",
                                          coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL")),
    "driver_sqrt_linear_N16": (16, 43, dict(stat=1, mu=8.0, mass=0.04, wilson_lines=6, langevin_steps=6,
                                            measurements=3, step=0.0004, evolution="MOMENTUM_EVOLUTION",
                                            coupling="SQRT_COUPLING_CONSTANT", kernel="LINEAR_KERNEL")),
    "driver_position_cholesky_N16": (16, 44, dict(stat=1, mu=8.0, mass=0.04, wilson_lines=6, langevin_steps=4,
                                                  measurements=2, step=0.0004, evolution="POSITION_EVOLUTION",
                                                  coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL")),
    # a size that is not a power of two (the reference compiles any Nx = Ny)
    "driver_sqrt_sin_N24": (24, 45, dict(stat=1, mu=12.0, mass=0.04, wilson_lines=6, langevin_steps=8,
                                         measurements=2, step=0.0004, evolution="MOMENTUM_EVOLUTION",
                                         coupling="SQRT_COUPLING_CONSTANT", kernel="SIN_KERNEL")),
}


def fixture_driver(o: Oracle, N: int, seed: int, cfg: dict) -> dict:
    """The reference's main_optimized (oracle/_ref/main_optimized_inject_<N>,
    serial, noise injected) on a config, fed the library's noise stream in the
    reference's draw order: per statistics sample the MV slices (stream index
    stat * Ny + i), then the Langevin steps (running index).  Returns the
    config text and the output table it writes."""
    import subprocess
    import tempfile
    exe = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", f"main_optimized_inject_{N}")
    text = config_text(file_name="output", **cfg)
    ny, steps, stats = cfg["wilson_lines"], cfg["langevin_steps"], cfg["stat"]
    chunks, g = [], 0
    for s in range(stats):
        chunks += [o.mv_normals(seed, s * ny + i, N).ravel() for i in range(ny)]
        for _ in range(steps):
            chunks.append(o.langevin_normals(seed, g, N).ravel())
            g += 1
    with tempfile.TemporaryDirectory() as d:
        zf = os.path.join(d, "noise.bin")
        np.concatenate(chunks).astype(np.float64).tofile(zf)
        cf = os.path.join(d, "config")
        with open(cf, "w") as fh:
            fh.write(text)
        r = subprocess.run([exe, "1", "1", cf], cwd=d, capture_output=True, text=True,
                           env=dict(os.environ, JW_INJECT_FILE=zf), timeout=600)
        if r.returncode not in (0, 1):
            raise SystemExit(f"reference main failed ({r.returncode}): {r.stderr[-500:]}")
        with open(os.path.join(d, f"output_optimized_{N}_{N}_mpi1_r0.dat")) as fh:
            dat = fh.read()
    return {"N": N, "seed": seed, "config": text, "dat": dat}


def check_oracle_position(o: Oracle, fx: dict) -> float:
    N, seed = int(fx["N"]), int(fx["seed"])
    cp = 1 if str(fx["coupling"]) == "NOISE_COUPLING_CONSTANT" else 0
    kn = 1 if str(fx["kernel"]) == "SIN_KERNEL" else 0
    L = o.cholesky(o.correlations(N)) if cp == 1 else None
    V1 = o.evolve_position(fx["V_mv"], int(fx["steps"]), 0, float(fx["step"]), cp, kn, 0, L, seed)
    return float(np.abs(V1 - fx["V_final"]).max())


def check_oracle(o: Oracle, fx: dict) -> float:
    N, seed = fx["N"], fx["seed"]
    V0 = o.initial_condition(N, fx["mu"], fx["mass"], fx["slices"], seed)
    cp = {"FIXED": FIXED, "NOISE_COUPLING_CONSTANT": 1, "SQRT_COUPLING_CONSTANT": 0}[fx["coupling"]]
    kn = 1 if fx["kernel"] == "SIN_KERNEL" else 0
    V1 = o.evolve_momentum(V0, fx["steps"], 0, fx["step"], cp, kn, seed)
    corr, _, _ = o.measure(V1)
    return max(np.abs(V0 - fx["V_mv"]).max(), np.abs(V1 - fx["V_final"]).max(),
               np.abs(corr - fx["corr"]).max() / np.abs(fx["corr"]).max())


def main(only: list[str]) -> None:
    """Writes every fixture, or only those named on the command line."""
    o = Oracle()

    def wanted(name: str) -> bool:
        return not only or name in only

    # lattice sizes that are not powers of two: the reference plans FFTW for
    # any N (mpi_fftw_class.h:165-186); 15 is odd, 24 = 2^3 3
    for name, N, seed in (("functions_N16", 16, 101), ("functions_N24", 24, 102), ("functions_N15", 15, 103)):
        if wanted(name):
            fns = fixture_functions(o, N, seed)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k: np.asarray(v) for k, v in fns.items()})
    runs = {
        # reference default main path: MOMENTUM + NOISE coupling (site-indexed noise factor), SIN kernel
        "evolve_noise_N16": dict(N=16, seed=7, coupling="NOISE_COUPLING_CONSTANT", steps=20, step=f32(0.0004),
                                 slices=10, mu=8.0, mass=f32(0.04)),
        # running coupling in momentum space
        "evolve_sqrt_N16": dict(N=16, seed=8, coupling="SQRT_COUPLING_CONSTANT", steps=20, step=f32(0.0004),
                                slices=10, mu=8.0, mass=f32(0.04)),
        # linear kernel (Nyquist rows make A non-Hermitian; exercised on purpose)
        "evolve_linear_N16": dict(N=16, seed=9, coupling="SQRT_COUPLING_CONSTANT", steps=10, step=f32(0.0004),
                                  slices=10, mu=8.0, mass=f32(0.04), kernel="LINEAR_KERNEL"),
        # first workload: 64^2, g^2 mu a = 0.5, m a = 0.02, 50 slices, 100 fixed-coupling steps,
        # step = alpha_s * ds / pi^2 with alpha_s = 0.15, ds = 1e-4
        "c1_N64": dict(N=64, seed=1, coupling="FIXED", steps=100, step=0.15 * 1e-4 / np.pi ** 2, slices=50,
                       mu=32.0, mass=f32(0.04)),
        # the reference's default step at 32^2 for a visible evolution
        "evolve_fixed_N32": dict(N=32, seed=3, coupling="FIXED", steps=50, step=f32(0.0004), slices=20, mu=16.0,
                                 mass=f32(0.04)),
        # sizes that are not powers of two
        "evolve_sqrt_N24": dict(N=24, seed=10, coupling="SQRT_COUPLING_CONSTANT", steps=12, step=f32(0.0004),
                                slices=6, mu=12.0, mass=f32(0.04)),
        "evolve_noise_N15": dict(N=15, seed=11, coupling="NOISE_COUPLING_CONSTANT", steps=12, step=f32(0.0004),
                                 slices=6, mu=7.5, mass=f32(0.04)),
    }
    for name, kw in runs.items():
        if not wanted(name):
            continue
        fx = fixture_evolution(o, **kw)
        d = check_oracle(o, fx)
        print(f"{name}: oracle vs reference max deviation {d:.3e}")
        if d > 1e-12:
            raise SystemExit(f"oracle disagrees with the reference on {name}")
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k: np.asarray(v) for k, v in fx.items()})
    pos = {
        "position_sqrt_sin_N16": dict(N=16, seed=21, coupling="SQRT_COUPLING_CONSTANT", kernel="SIN_KERNEL", steps=4,
                                      slices=6),
        "position_sqrt_linear_N8": dict(N=8, seed=22, coupling="SQRT_COUPLING_CONSTANT", kernel="LINEAR_KERNEL",
                                        steps=4, slices=6),
        "position_cholesky_N8": dict(N=8, seed=23, coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL", steps=4,
                                     slices=6),
        "position_cholesky_N16": dict(N=16, seed=24, coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL",
                                      steps=3, slices=6),
        "position_sqrt_sin_N15": dict(N=15, seed=25, coupling="SQRT_COUPLING_CONSTANT", kernel="SIN_KERNEL", steps=3,
                                      slices=6),
        # Cholesky-correlated noise where N^2 is not a multiple of the factor's blocking
        "position_cholesky_N10": dict(N=10, seed=26, coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL", steps=3,
                                      slices=6),
        "position_cholesky_N12": dict(N=12, seed=27, coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL", steps=3,
                                      slices=6),
    }
    for name, kw in pos.items():
        if not wanted(name):
            continue
        fx = fixture_position(o, **kw)
        d = check_oracle_position(o, fx)
        print(f"{name}: oracle vs reference max deviation {d:.3e}")
        if d > 1e-12:
            raise SystemExit(f"oracle disagrees with the reference on {name}")
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k: np.asarray(v) for k, v in fx.items()})
    for name, (N, seed, cfg) in DRIVER_RUNS.items():
        if not wanted(name):
            continue
        fx = fixture_driver(o, N, seed, cfg)
        print(f"{name}: {len(fx['dat'].splitlines())} output lines")
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k: np.asarray(v) for k, v in fx.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
