"""The main_optimized-equivalent driver (softx-d-21-00092_b200/host/): its noise
order and output table against the reference's own main_optimized run on the
same configuration and noise (tests/golden/driver_*.npz, written by
oracle/_ref/main_optimized_inject_16).  The CPU test replays the driver's
sequence on the oracle and must reproduce the reference's table text exactly;
the GPU test runs the driver binary."""
import math
import os
import subprocess

import numpy as np
import pytest

from jwref import f32

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(REPO, "softx-d-21-00092_b200", "bin", "jimwlk_main")
NAMES = ["driver_sqrt_sin_N16", "driver_noise_sin_N16", "driver_sqrt_linear_N16", "driver_position_cholesky_N16",
         "driver_sqrt_sin_N24"]
COUPLING = {"SQRT_COUPLING_CONSTANT": 0, "NOISE_COUPLING_CONSTANT": 1, "HATTA_COUPLING_CONSTANT": 2}


def parse_config(text: str) -> dict:
    kv = dict(line.split(" = ", 1) for line in text.strip().splitlines())
    return {"stat": int(kv["stat"]), "mu": f32(float(kv["mu"])), "mass": f32(float(kv["mass"])),
            "ny": int(kv["elementaryWilsonLines"]), "steps": int(kv["langevin_steps"]),
            "meas": int(kv["measurements"]), "step": f32(float(kv["step"])), "evolution": kv["EvolutionChoice"],
            "coupling": COUPLING[kv["CouplingChoice"]], "kernel": 1 if kv["KernelChoice"] == "SIN_KERNEL" else 0}


def table(N: int, measurement: int, s: np.ndarray, e: np.ndarray, x: float) -> str:
    """print (field.h:2521-2547) for |kx - ky| <= 4."""
    out = []
    for xx in range(N):
        for yy in range(N):
            if abs(xx - yy) <= 4:
                ph2 = 4.0 * math.pow(math.sin(math.pi * xx / N), 2.0) + 4.0 * math.pow(math.sin(math.pi * yy / N), 2.0)
                out.append("%i %i %i \t %f %e %e\n" % (measurement, xx, yy, math.sqrt(ph2), x * ph2 * s[xx, yy].real,
                                                        x * ph2 * e[xx, yy].real))
    return "".join(out)


def parse_dat(text: str) -> np.ndarray:
    return np.array([[float(v) for v in line.split()] for line in text.strip().splitlines()])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_replays_reference_main(oracle, gold, name):
    fx = gold(name)
    N, seed = int(fx["N"]), int(fx["seed"])
    c = parse_config(str(fx["config"]))
    L = oracle.cholesky(oracle.correlations(N)) if (c["evolution"] == "POSITION_EVOLUTION" and
                                                     c["coupling"] == 1) else None
    every = c["steps"] // c["meas"]
    sums = [np.zeros((N, N), np.complex128) for _ in range(c["meas"])]
    errs = [np.zeros((N, N), np.complex128) for _ in range(c["meas"])]
    g = 1.0
    mu = c["mu"] / N
    step_index = 0
    for s in range(c["stat"]):
        V = np.zeros((N, N, 9), np.complex128)
        V[..., 0] = V[..., 4] = V[..., 8] = 1.0
        for i in range(c["ny"]):
            f = oracle.set_mv_model(oracle.mv_normals(seed, s * c["ny"] + i, N), g * mu / math.sqrt(c["ny"]))
            f = oracle.execute2D(f, 1)
            f = oracle.solve_poisson(f, c["mass"] * g * g * mu, g)
            f = oracle.execute2D(f, 0)
            V = oracle.mul_exp(V, f)
        for lv in range(c["steps"]):
            if c["evolution"] == "MOMENTUM_EVOLUTION":
                V = oracle.evolve_momentum(V, 1, step_index, c["step"], c["coupling"], c["kernel"], seed)
            else:
                V = oracle.evolve_position(V, 1, step_index, c["step"], c["coupling"], c["kernel"], 0, L, seed)
            step_index += 1
            if lv % every == 0:
                t = lv * c["meas"] // c["steps"]
                _, sums[t], errs[t] = oracle.measure(V, sums[t], errs[t])
    m = c["meas"] - 1
    assert table(N, m, sums[m], errs[m], 1.0 / 3.0 / c["stat"]) == str(fx["dat"])


HATTA_CONFIG = ("stat = 1\nmu = 8\nmass = 0.04\nelementaryWilsonLines = 4\nfile_name = output\n"
                "langevin_steps = 3\nmeasurements = 3\nstep = 0.0004\nEvolutionChoice = POSITION_EVOLUTION\n"
                "CouplingChoice = HATTA_COUPLING_CONSTANT\nKernelChoice = SIN_KERNEL\n")


def hatta_table(oracle, N: int, seed: int) -> str:
    """The driver's Hatta run replayed on the oracle: branches (ix, iy) in the
    reference's order (main_optimized.cpp:200-216), each from the initial
    condition with rr = |(ix, iy)|^2 and its own block of noise indices,
    reduce_hatta at (ix, iy) (field.h:1538-1564).  The reference leaves the
    HATTA coupling uninitialised, so this is the formula's intent, not a
    reference output."""
    c = parse_config(HATTA_CONFIG)
    g, mu = 1.0, c["mu"] / N
    V0 = np.zeros((N, N, 9), np.complex128)
    V0[..., 0] = V0[..., 4] = V0[..., 8] = 1.0
    for i in range(c["ny"]):
        f = oracle.set_mv_model(oracle.mv_normals(seed, i, N), g * mu / math.sqrt(c["ny"]))
        f = oracle.solve_poisson(oracle.execute2D(f, 1), c["mass"] * g * g * mu, g)
        V0 = oracle.mul_exp(V0, oracle.execute2D(f, 0))
    every = c["steps"] // c["meas"]
    sums = [np.zeros((N, N), np.complex128) for _ in range(c["meas"])]
    errs = [np.zeros((N, N), np.complex128) for _ in range(c["meas"])]
    step_index = 0
    for ix in range(N):
        for iy in range(ix - 1, ix + 2):
            if not 0 <= iy < N:
                continue
            dix = ix - N if ix >= N // 2 else ix
            diy = iy - N if iy >= N // 2 else iy
            rr = dix * dix + diy * diy
            V = V0.copy()
            for lv in range(c["steps"]):
                V = oracle.evolve_position(V, 1, step_index, c["step"], 2, c["kernel"], rr, None, seed)
                step_index += 1
                if lv % every == 0:
                    t = lv * c["meas"] // c["steps"]
                    corr, _, _ = oracle.measure(V)
                    sums[t][ix, iy] += corr[ix, iy].real
                    errs[t][ix, iy] += corr[ix, iy].real ** 2
    m = c["meas"] - 1
    return table(N, m, sums[m], errs[m], 1.0 / 3.0 / c["stat"])


def test_driver_usage_without_arguments():
    if not os.path.exists(DRIVER):
        pytest.skip("driver not built (make -C softx-d-21-00092_b200)")
    r = subprocess.run([DRIVER], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["fused", "call-for-call"])
@pytest.mark.parametrize("name", NAMES)
def test_driver_matches_reference_main(gold, tmp_path, name, mode):
    fx = gold(name)
    N, seed = int(fx["N"]), int(fx["seed"])
    cfg = tmp_path / "config"
    cfg.write_text(str(fx["config"]))
    args = [DRIVER, "1", "1", str(cfg), "--N", str(N), "--seed", str(seed)]
    if mode == "call-for-call":
        args.append("--call-for-call")
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Evolution time:" in r.stdout and "Initial condition time:" in r.stdout
    got = parse_dat((tmp_path / f"output_optimized_{N}_{N}_mpi1_r0.dat").read_text())
    want = parse_dat(str(fx["dat"]))
    assert got.shape == want.shape
    assert np.array_equal(got[:, :3], want[:, :3])
    # the table prints 7 significant digits
    assert np.allclose(got[:, 3:], want[:, 3:], rtol=2e-6, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,N", [("batched", 8), ("batched-mixed", 8), ("call-for-call", 8), ("batched", 6)])
def test_driver_hatta_matches_oracle(oracle, tmp_path, mode, N):
    """The Hatta branches as engine events (batched), or one after another:
    with --call-for-call, and at a size that is not a power of two (6), which
    the engine does not take, whatever the mode."""
    seed = 5
    cfg = tmp_path / "config"
    cfg.write_text(HATTA_CONFIG)
    args = [DRIVER, "1", "1", str(cfg), "--N", str(N), "--seed", str(seed)]
    args += {"batched": [], "batched-mixed": ["--mixed"], "call-for-call": ["--call-for-call"]}[mode]
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = parse_dat((tmp_path / f"output_optimized_{N}_{N}_mpi1_r0.dat").read_text())
    want = parse_dat(hatta_table(oracle, N, seed))
    assert np.array_equal(got[:, :3], want[:, :3])
    rtol = 2e-6 if mode != "batched-mixed" else 2e-4
    assert np.allclose(got[:, 3:], want[:, 3:], rtol=rtol, atol=1e-14)
