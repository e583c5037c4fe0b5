"""ctypes bindings of the two CPU checkers (test infrastructure only).

* ``Oracle``   -- oracle/build/libjw_oracle.so, the C restatement of the hot
  path (oracle/jw_oracle.c), any lattice size N.
* ``Reference`` -- oracle/_ref/libref_<N>.so, the reference solver's own
  field.h / su3_matrix.h / zheevh3 code compiled here for one N with
  single-rank MPI and FFTW shims and injected noise (oracle/ref_harness.cpp).
  Each instance owns one process-wide context (one config file); build it with
  ``reference(N, config_text)`` which loads a private copy of the library so
  several configurations can coexist in one test process.

Fields are numpy complex128 arrays in the reference's site-major layout,
shape (N, N, t) with t = 9 (3x3 row-major) or 1.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import tempfile

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "build", "libjw_oracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def build_oracle() -> None:
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)


class Oracle:
    def __init__(self) -> None:
        build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        self.L = L
        u64 = ctypes.c_uint64
        L.jwo_langevin_normals.argtypes = [u64, u64, ctypes.c_int, _dp]
        L.jwo_mv_normals.argtypes = [u64, ctypes.c_int, ctypes.c_int, _dp]
        L.jwo_execute2D.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.jwo_generate_gaussian.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.jwo_set_mv_model.argtypes = [_dp, ctypes.c_double, _dp, ctypes.c_int]
        L.jwo_solve_poisson.argtypes = [_dp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.jwo_mul_exp.argtypes = [_dp, _dp, ctypes.c_int]
        L.jwo_prepare_A_local.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.jwo_uxiulocal.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int]
        L.jwo_update_uf.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_double]
        L.jwo_su3_exponentiate.argtypes = [_dp, ctypes.c_double]
        L.jwo_su3_exponentiate.restype = ctypes.c_int
        L.jwo_zheevh3.argtypes = [_dp, _dp, _dp]
        L.jwo_zheevh3.restype = ctypes.c_int
        L.jwo_trace.argtypes = [_dp, _dp, ctypes.c_int]
        L.jwo_average_and_symmetrize.argtypes = [_dp, ctypes.c_int]
        L.jwo_reduce.argtypes = [_dp, _dp, _dp, ctypes.c_int]
        L.jwo_initial_condition.argtypes = [_dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, u64]
        L.jwo_evolve_momentum.argtypes = [_dp, ctypes.c_int, ctypes.c_int, u64, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, u64]
        L.jwo_measure.argtypes = [_dp, ctypes.c_int, _dp, _dp, _dp]
        L.jwo_prepare_A_and_B.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int]
        L.jwo_position_kernel.argtypes = [ctypes.c_int] * 6 + [_dp, _dp]
        L.jwo_correlations.argtypes = [ctypes.c_int, _dp]
        L.jwo_cholesky.argtypes = [_dp, ctypes.c_int, _dp]
        L.jwo_multiply_by_cholesky.argtypes = [_dp, _dp, ctypes.c_int]
        L.jwo_evolve_position.argtypes = [_dp, ctypes.c_int, ctypes.c_int, u64, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, _dp, u64]
        L.jwo_reduce_hatta.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.jwo_dipole_position.argtypes = [_dp, ctypes.c_int, _dp]
        L.jwo_dipole_radial.argtypes = [_dp, ctypes.c_int, _dp, _dp, _ip]
        L.jwo_dipole_radial.restype = ctypes.c_int
        L.jwo_saturation_scale.argtypes = [_dp, _dp, ctypes.c_int]
        L.jwo_saturation_scale.restype = ctypes.c_double

    # ---- noise ----
    def langevin_normals(self, seed: int, step: int, N: int) -> np.ndarray:
        z = np.empty((N, N, 16), np.float64)
        self.L.jwo_langevin_normals(seed, step, N, _ptr(z))
        return z

    def mv_normals(self, seed: int, slice_: int, N: int) -> np.ndarray:
        z = np.empty((N, N, 8), np.float64)
        self.L.jwo_mv_normals(seed, slice_, N, _ptr(z))
        return z

    # ---- primitives ----
    def execute2D(self, f: np.ndarray, direction: int) -> np.ndarray:
        f = np.ascontiguousarray(f, np.complex128).copy()
        N, t = f.shape[0], f.shape[2]
        self.L.jwo_execute2D(_ptr(f.view(np.float64)), N, t, direction)
        return f

    def generate_gaussian(self, z16: np.ndarray, with_coupling: bool):
        N = z16.shape[0]
        xx = np.empty((N, N, 9), np.complex128)
        xy = np.empty((N, N, 9), np.complex128)
        self.L.jwo_generate_gaussian(_ptr(np.ascontiguousarray(z16)), _ptr(xx.view(np.float64)),
                                     _ptr(xy.view(np.float64)), N, int(with_coupling))
        return xx, xy

    def set_mv_model(self, z8: np.ndarray, sigma: float) -> np.ndarray:
        N = z8.shape[0]
        f = np.empty((N, N, 9), np.complex128)
        self.L.jwo_set_mv_model(_ptr(np.ascontiguousarray(z8)), sigma, _ptr(f.view(np.float64)), N)
        return f

    def solve_poisson(self, f: np.ndarray, mass: float, g: float) -> np.ndarray:
        f = np.ascontiguousarray(f, np.complex128).copy()
        self.L.jwo_solve_poisson(_ptr(f.view(np.float64)), f.shape[0], mass, g)
        return f

    def mul_exp(self, V: np.ndarray, f: np.ndarray) -> np.ndarray:
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.jwo_mul_exp(_ptr(V.view(np.float64)), _ptr(np.ascontiguousarray(f).view(np.float64)), V.shape[0])
        return V

    def prepare_A_local(self, xi_x, xi_y, coupling: int, kernel: int) -> np.ndarray:
        N = xi_x.shape[0]
        A = np.empty((N, N, 9), np.complex128)
        self.L.jwo_prepare_A_local(_ptr(A.view(np.float64)), _ptr(np.ascontiguousarray(xi_x).view(np.float64)),
                                   _ptr(np.ascontiguousarray(xi_y).view(np.float64)), N, coupling, kernel)
        return A

    def uxiulocal(self, V, xi_x, xi_y):
        N = V.shape[0]
        ux = np.empty((N, N, 9), np.complex128)
        uy = np.empty((N, N, 9), np.complex128)
        self.L.jwo_uxiulocal(_ptr(ux.view(np.float64)), _ptr(uy.view(np.float64)),
                             _ptr(np.ascontiguousarray(V).view(np.float64)),
                             _ptr(np.ascontiguousarray(xi_x).view(np.float64)),
                             _ptr(np.ascontiguousarray(xi_y).view(np.float64)), N)
        return ux, uy

    def update_uf(self, V, B, A, step: float) -> np.ndarray:
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.jwo_update_uf(_ptr(V.view(np.float64)), _ptr(np.ascontiguousarray(B).view(np.float64)),
                             _ptr(np.ascontiguousarray(A).view(np.float64)), V.shape[0], step)
        return V

    def su3_exponentiate(self, m: np.ndarray, sign: float):
        m = np.ascontiguousarray(m, np.complex128).reshape(-1, 9).copy()
        status = [self.L.jwo_su3_exponentiate(_ptr(row.view(np.float64)), sign) for row in m]
        return m, np.array(status)

    def zheevh3(self, A: np.ndarray):
        A = np.ascontiguousarray(A, np.complex128).reshape(9)
        Q = np.empty(9, np.complex128)
        w = np.empty(3, np.float64)
        s = self.L.jwo_zheevh3(_ptr(A.view(np.float64)), _ptr(Q.view(np.float64)), _ptr(w))
        return Q.reshape(3, 3), w, s

    # ---- compositions ----
    def initial_condition(self, N: int, mu_cfg: float, mass_cfg: float, nslices: int, seed: int) -> np.ndarray:
        V = np.empty((N, N, 9), np.complex128)
        self.L.jwo_initial_condition(_ptr(V.view(np.float64)), N, mu_cfg, mass_cfg, nslices, seed)
        return V

    def evolve_momentum(self, V, steps: int, step0: int, step: float, coupling: int, kernel: int, seed: int):
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.jwo_evolve_momentum(_ptr(V.view(np.float64)), V.shape[0], steps, step0, step, coupling, kernel, seed)
        return V

    def measure(self, V, sum_=None, err=None):
        N = V.shape[0]
        corr = np.zeros((N, N), np.complex128)
        sum_ = np.zeros((N, N), np.complex128) if sum_ is None else sum_.copy()
        err = np.zeros((N, N), np.complex128) if err is None else err.copy()
        self.L.jwo_measure(_ptr(np.ascontiguousarray(V).view(np.float64)), N, _ptr(corr.view(np.float64)),
                           _ptr(sum_.view(np.float64)), _ptr(err.view(np.float64)))
        return corr, sum_, err

    def prepare_A_and_B(self, xi_x, xi_y, V, rr: int, coupling: int, kernel: int):
        N = V.shape[0]
        A = np.empty((N, N, 9), np.complex128)
        B = np.empty((N, N, 9), np.complex128)
        self.L.jwo_prepare_A_and_B(_ptr(A.view(np.float64)), _ptr(B.view(np.float64)),
                                   _ptr(np.ascontiguousarray(xi_x).view(np.float64)),
                                   _ptr(np.ascontiguousarray(xi_y).view(np.float64)),
                                   _ptr(np.ascontiguousarray(V).view(np.float64)), N, rr, coupling, kernel)
        return A, B

    def correlations(self, N: int) -> np.ndarray:
        c = np.empty((N, N), np.complex128)
        self.L.jwo_correlations(N, _ptr(c.view(np.float64)))
        return c

    def cholesky(self, corr: np.ndarray) -> np.ndarray:
        N = corr.shape[0]
        L = np.empty((N * N, N * N), np.complex128)
        self.L.jwo_cholesky(_ptr(np.ascontiguousarray(corr).view(np.float64)), N, _ptr(L.view(np.float64)))
        return L

    def multiply_by_cholesky(self, L, xi):
        xi = np.ascontiguousarray(xi, np.complex128).copy()
        self.L.jwo_multiply_by_cholesky(_ptr(np.ascontiguousarray(L).view(np.float64)), _ptr(xi.view(np.float64)),
                                        xi.shape[0])
        return xi

    def evolve_position(self, V, steps, step0, step, coupling, kernel, rr, L, seed):
        V = np.ascontiguousarray(V, np.complex128).copy()
        Lp = _ptr(np.ascontiguousarray(L).view(np.float64)) if L is not None else None
        self.L.jwo_evolve_position(_ptr(V.view(np.float64)), V.shape[0], steps, step0, step, coupling, kernel, rr,
                                   Lp, seed)
        return V

    def dipole(self, corr_sym: np.ndarray):
        N = corr_sym.shape[0]
        Sxy = np.empty((N, N), np.float64)
        self.L.jwo_dipole_position(_ptr(np.ascontiguousarray(corr_sym, np.complex128).view(np.float64)), N, _ptr(Sxy))
        nb = N // 2 + 1
        Sb = np.empty(nb)
        rb = np.empty(nb)
        cb = np.empty(nb, np.int32)
        self.L.jwo_dipole_radial(_ptr(Sxy), N, _ptr(Sb), _ptr(rb), cb.ctypes.data_as(_ip))
        qs = self.L.jwo_saturation_scale(_ptr(Sb), _ptr(rb), nb)
        return Sxy, Sb, rb, cb, qs


class Reference:
    """The reference's own code for one lattice size and one config file."""

    def __init__(self, N: int, config_text: str | None = None) -> None:
        src = os.path.join(REF_DIR, f"libref_{N}.so")
        if not os.path.exists(src):
            raise FileNotFoundError(src)
        self._tmp = tempfile.mkdtemp(prefix="jwref_")
        so = os.path.join(self._tmp, f"libref_{N}.so")
        shutil.copy(src, so)  # private copy: one config per loaded instance
        L = ctypes.CDLL(so, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        self.L = L
        self.N = N
        L.ref_init.argtypes = [ctypes.c_char_p]
        L.ref_config.argtypes = [_dp, _ip]
        L.ref_set_injection.argtypes = [_dp, ctypes.c_long]
        L.ref_injection_consumed.restype = ctypes.c_long
        L.ref_execute2D.argtypes = [_dp, ctypes.c_int, ctypes.c_int]
        L.ref_generate_gaussian.argtypes = [_dp, _dp, ctypes.c_int]
        L.ref_set_mv_model.argtypes = [_dp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ref_solve_poisson.argtypes = [_dp, ctypes.c_double, ctypes.c_double]
        L.ref_mul_exp.argtypes = [_dp, _dp]
        L.ref_prepare_A_local.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.ref_uxiulocal.argtypes = [_dp, _dp, _dp, _dp, _dp]
        L.ref_update_uf.argtypes = [_dp, _dp, _dp, ctypes.c_double]
        L.ref_su3_exponentiate.argtypes = [_dp, ctypes.c_long, ctypes.c_double]
        L.ref_su3_exponentiate.restype = ctypes.c_int
        L.ref_initial_condition.argtypes = [_dp]
        L.ref_evolve_momentum.argtypes = [_dp, ctypes.c_int]
        L.ref_evolve_momentum_fixed.argtypes = [_dp, ctypes.c_int]
        L.ref_measure.argtypes = [_dp, _dp, _dp, _dp]
        L.ref_print.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_char_p]
        L.ref_prepare_A_and_B.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ref_cholesky_setup.argtypes = [_dp, _dp]
        L.ref_multiply_by_cholesky.argtypes = [_dp]
        L.ref_evolve_position.argtypes = [_dp, ctypes.c_int, ctypes.c_int]
        L.ref_measure_hatta.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        path = b""
        if config_text is not None:
            cfg = os.path.join(self._tmp, "config")
            with open(cfg, "w") as fh:
                fh.write(config_text)
            path = cfg.encode()
        L.ref_init(path)
        self._keep = None

    def config(self):
        d = np.zeros(3)
        i = np.zeros(7, np.int32)
        self.L.ref_config(_ptr(d), i.ctypes.data_as(_ip))
        return dict(mu=d[0], mass=d[1], step=d[2], stat=int(i[0]), elementaryWilsonLines=int(i[1]),
                    langevin_steps=int(i[2]), measurements=int(i[3]), evolution=int(i[4]),
                    coupling=int(i[5]), kernel=int(i[6]))

    def inject(self, z: np.ndarray) -> None:
        self._keep = np.ascontiguousarray(z, np.float64).ravel()
        self.L.ref_set_injection(_ptr(self._keep), self._keep.size)

    def consumed(self) -> int:
        return int(self.L.ref_injection_consumed())

    def execute2D(self, f: np.ndarray, direction: int) -> np.ndarray:
        f = np.ascontiguousarray(f, np.complex128).copy()
        self.L.ref_execute2D(_ptr(f.view(np.float64)), f.shape[2], direction)
        return f

    def generate_gaussian(self, z16: np.ndarray, with_coupling: bool):
        N = self.N
        self.inject(z16)
        xx = np.empty((N, N, 9), np.complex128)
        xy = np.empty((N, N, 9), np.complex128)
        self.L.ref_generate_gaussian(_ptr(xx.view(np.float64)), _ptr(xy.view(np.float64)), int(with_coupling))
        return xx, xy

    def set_mv_model(self, z8: np.ndarray, g: float, mu: float, nslices: int) -> np.ndarray:
        self.inject(z8)
        f = np.empty((self.N, self.N, 9), np.complex128)
        self.L.ref_set_mv_model(_ptr(f.view(np.float64)), g, mu, nslices)
        return f

    def solve_poisson(self, f, mass, g):
        f = np.ascontiguousarray(f, np.complex128).copy()
        self.L.ref_solve_poisson(_ptr(f.view(np.float64)), mass, g)
        return f

    def mul_exp(self, V, f):
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.ref_mul_exp(_ptr(V.view(np.float64)), _ptr(np.ascontiguousarray(f).view(np.float64)))
        return V

    def prepare_A_local(self, xi_x, xi_y, coupling, kernel):
        A = np.empty((self.N, self.N, 9), np.complex128)
        self.L.ref_prepare_A_local(_ptr(A.view(np.float64)), _ptr(np.ascontiguousarray(xi_x).view(np.float64)),
                                   _ptr(np.ascontiguousarray(xi_y).view(np.float64)), coupling, kernel)
        return A

    def uxiulocal(self, V, xi_x, xi_y):
        ux = np.empty((self.N, self.N, 9), np.complex128)
        uy = np.empty((self.N, self.N, 9), np.complex128)
        self.L.ref_uxiulocal(_ptr(ux.view(np.float64)), _ptr(uy.view(np.float64)),
                             _ptr(np.ascontiguousarray(V).view(np.float64)),
                             _ptr(np.ascontiguousarray(xi_x).view(np.float64)),
                             _ptr(np.ascontiguousarray(xi_y).view(np.float64)))
        return ux, uy

    def update_uf(self, V, B, A, step):
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.ref_update_uf(_ptr(V.view(np.float64)), _ptr(np.ascontiguousarray(B).view(np.float64)),
                             _ptr(np.ascontiguousarray(A).view(np.float64)), step)
        return V

    def su3_exponentiate(self, m, sign):
        m = np.ascontiguousarray(m, np.complex128).reshape(-1, 9).copy()
        bad = self.L.ref_su3_exponentiate(_ptr(m.view(np.float64)), m.shape[0], sign)
        return m, bad

    def initial_condition(self, z_all: np.ndarray) -> np.ndarray:
        self.inject(z_all)
        V = np.empty((self.N, self.N, 9), np.complex128)
        self.L.ref_initial_condition(_ptr(V.view(np.float64)))
        return V

    def evolve_momentum(self, V, z_all: np.ndarray, steps: int) -> np.ndarray:
        self.inject(z_all)
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.ref_evolve_momentum(_ptr(V.view(np.float64)), steps)
        return V

    def evolve_momentum_fixed(self, V, z_all: np.ndarray, steps: int) -> np.ndarray:
        self.inject(z_all)
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.ref_evolve_momentum_fixed(_ptr(V.view(np.float64)), steps)
        return V

    def prepare_A_and_B(self, xi_x, xi_y, V, rr, coupling, kernel):
        N = self.N
        A = np.empty((N, N, 9), np.complex128)
        B = np.empty((N, N, 9), np.complex128)
        self.L.ref_prepare_A_and_B(_ptr(A.view(np.float64)), _ptr(B.view(np.float64)),
                                   _ptr(np.ascontiguousarray(xi_x).view(np.float64)),
                                   _ptr(np.ascontiguousarray(xi_y).view(np.float64)),
                                   _ptr(np.ascontiguousarray(V).view(np.float64)), rr, coupling, kernel)
        return A, B

    def cholesky_setup(self):
        N = self.N
        L = np.empty((N * N, N * N), np.complex128)
        c = np.empty((N, N), np.complex128)
        self.L.ref_cholesky_setup(_ptr(L.view(np.float64)), _ptr(c.view(np.float64)))
        return L, c

    def multiply_by_cholesky(self, xi):
        xi = np.ascontiguousarray(xi, np.complex128).copy()
        self.L.ref_multiply_by_cholesky(_ptr(xi.view(np.float64)))
        return xi

    def evolve_position(self, V, z_all, steps, rr=0):
        self.inject(z_all)
        V = np.ascontiguousarray(V, np.complex128).copy()
        self.L.ref_evolve_position(_ptr(V.view(np.float64)), steps, rr)
        return V

    def measure(self, V, sum_=None, err=None):
        N = self.N
        corr = np.zeros((N, N), np.complex128)
        sum_ = np.zeros((N, N), np.complex128) if sum_ is None else sum_.copy()
        err = np.zeros((N, N), np.complex128) if err is None else err.copy()
        self.L.ref_measure(_ptr(np.ascontiguousarray(V).view(np.float64)), _ptr(corr.view(np.float64)),
                           _ptr(sum_.view(np.float64)), _ptr(err.view(np.float64)))
        return corr, sum_, err


def reference_available(N: int) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{N}.so"))


def config_text(*, stat=1, mu=30.72, mass=0.0001, wilson_lines=50, file_name="output", langevin_steps=100,
                measurements=100, step=0.0004, evolution="MOMENTUM_EVOLUTION",
                coupling="NOISE_COUPLING_CONSTANT", kernel="SIN_KERNEL") -> str:
    """A config file in the reference's grammar (config.h:83-101)."""
    return (f"stat = {stat}\nmu = {mu}\nmass = {mass}\nelementaryWilsonLines = {wilson_lines}\n"
            f"file_name = {file_name}\nlangevin_steps = {langevin_steps}\nmeasurements = {measurements}\n"
            f"step = {step}\nEvolutionChoice = {evolution}\nCouplingChoice = {coupling}\n"
            f"KernelChoice = {kernel}\n")


def f32(x: float) -> float:
    """The value the reference holds after parsing x through `float` (config.h:84-93)."""
    return float(np.float32(x))
