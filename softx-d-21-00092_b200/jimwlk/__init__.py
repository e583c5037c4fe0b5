"""Python binding of libjimwlk (include/jimwlk.h) over ctypes.

The product is the CUDA library ``lib/libjimwlk.so`` built from ``csrc/``;
this module only marshals arguments.  It has no CPU fallback: if the library
is missing, importing raises ``JimwlkError``.

Host field arrays are numpy complex128 arrays of shape (N, N, t) in the
reference solver's site-major layout (t = 9: row-major 3x3; t = 1: scalar).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libjimwlk.so")

OK, EINVAL, ENOMEM, ECUDA, ENOCONV, ENAN, ETIMEOUT, EUNSUPPORTED, ENOTFOUND, EBUSY = 0, -1, -2, -3, -4, -5, -6, -7, -8, -9
POSITION_EVOLUTION, MOMENTUM_EVOLUTION = 0, 1
SQRT_COUPLING_CONSTANT, NOISE_COUPLING_CONSTANT, HATTA_COUPLING_CONSTANT, FIXED_COUPLING_CONSTANT = 0, 1, 2, 3
LINEAR_KERNEL, SIN_KERNEL = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1


class JimwlkError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = _lib.jw_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{where}: {msg} ({status})" if where else f"{msg} ({status})")


class jw_config(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("stat", ctypes.c_int), ("mu", ctypes.c_double),
                ("mass", ctypes.c_double), ("elementaryWilsonLines", ctypes.c_int), ("file_name", ctypes.c_char * 64),
                ("langevin_steps", ctypes.c_int), ("measurements", ctypes.c_int), ("step", ctypes.c_double),
                ("EvolutionChoice", ctypes.c_int), ("CouplingChoice", ctypes.c_int), ("KernelChoice", ctypes.c_int),
                ("seed", ctypes.c_uint64)]


class jw_engine_options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("reunitarize", ctypes.c_int), ("max_bytes", ctypes.c_size_t),
                ("max_batch", ctypes.c_int), ("max_batch_sites", ctypes.c_size_t), ("autotune", ctypes.c_int)]


class jw_event_desc(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("ny_slices", ctypes.c_int), ("mu", ctypes.c_double), ("mass", ctypes.c_double),
                ("step", ctypes.c_double), ("coupling", ctypes.c_int), ("kernel", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("position_space", ctypes.c_int), ("rr", ctypes.c_int),
                ("step0", ctypes.c_uint64)]


class jw_server_options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("reunitarize", ctypes.c_int), ("max_bytes", ctypes.c_size_t),
                ("max_steps_per_tick", ctypes.c_int), ("max_active", ctypes.c_int), ("fake_device", ctypes.c_int),
                ("fake_ns_per_site_step", ctypes.c_double), ("tick_sites", ctypes.c_size_t)]


class jw_request_desc(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("ny_slices", ctypes.c_int), ("mu", ctypes.c_double), ("mass", ctypes.c_double),
                ("step", ctypes.c_double), ("coupling", ctypes.c_int), ("kernel", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("steps", ctypes.c_int)]


class jw_request_result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("N", ctypes.c_int), ("steps", ctypes.c_int), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double), ("Qs", ctypes.c_double),
                ("nbins", ctypes.c_int)]


class jw_server_stats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("queued", ctypes.c_int64), ("site_steps", ctypes.c_double), ("max_active", ctypes.c_int),
                ("now", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_mv", ctypes.c_double),
                ("t_step", ctypes.c_double), ("t_retire", ctypes.c_double)]


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libjimwlk is not built ({LIB_PATH}); run `make -C softx-d-21-00092_b200` "
                          "or __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "jw_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "jw_config_defaults": ([ctypes.POINTER(jw_config)], ctypes.c_int),
        "jw_config_read": ([ctypes.POINTER(jw_config), ctypes.c_char_p], ctypes.c_int),
        "jw_context_create": ([ctypes.POINTER(jw_config), ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
        "jw_context_destroy": ([_vp], ctypes.c_int),
        "jw_context_sync": ([_vp], ctypes.c_int),
        "jw_context_stream": ([_vp], _vp),
        "jw_field_create": ([_vp, ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
        "jw_field_destroy": ([_vp], ctypes.c_int),
        "jw_field_set": ([_vp, _dp], ctypes.c_int),
        "jw_field_get": ([_vp, _dp], ctypes.c_int),
        "jw_field_copy": ([_vp, _vp], ctypes.c_int),
        "jw_field_save": ([_vp, ctypes.c_char_p], ctypes.c_int),
        "jw_field_load": ([_vp, ctypes.c_char_p], ctypes.c_int),
        "jw_engine_save_event": ([_vp, ctypes.c_int, ctypes.c_char_p], ctypes.c_int),
        "jw_engine_load_event": ([_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "jw_field_set_unit": ([_vp], ctypes.c_int),
        "jw_field_set_zero": ([_vp], ctypes.c_int),
        "jw_execute2D": ([_vp, _vp, ctypes.c_int], ctypes.c_int),
        "jw_generate_gaussian": ([_vp, _vp, _vp, ctypes.c_uint64, ctypes.c_int], ctypes.c_int),
        "jw_set_mv_model": ([_vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int], ctypes.c_int),
        "jw_solve_poisson": ([_vp, _vp, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "jw_mul_exp": ([_vp, _vp, _vp], ctypes.c_int),
        "jw_prepare_A_local": ([_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "jw_uxiulocal": ([_vp, _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
        "jw_update_uf": ([_vp, _vp, _vp, _vp, ctypes.c_double], ctypes.c_int),
        "jw_trace": ([_vp, _vp, _vp], ctypes.c_int),
        "jw_average_and_symmetrize": ([_vp, _vp], ctypes.c_int),
        "jw_reduce": ([_vp, _vp, _vp, _vp], ctypes.c_int),
        "jw_print": ([_vp, ctypes.c_int, _vp, _vp, ctypes.c_double, ctypes.c_char_p], ctypes.c_int),
        "jw_initial_condition": ([_vp, _vp], ctypes.c_int),
        "jw_evolve_momentum": ([_vp, _vp, ctypes.c_uint64, ctypes.c_int], ctypes.c_int),
        "jw_prepare_A_and_B": ([_vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int],
                               ctypes.c_int),
        "jw_set_correlations_for_coupling_constant": ([_vp, _vp], ctypes.c_int),
        "jw_cholesky_decompose": ([_vp, _vp, ctypes.POINTER(_vp)], ctypes.c_int),
        "jw_cholesky_destroy": ([_vp], ctypes.c_int),
        "jw_cholesky_get": ([_vp, _dp], ctypes.c_int),
        "jw_multiply_by_cholesky": ([_vp, _vp, _vp], ctypes.c_int),
        "jw_dipole": ([_vp, _vp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                       ctypes.POINTER(ctypes.c_int), _dp], ctypes.c_int),
        "jw_reduce_hatta": ([_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "jw_evolve_position": ([_vp, _vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _vp], ctypes.c_int),
        "jw_engine_create": ([ctypes.POINTER(jw_engine_options), ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
        "jw_engine_destroy": ([_vp], ctypes.c_int),
        "jw_engine_sync": ([_vp], ctypes.c_int),
        "jw_engine_stream": ([_vp], _vp),
        "jw_engine_event_bytes": ([_vp, ctypes.POINTER(jw_event_desc)], ctypes.c_size_t),
        "jw_engine_add_event": ([_vp, ctypes.POINTER(jw_event_desc), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "jw_engine_remove_event": ([_vp, ctypes.c_int], ctypes.c_int),
        "jw_engine_init_mv": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
        "jw_engine_set_V": ([_vp, ctypes.c_int, _dp], ctypes.c_int),
        "jw_engine_get_V": ([_vp, ctypes.c_int, _dp], ctypes.c_int),
        "jw_engine_step": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "jw_engine_measure": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
        "jw_engine_get_correlator": ([_vp, ctypes.c_int, _dp, _dp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "jw_engine_reset_correlator": ([_vp, ctypes.c_int], ctypes.c_int),
        "jw_engine_copy_V": ([_vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "jw_engine_reset_correlators": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
        "jw_engine_correlator_at": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), _dp, _dp], ctypes.c_int),
        "jw_engine_event_steps": ([_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "jw_server_create": ([ctypes.POINTER(jw_server_options), ctypes.c_int, ctypes.POINTER(_vp)], ctypes.c_int),
        "jw_server_destroy": ([_vp], ctypes.c_int),
        "jw_server_submit": ([_vp, ctypes.POINTER(jw_request_desc), ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "jw_server_wait": ([_vp, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(jw_request_result), _dp, _dp,
                            ctypes.c_int], ctypes.c_int),
        "jw_server_get_stats": ([_vp, ctypes.POINTER(jw_server_stats)], ctypes.c_int),
        "jw_server_size_stats": ([_vp, _ip, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int, _ip],
                                 ctypes.c_int),
        "jw_engine_dipole": ([_vp, ctypes.c_int, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                              ctypes.POINTER(ctypes.c_int), _dp], ctypes.c_int),
        "jw_engine_measure_ensemble": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, _dp, _dp], ctypes.c_int),
        "jw_engine_step_measure_ensemble": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, _dp, _dp],
                                            ctypes.c_int),
        "jw_engine_tuning": ([_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "jw_engine_set_tuning": ([_vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "jw_engine_step_timed": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, _dp,
                                  ctypes.POINTER(ctypes.c_int), _dp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


_lib = None
_lib = _load()


def lib():
    return _lib


def _ck(status: int, where: str) -> None:
    if status != OK:
        raise JimwlkError(status, where)


def config_defaults(**kw) -> jw_config:
    c = jw_config()
    _ck(_lib.jw_config_defaults(ctypes.byref(c)), "jw_config_defaults")
    for k, v in kw.items():
        if k == "file_name":
            v = v.encode() if isinstance(v, str) else v
        setattr(c, k, v)
    return c


def config_read(path: str, base: jw_config | None = None) -> jw_config:
    c = base if base is not None else config_defaults()
    _ck(_lib.jw_config_read(ctypes.byref(c), path.encode()), "jw_config_read")
    return c


class Context:
    """A device context for one lattice size (jw_context)."""

    def __init__(self, cfg: jw_config, device: int = 0):
        self._h = _vp()
        _ck(_lib.jw_context_create(ctypes.byref(cfg), device, ctypes.byref(self._h)), "jw_context_create")
        self.cfg = cfg
        self.N = cfg.Nx
        import weakref
        self._fields = weakref.WeakSet()

    def close(self):
        if self._h:
            # the context releases its fields; detach the Python handles first
            for f in list(self._fields):
                f._h = _vp()
            self._fields.clear()
            _lib.jw_context_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self) -> int:
        return _lib.jw_context_sync(self._h)

    def field(self, t: int = 9) -> "Field":
        return Field(self, t)

    # reference hot-path calls
    def execute2D(self, f, direction):
        _ck(_lib.jw_execute2D(self._h, f._h, direction), "jw_execute2D")

    def generate_gaussian(self, xi_x, xi_y, step_index: int, with_coupling: bool):
        _ck(_lib.jw_generate_gaussian(self._h, xi_x._h, xi_y._h, step_index, int(with_coupling)),
            "jw_generate_gaussian")

    def set_mv_model(self, f, slice_: int, g: float, mu: float, ny_slices: int):
        _ck(_lib.jw_set_mv_model(self._h, f._h, slice_, g, mu, ny_slices), "jw_set_mv_model")

    def solve_poisson(self, f, mass: float, g: float):
        _ck(_lib.jw_solve_poisson(self._h, f._h, mass, g), "jw_solve_poisson")

    def mul_exp(self, V, f):
        _ck(_lib.jw_mul_exp(self._h, V._h, f._h), "jw_mul_exp")

    def prepare_A_local(self, out, xi_x, xi_y, coupling: int, kernel: int):
        _ck(_lib.jw_prepare_A_local(self._h, out._h, xi_x._h, xi_y._h, coupling, kernel), "jw_prepare_A_local")

    def uxiulocal(self, ux, uy, V, xi_x, xi_y):
        _ck(_lib.jw_uxiulocal(self._h, ux._h, uy._h, V._h, xi_x._h, xi_y._h), "jw_uxiulocal")

    def update_uf(self, V, B, A, step: float):
        _ck(_lib.jw_update_uf(self._h, V._h, B._h, A._h, step), "jw_update_uf")

    def trace(self, Vk, corr):
        _ck(_lib.jw_trace(self._h, Vk._h, corr._h), "jw_trace")

    def average_and_symmetrize(self, corr):
        _ck(_lib.jw_average_and_symmetrize(self._h, corr._h), "jw_average_and_symmetrize")

    def reduce(self, corr, sum_, err):
        _ck(_lib.jw_reduce(self._h, corr._h, sum_._h, err._h), "jw_reduce")

    def print(self, measurement: int, sum_, err, x: float, fileroot: str):
        _ck(_lib.jw_print(self._h, measurement, sum_._h, err._h, x, fileroot.encode()), "jw_print")

    def initial_condition(self, V):
        _ck(_lib.jw_initial_condition(self._h, V._h), "jw_initial_condition")

    def evolve_momentum(self, V, step0: int, n: int):
        _ck(_lib.jw_evolve_momentum(self._h, V._h, step0, n), "jw_evolve_momentum")

    # position-space evolution (main_optimized.cpp:271-304)
    def prepare_A_and_B(self, A, B, xi_x, xi_y, V, rr: int, coupling: int, kernel: int):
        _ck(_lib.jw_prepare_A_and_B(self._h, A._h, B._h, xi_x._h, xi_y._h, V._h, rr, coupling, kernel),
            "jw_prepare_A_and_B")

    def set_correlations_for_coupling_constant(self, corr):
        _ck(_lib.jw_set_correlations_for_coupling_constant(self._h, corr._h),
            "jw_set_correlations_for_coupling_constant")

    def cholesky(self, corr) -> "Cholesky":
        """gmatrix::decompose of the backward-transformed correlation `corr`."""
        return Cholesky(self, corr)

    def multiply_by_cholesky(self, xi, L: "Cholesky"):
        _ck(_lib.jw_multiply_by_cholesky(self._h, xi._h, L._h), "jw_multiply_by_cholesky")

    def dipole(self, corr, with_xy: bool = False):
        """S(r) bins, r bins, counts, Q_s (and S(x, y)) of a symmetrised correlator."""
        N = self.N
        nb = N // 2 + 1
        Sb, rb = np.zeros(nb), np.zeros(nb)
        cb = np.zeros(nb, np.int32)
        nbins, qs = ctypes.c_int(), ctypes.c_double()
        Sxy = np.zeros((N, N)) if with_xy else None
        _ck(_lib.jw_dipole(self._h, corr._h, Sxy.ctypes.data_as(_dp) if with_xy else None, Sb.ctypes.data_as(_dp),
                           rb.ctypes.data_as(_dp), cb.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), nb,
                           ctypes.byref(nbins), ctypes.byref(qs)), "jw_dipole")
        out = (Sb, rb, cb, qs.value)
        return out + (Sxy,) if with_xy else out

    def reduce_hatta(self, corr, sum_, err, xr: int, yr: int):
        _ck(_lib.jw_reduce_hatta(self._h, corr._h, sum_._h, err._h, xr, yr), "jw_reduce_hatta")

    def evolve_position(self, V, step0: int, n: int, rr: int = 0, L: "Cholesky | None" = None):
        _ck(_lib.jw_evolve_position(self._h, V._h, step0, n, rr, L._h if L is not None else None),
            "jw_evolve_position")


class Cholesky:
    """The device Cholesky factor of the site-site correlation (jw_cholesky)."""

    def __init__(self, ctx: Context, corr: "Field"):
        self.ctx = ctx
        self._h = _vp()
        _ck(_lib.jw_cholesky_decompose(ctx._h, corr._h, ctypes.byref(self._h)), "jw_cholesky_decompose")
        ctx._fields.add(self)

    def get(self) -> np.ndarray:
        n = self.ctx.N * self.ctx.N
        a = np.empty((n, n), np.complex128)
        _ck(_lib.jw_cholesky_get(self._h, a.ctypes.data_as(_dp)), "jw_cholesky_get")
        return a

    def close(self):
        if self._h and self.ctx._h:
            _lib.jw_cholesky_destroy(self._h)
        self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field:
    """A device field lfield<double,t> (jw_field)."""

    def __init__(self, ctx: Context, t: int = 9):
        self.ctx = ctx
        self.t = t
        self._h = _vp()
        _ck(_lib.jw_field_create(ctx._h, t, ctypes.byref(self._h)), "jw_field_create")
        ctx._fields.add(self)

    def close(self):
        if self._h and self.ctx._h:
            _lib.jw_field_destroy(self._h)
        self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, a: np.ndarray) -> "Field":
        N = self.ctx.N
        a = np.ascontiguousarray(a, np.complex128)
        if a.shape != (N, N, self.t):
            raise ValueError(f"expected shape {(N, N, self.t)}, got {a.shape}")
        _ck(_lib.jw_field_set(self._h, a.ctypes.data_as(_dp)), "jw_field_set")
        return self

    def get(self) -> np.ndarray:
        N = self.ctx.N
        a = np.empty((N, N, self.t), np.complex128)
        _ck(_lib.jw_field_get(self._h, a.ctypes.data_as(_dp)), "jw_field_get")
        return a

    def save(self, path: str):
        _ck(_lib.jw_field_save(self._h, os.fsencode(path)), "jw_field_save")

    def load(self, path: str) -> "Field":
        _ck(_lib.jw_field_load(self._h, os.fsencode(path)), "jw_field_load")
        return self

    def copy_from(self, other: "Field"):
        _ck(_lib.jw_field_copy(self._h, other._h), "jw_field_copy")

    def set_unit(self):
        _ck(_lib.jw_field_set_unit(self._h), "jw_field_set_unit")

    def set_zero(self):
        _ck(_lib.jw_field_set_zero(self._h), "jw_field_set_zero")


def _ids(ids):
    ids = list(ids)
    arr = (ctypes.c_int * max(len(ids), 1))(*ids)
    return arr, len(ids)


class Engine:
    """The batched engine (jw_engine): resident events advanced by fused kernels."""

    def __init__(self, precision: int = PRECISION_MIXED, reunitarize: bool = False, max_bytes: int = 0,
                 max_batch: int = 0, device: int = 0, max_batch_sites: int = 0, autotune: int = 0):
        self.opt = jw_engine_options(precision, int(reunitarize), max_bytes, max_batch, max_batch_sites,
                                     int(autotune))
        self._h = _vp()
        _ck(_lib.jw_engine_create(ctypes.byref(self.opt), device, ctypes.byref(self._h)), "jw_engine_create")
        self.N = {}

    def close(self):
        if self._h:
            _lib.jw_engine_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return _lib.jw_engine_stream(self._h) or 0

    def sync(self) -> int:
        return _lib.jw_engine_sync(self._h)

    def event_bytes(self, **desc) -> int:
        d = jw_event_desc(**desc)
        return _lib.jw_engine_event_bytes(self._h, ctypes.byref(d))

    def add_event(self, N: int, ny_slices: int = 50, mu: float | None = None, mass: float = 0.04,
                  step: float = 0.0004, coupling: int = FIXED_COUPLING_CONSTANT, kernel: int = SIN_KERNEL,
                  seed: int = 1, position_space: bool = False, rr: int = 0, step0: int = 0) -> int:
        d = jw_event_desc(N, ny_slices, 0.5 * N if mu is None else mu, mass, step, coupling, kernel, seed,
                          int(position_space), rr, step0)
        eid = ctypes.c_int(-1)
        _ck(_lib.jw_engine_add_event(self._h, ctypes.byref(d), ctypes.byref(eid)), "jw_engine_add_event")
        self.N[eid.value] = N
        return eid.value

    def try_add_event(self, **kw):
        """add_event returning (status, id) instead of raising."""
        N = kw["N"]
        d = jw_event_desc(N, kw.get("ny_slices", 50), kw.get("mu", 0.5 * N), kw.get("mass", 0.04),
                          kw.get("step", 0.0004), kw.get("coupling", FIXED_COUPLING_CONSTANT),
                          kw.get("kernel", SIN_KERNEL), kw.get("seed", 1), int(kw.get("position_space", False)),
                          kw.get("rr", 0), kw.get("step0", 0))
        eid = ctypes.c_int(-1)
        st = _lib.jw_engine_add_event(self._h, ctypes.byref(d), ctypes.byref(eid))
        if st == OK:
            self.N[eid.value] = N
        return st, eid.value

    def remove_event(self, eid: int):
        _ck(_lib.jw_engine_remove_event(self._h, eid), "jw_engine_remove_event")
        self.N.pop(eid, None)

    def init_mv(self, ids):
        arr, n = _ids(ids)
        _ck(_lib.jw_engine_init_mv(self._h, arr, n), "jw_engine_init_mv")

    def step(self, ids, nsteps: int = 1):
        arr, n = _ids(ids)
        _ck(_lib.jw_engine_step(self._h, arr, n, nsteps), "jw_engine_step")

    def measure(self, ids):
        arr, n = _ids(ids)
        _ck(_lib.jw_engine_measure(self._h, arr, n), "jw_engine_measure")

    def set_V(self, eid: int, V: np.ndarray):
        N = self.N[eid]
        V = np.ascontiguousarray(V, np.complex128)
        assert V.shape == (N, N, 9)
        _ck(_lib.jw_engine_set_V(self._h, eid, V.ctypes.data_as(_dp)), "jw_engine_set_V")

    def get_V(self, eid: int) -> np.ndarray:
        N = self.N[eid]
        V = np.empty((N, N, 9), np.complex128)
        _ck(_lib.jw_engine_get_V(self._h, eid, V.ctypes.data_as(_dp)), "jw_engine_get_V")
        return V

    def correlator(self, eid: int):
        N = self.N[eid]
        s = np.empty((N, N), np.complex128)
        e = np.empty((N, N), np.complex128)
        n = ctypes.c_int(0)
        _ck(_lib.jw_engine_get_correlator(self._h, eid, s.ctypes.data_as(_dp), e.ctypes.data_as(_dp),
                                          ctypes.byref(n)), "jw_engine_get_correlator")
        return s, e, n.value

    def save_event(self, eid: int, path: str):
        _ck(_lib.jw_engine_save_event(self._h, eid, os.fsencode(path)), "jw_engine_save_event")

    def load_event(self, path: str) -> int:
        eid = ctypes.c_int(-1)
        _ck(_lib.jw_engine_load_event(self._h, os.fsencode(path), ctypes.byref(eid)), "jw_engine_load_event")
        d = jw_event_desc()
        with open(path, "rb") as fh:
            fh.seek(8)
            fh.readinto(d)
        self.N[eid.value] = d.N
        return eid.value

    def copy_V(self, dst: int, src: int):
        _ck(_lib.jw_engine_copy_V(self._h, dst, src), "jw_engine_copy_V")

    def reset_correlators(self, ids):
        arr, n = _ids(ids)
        _ck(_lib.jw_engine_reset_correlators(self._h, arr, n), "jw_engine_reset_correlators")

    def correlator_at(self, ids, xr, yr):
        """(sum, err) of each event's accumulated correlator at (xr[i], yr[i])."""
        arr, n = _ids(ids)
        x = (ctypes.c_int * n)(*[int(v) for v in xr])
        y = (ctypes.c_int * n)(*[int(v) for v in yr])
        s_, e_ = np.zeros(n), np.zeros(n)
        _ck(_lib.jw_engine_correlator_at(self._h, arr, n, x, y, s_.ctypes.data_as(_dp), e_.ctypes.data_as(_dp)),
            "jw_engine_correlator_at")
        return s_, e_

    def reset_correlator(self, eid: int):
        _ck(_lib.jw_engine_reset_correlator(self._h, eid), "jw_engine_reset_correlator")

    def steps_taken(self, eid: int) -> int:
        v = ctypes.c_uint64(0)
        _ck(_lib.jw_engine_event_steps(self._h, eid, ctypes.byref(v)), "jw_engine_event_steps")
        return v.value

    def measure_ensemble(self, ids, sum_out: np.ndarray | None = None, err_out: np.ndarray | None = None):
        ids = list(ids)
        N = self.N[ids[0]]
        s = np.empty((N, N), np.complex128) if sum_out is None else sum_out
        e = np.empty((N, N), np.complex128) if err_out is None else err_out
        arr, n = _ids(ids)
        _ck(_lib.jw_engine_measure_ensemble(self._h, arr, n, s.ctypes.data_as(_dp), e.ctypes.data_as(_dp)),
            "jw_engine_measure_ensemble")
        return s, e

    def step_measure_ensemble(self, ids, nsteps: int = 1, sum_out: np.ndarray | None = None,
                              err_out: np.ndarray | None = None):
        """nsteps Langevin steps of the events, then one ensemble measurement."""
        ids = list(ids)
        N = self.N[ids[0]]
        s = np.empty((N, N), np.complex128) if sum_out is None else sum_out
        e = np.empty((N, N), np.complex128) if err_out is None else err_out
        arr, n = _ids(ids)
        _ck(_lib.jw_engine_step_measure_ensemble(self._h, arr, n, int(nsteps), s.ctypes.data_as(_dp),
                                                 e.ctypes.data_as(_dp)), "jw_engine_step_measure_ensemble")
        return s, e

    def tuning(self, N: int) -> int:
        """Column-tile width the autotuner chose for size N (0 if it has not run)."""
        c = ctypes.c_int(0)
        _ck(_lib.jw_engine_tuning(self._h, int(N), ctypes.byref(c)), "jw_engine_tuning")
        return c.value

    def set_tuning(self, N: int, p2_cols: int) -> None:
        _ck(_lib.jw_engine_set_tuning(self._h, int(N), int(p2_cols)), "jw_engine_set_tuning")


    def step_timed(self, ids, nsteps: int):
        """nsteps steps with every kernel timed: ({kind: (total ms, launches)}, total ms)."""
        arr, n = _ids(ids)
        p = (ctypes.c_double * 4)()
        c = (ctypes.c_int * 4)()
        tot = ctypes.c_double(0)
        _ck(_lib.jw_engine_step_timed(self._h, arr, n, nsteps, p, c, ctypes.byref(tot)), "jw_engine_step_timed")
        kinds = ("pass1", "pass2", "pass3", "pass31")
        return {k: (p[i], c[i]) for i, k in enumerate(kinds)}, tot.value

    def dipole(self, eid: int, with_xy: bool = False):
        """(S_bins, r_bins, counts, Q_s[, S_xy]) from the event's accumulated correlator."""
        N = self.N[eid]
        nb = N // 2 + 1
        sb, rb = np.empty(nb), np.empty(nb)
        cb = np.empty(nb, np.int32)
        q = ctypes.c_double(0)
        n = ctypes.c_int(0)
        sxy = np.empty((N, N)) if with_xy else None
        _ck(_lib.jw_engine_dipole(self._h, eid, sxy.ctypes.data_as(_dp) if with_xy else None, sb.ctypes.data_as(_dp),
                                  rb.ctypes.data_as(_dp), cb.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), nb,
                                  ctypes.byref(n), ctypes.byref(q)), "jw_engine_dipole")
        out = (sb, rb, cb, q.value)
        return out + (sxy,) if with_xy else out


class Server:
    """Continuous-batching evolution server (jw_server_*)."""

    def __init__(self, precision: int = PRECISION_MIXED, max_bytes: int = 0, max_steps_per_tick: int = 8,
                 max_active: int = 0, reunitarize: bool = False, fake_device: bool = False,
                 fake_ns_per_site_step: float = 0.0, device: int = 0, tick_sites: int = 0):
        o = jw_server_options(precision, int(reunitarize), max_bytes, max_steps_per_tick, max_active,
                              int(fake_device), fake_ns_per_site_step, tick_sites)
        self._h = _vp()
        _ck(_lib.jw_server_create(ctypes.byref(o), device, ctypes.byref(self._h)), "jw_server_create")

    def close(self):
        if self._h:
            _lib.jw_server_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, N: int, steps: int, ny_slices: int = 50, mu: float | None = None, mass: float = 0.04,
               step: float = 0.0004, coupling: int = FIXED_COUPLING_CONSTANT, kernel: int = SIN_KERNEL,
               seed: int = 1) -> int:
        d = jw_request_desc(N, ny_slices, 0.5 * N if mu is None else mu, mass, step, coupling, kernel, seed, steps)
        rid = ctypes.c_int64(-1)
        _ck(_lib.jw_server_submit(self._h, ctypes.byref(d), ctypes.byref(rid)), "jw_server_submit")
        return rid.value

    def try_submit(self, **kw):
        N = kw["N"]
        d = jw_request_desc(N, kw.get("ny_slices", 50), kw.get("mu", 0.5 * N), kw.get("mass", 0.04),
                            kw.get("step", 0.0004), kw.get("coupling", FIXED_COUPLING_CONSTANT),
                            kw.get("kernel", SIN_KERNEL), kw.get("seed", 1), kw.get("steps", 1))
        rid = ctypes.c_int64(-1)
        st = _lib.jw_server_submit(self._h, ctypes.byref(d), ctypes.byref(rid))
        return st, rid.value

    def wait(self, rid: int, timeout: float = 600.0):
        """(status, result struct, S_bins, r_bins); raises on JW_ETIMEOUT / unknown id."""
        res = jw_request_result()
        cap = 2048 // 2 + 1
        sb, rb = np.zeros(cap), np.zeros(cap)
        _ck(_lib.jw_server_wait(self._h, rid, timeout, ctypes.byref(res), sb.ctypes.data_as(_dp),
                                rb.ctypes.data_as(_dp), cap), "jw_server_wait")
        return res.status, res, sb[:res.nbins].copy(), rb[:res.nbins].copy()

    def try_wait(self, rid: int, timeout: float):
        res = jw_request_result()
        return _lib.jw_server_wait(self._h, rid, timeout, ctypes.byref(res), None, None, 0), res

    def stats(self) -> jw_server_stats:
        st = jw_server_stats()
        _ck(_lib.jw_server_get_stats(self._h, ctypes.byref(st)), "jw_server_get_stats")
        return st

    def size_stats(self) -> dict:
        """{N: dict(site_steps, step_ms, mv_ms, ticks)} per lattice size served so far."""
        cnt = ctypes.c_int(0)
        _ck(_lib.jw_server_size_stats(self._h, None, None, None, None, None, 0, ctypes.byref(cnt)),
            "jw_server_size_stats")
        n = cnt.value
        Ns = (ctypes.c_int * max(n, 1))()
        ss, sm, mm = ((ctypes.c_double * max(n, 1))() for _ in range(3))
        tk = (ctypes.c_int64 * max(n, 1))()
        _ck(_lib.jw_server_size_stats(self._h, Ns, ss, sm, mm, tk, n, ctypes.byref(cnt)), "jw_server_size_stats")
        return {Ns[i]: dict(site_steps=ss[i], step_ms=sm[i], mv_ms=mm[i], ticks=tk[i]) for i in range(min(n, cnt.value))}
