"""Python host mirror of the reference's interface, over the C ABI of
libquasi_gpu.so (ctypes; plain pointers and sizes).

The reference exposes no API: its state lives in main() of quasi/quasi.cpp.
``Simulation`` names its methods after the reference's phases (set the
initial psi, the pre-loop, the time loop, the diagnostics and dumps) and
``R2RPlan`` mirrors ``fftw_mpi_plan_r2r_3d`` / ``fftw_execute``.

There is no CPU fallback: if the shared library or a CUDA device is missing,
every call raises.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "libquasi_gpu.so"

VARIANT = {"quasi": 0, "stb": 1}
PRECISION = {"fp64": 0, "fp32": 1, "bf16x3": 2}
FIELD = {"psi": 0, "rho": 1, "vx": 2, "vy": 3, "vz": 4, "p": 5, "divv": 6, "psiq": 7, "psiq_old": 8,
         "dtpsi": 9, "df": 10}
KIND = {"REDFT10": 0, "REDFT01": 1, "RODFT10": 2, "RODFT01": 3}
PLAN_KINDS = {
    "CT": (0, 0, 0), "iCT": (1, 1, 1), "STx": (2, 0, 0), "STy": (0, 2, 0), "STz": (0, 0, 2),
    "iSTx": (3, 1, 1), "iSTy": (1, 3, 1), "iSTz": (1, 1, 3),
}

# Every entry point of include/quasi_gpu.h
EXPORTS = [
    "quasi_abi_version", "quasi_last_error", "quasi_config_default", "quasi_create", "quasi_destroy",
    "quasi_set_psi", "quasi_init", "quasi_step", "quasi_step_timed", "quasi_step_count", "quasi_get_field",
    "quasi_diagnostics", "quasi_growth_rate", "quasi_save", "quasi_load", "quasi_r2r_plan_create",
    "quasi_r2r_execute_device", "quasi_r2r_execute_host", "quasi_r2r_plan_destroy",
    "quasi_ic_default", "quasi_initial_condition", "quasi_step_kernels", "quasi_time_axis_pass",
    "quasi_step_async", "quasi_synchronize", "quasi_diagnostics_noalloc", "quasi_r2r_inject_wait_timeout",
    "quasi_tuning",
    "quasi_ensemble_create", "quasi_ensemble_size", "quasi_ensemble_member", "quasi_ensemble_init",
    "quasi_ensemble_step", "quasi_ensemble_growth_rates", "quasi_ensemble_destroy",
]
IC_KIND = {"planar": 0, "undulated": 1, "interface": 2, "droplet": 3, "stb": 4, "focal_conic": 5}


class QuasiError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libquasi_gpu error {code}: {msg}")
        self.code = code


class Config(ctypes.Structure):
    """``struct quasi_config`` (include/quasi_gpu.h)."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("variant", ctypes.c_int), ("precision", ctypes.c_int), ("emulate_ranks", ctypes.c_int),
        ("device", ctypes.c_int),
        ("nu_arg", ctypes.c_double), ("ep_arg", ctypes.c_double),
        ("gamma", ctypes.c_double), ("beta", ctypes.c_double), ("alpha", ctypes.c_double), ("q0", ctypes.c_double),
        ("amp", ctypes.c_double), ("rho_0", ctypes.c_double), ("kp", ctypes.c_double), ("rho_m", ctypes.c_double),
        ("dt", ctypes.c_double), ("nw", ctypes.c_int), ("divv_switch", ctypes.c_int), ("q_pert", ctypes.c_double),
        ("autotune", ctypes.c_int),
    ]


class IC(ctypes.Structure):
    """``struct quasi_ic`` (include/quasi_gpu.h)."""
    _fields_ = [
        ("kind", ctypes.c_int), ("seed", ctypes.c_ulonglong), ("noise", ctypes.c_double),
        ("delta", ctypes.c_double), ("eps_h", ctypes.c_double), ("q_h", ctypes.c_double),
        ("radius_frac", ctypes.c_double), ("width_wavelengths", ctypes.c_double), ("amp0", ctypes.c_double),
        ("fc_size", ctypes.c_double),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libquasi_gpu.so once.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise QuasiError(-6, f"{LIB_PATH} is missing: build it with python -m smaiso_quasi_b200.build")
        L = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        L.quasi_last_error.restype = ctypes.c_char_p
        L.quasi_config_default.argtypes = [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int]
        L.quasi_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]
        L.quasi_destroy.argtypes = [ctypes.c_void_p]
        L.quasi_set_psi.argtypes = [ctypes.c_void_p, dp]
        L.quasi_init.argtypes = [ctypes.c_void_p]
        L.quasi_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.quasi_step_timed.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.quasi_step_async.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.quasi_synchronize.argtypes = [ctypes.c_void_p]
        L.quasi_step_count.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        L.quasi_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.quasi_diagnostics.argtypes = [ctypes.c_void_p, dp]
        L.quasi_growth_rate.argtypes = [ctypes.c_void_p, dp]
        L.quasi_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.quasi_load.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.quasi_r2r_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                            ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.quasi_r2r_execute_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.quasi_r2r_execute_host.argtypes = [ctypes.c_void_p, dp, dp]
        L.quasi_r2r_plan_destroy.argtypes = [ctypes.c_void_p]
        L.quasi_r2r_inject_wait_timeout.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint]
        L.quasi_step_kernels.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.quasi_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.quasi_time_axis_pass.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.quasi_ic_default.argtypes = [ctypes.POINTER(IC), ctypes.c_int]
        L.quasi_initial_condition.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(IC), dp]
        L.quasi_ensemble_create.argtypes = [ctypes.c_int, ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]
        L.quasi_ensemble_size.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.quasi_ensemble_member.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.quasi_ensemble_init.argtypes = [ctypes.c_void_p]
        L.quasi_ensemble_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.quasi_ensemble_growth_rates.argtypes = [ctypes.c_void_p, dp]
        L.quasi_ensemble_destroy.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise QuasiError(rc, lib().quasi_last_error().decode(errors="replace"))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def default_config(variant: str = "quasi", nx: int = 64, ny: int = 64, nz: int = 128, **overrides) -> Config:
    c = Config()
    _check(lib().quasi_config_default(ctypes.byref(c), VARIANT[variant], nx, ny, nz))
    for k, v in overrides.items():
        if k == "precision" and isinstance(v, str):
            v = PRECISION[v]
        setattr(c, k, v)
    return c


def initial_condition(cfg: Config, kind: str = "planar", **params) -> np.ndarray:
    """Seeded initial psi computed by the library's host code (no device)."""
    ic = IC()
    _check(lib().quasi_ic_default(ctypes.byref(ic), IC_KIND[kind]))
    for k, v in params.items():
        setattr(ic, k, v)
    out = np.empty((cfg.nx, cfg.ny, cfg.nz), dtype=np.float64)
    _check(lib().quasi_initial_condition(ctypes.byref(cfg), ctypes.byref(ic), _dptr(out)))
    return out


class Simulation:
    """One instance of the step on one GPU (a ``quasi_handle``)."""

    def __init__(self, cfg: Config, _handle=None, _owner=None):
        self.cfg = cfg
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self._owner = _owner   # an Ensemble that owns the handle, else None
        if _handle is not None:
            self._h = _handle
            return
        h = ctypes.c_void_p()
        _check(lib().quasi_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            if self._owner is None:
                lib().quasi_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_psi(self, psi: np.ndarray) -> None:
        a = np.ascontiguousarray(psi, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"psi shape {a.shape} != grid {self.shape}")
        _check(lib().quasi_set_psi(self._h, _dptr(a)))

    def init(self) -> None:
        _check(lib().quasi_init(self._h))

    def step(self, n: int = 1) -> None:
        _check(lib().quasi_step(self._h, int(n)))

    def step_async(self, n: int = 1) -> None:
        """Enqueue n steps and return (see synchronize)."""
        _check(lib().quasi_step_async(self._h, int(n)))

    def synchronize(self) -> None:
        _check(lib().quasi_synchronize(self._h))

    def step_timed(self, n: int) -> float:
        ms = ctypes.c_double()
        _check(lib().quasi_step_timed(self._h, int(n), ctypes.byref(ms)))
        return ms.value

    @property
    def nloop(self) -> int:
        v = ctypes.c_long()
        _check(lib().quasi_step_count(self._h, ctypes.byref(v)))
        return v.value

    def step_kernels(self) -> int:
        n = ctypes.c_int()
        _check(lib().quasi_step_kernels(self._h, ctypes.byref(n)))
        return n.value

    def tuning(self) -> dict:
        """The autotuner's choices (quasi_tuning)."""
        out = (ctypes.c_int * 4)()
        _check(lib().quasi_tuning(self._h, out))
        names = ("z", "x", "y")
        return {"warp_tiles_float": [n for b, n in enumerate(names) if out[0] >> b & 1],
                "warp_tiles_double": [n for b, n in enumerate(names) if out[1] >> b & 1],
                "tensor_core_axes": int(out[2]), "measured": bool(out[3])}

    def time_axis_pass(self, axis: int, reps: int = 20) -> float:
        ms = ctypes.c_double()
        _check(lib().quasi_time_axis_pass(self._h, int(axis), int(reps), ctypes.byref(ms)))
        return ms.value

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        _check(lib().quasi_get_field(self._h, FIELD[name], _dptr(out)))
        return out

    def diagnostics(self) -> tuple[float, float, float]:
        out = np.zeros(3)
        _check(lib().quasi_diagnostics(self._h, _dptr(out)))
        return float(out[0]), float(out[1]), float(out[2])

    def growth_rate(self) -> float:
        v = ctypes.c_double()
        _check(lib().quasi_growth_rate(self._h, ctypes.byref(v)))
        return v.value

    def save(self, path: str) -> None:
        _check(lib().quasi_save(self._h, str(path).encode()))

    def load(self, path: str) -> None:
        _check(lib().quasi_load(self._h, str(path).encode()))


class Ensemble:
    """Independent instances stepped together (a ``quasi_ensemble``): every
    member's steps are enqueued on its own stream before any is waited for.
    ``members[m]`` is a Simulation view of member m (owned by the ensemble)."""

    def __init__(self, configs: list[Config]):
        arr = (Config * len(configs))(*configs)
        h = ctypes.c_void_p()
        _check(lib().quasi_ensemble_create(len(configs), arr, ctypes.byref(h)))
        self._h = h
        self.members = []
        for m, cfg in enumerate(configs):
            mh = ctypes.c_void_p()
            _check(lib().quasi_ensemble_member(self._h, m, ctypes.byref(mh)))
            self.members.append(Simulation(cfg, _handle=mh, _owner=self))

    def __len__(self) -> int:
        n = ctypes.c_int()
        _check(lib().quasi_ensemble_size(self._h, ctypes.byref(n)))
        return n.value

    def init(self) -> None:
        _check(lib().quasi_ensemble_init(self._h))

    def step(self, n: int = 1) -> None:
        _check(lib().quasi_ensemble_step(self._h, int(n)))

    def growth_rates(self) -> np.ndarray:
        out = np.zeros(len(self.members))
        _check(lib().quasi_ensemble_growth_rates(self._h, _dptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            for s in self.members:
                s._h = None
            lib().quasi_ensemble_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class R2RPlan:
    """``fftw_mpi_plan_r2r_3d`` counterpart: one in-place 3-D r2r transform."""

    def __init__(self, nx: int, ny: int, nz: int, kinds, precision: str = "fp64", device: int = 0):
        if isinstance(kinds, str):
            kinds = PLAN_KINDS[kinds]
        k = (ctypes.c_int * 3)(*[KIND[x] if isinstance(x, str) else int(x) for x in kinds])
        p = ctypes.c_void_p()
        _check(lib().quasi_r2r_plan_create(nx, ny, nz, k, PRECISION[precision], device, ctypes.byref(p)))
        self._p = p
        self.shape = (nx, ny, nz)

    def execute_host(self, a: np.ndarray) -> np.ndarray:
        src = np.ascontiguousarray(a, dtype=np.float64)
        out = np.empty(self.shape, dtype=np.float64)
        _check(lib().quasi_r2r_execute_host(self._p, _dptr(src), _dptr(out)))
        return out

    def execute_device(self, data_ptr: int, stream: int | None = None) -> None:
        _check(lib().quasi_r2r_execute_device(self._p, ctypes.c_void_p(data_ptr),
                                              ctypes.c_void_p(stream) if stream else None))

    def inject_wait_timeout(self, skip_tile: int = 0, poll_limit: int = 64) -> None:
        """Failure-detection test hook: the next execution skips one tile's
        copy and raises QuasiError(QUASI_ERR_TIMEOUT)."""
        _check(lib().quasi_r2r_inject_wait_timeout(self._p, int(skip_tile), int(poll_limit)))

    def close(self) -> None:
        if getattr(self, "_p", None):
            lib().quasi_r2r_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
