"""Python binding of the crp C ABI (include/crp.h), for tests and benchmarks.

The simulation itself runs in the CUDA library ``libcrp.so`` built from
``cuda-rp_b200/csrc``; this module only loads it with ctypes and converts
arrays.  There is no Python or CPU fallback: if the library is missing,
``load()`` raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "build", "libcrp.so")

c_int = ctypes.c_int32
c_dbl = ctypes.c_double


class Config(ctypes.Structure):
    """Mirror of struct crp_config."""

    _fields_ = [
        ("grid_x", c_int), ("grid_y", c_int), ("grid_lx", c_dbl), ("grid_ly", c_dbl),
        ("pml_x0", c_int), ("pml_x1", c_int), ("pml_y0", c_int), ("pml_y1", c_int),
        ("pml_grid_number", c_int), ("pml_sigma", c_dbl), ("pml_order", c_int),
        ("sim_cfl", c_dbl), ("sim_dt0", c_dbl), ("sim_n_step_max", c_int), ("sim_t_step_max", c_dbl),
        ("sim_save_interval", c_int), ("sim_order", c_int), ("sim_smooth_delta_band", c_int),
        ("tr_amp", c_dbl), ("tr_freq", c_dbl), ("tr_focal_dist", c_dbl),
        ("tr_pid", c_int), ("tr_pid_start_step", c_int), ("tr_init_control", c_dbl),
        ("tr_pid_iterate", c_int), ("tr_box_size", c_dbl), ("tr_cylindrical", c_int),
        ("tr_on_wave", c_int), ("tr_off_wave", c_int),
        ("tr_plane_v", c_int), ("tr_plane_p", c_int), ("tr_focused_v", c_int), ("tr_focused_p", c_int),
        ("bub_enable", c_int), ("bub_fg0", c_dbl), ("bub_R0", c_dbl), ("bub_P0", c_dbl),
        ("bub_T0", c_dbl), ("bub_gamma", c_dbl), ("bub_sigma", c_dbl), ("bub_mu", c_dbl),
        ("bub_rho", c_dbl), ("bub_K0", c_dbl),
        ("dbg_display", c_int), ("dbg_fg", c_int), ("dbg_T", c_int), ("dbg_p", c_int),
        ("dbg_v", c_int), ("dbg_bubbles", c_int),
        ("opt_ascii", c_int), ("opt_sph", c_int),
        ("ext_rho_inf", c_dbl), ("ext_c_inf", c_dbl), ("ext_p_inf", c_dbl),
        ("ext_source_row", c_int), ("ext_ramp_cycles", c_dbl), ("ext_precision", c_int),
        ("ext_picard_cap", c_int), ("ext_rp_step_cap", c_int), ("ext_bubble_count", c_int),
        ("ext_bubble_seed", ctypes.c_uint64), ("ext_r0_sigma_ln", c_dbl), ("ext_cloud_shape", c_int),
        ("ext_cloud_r", c_dbl), ("ext_cloud_h", c_dbl), ("ext_n_b", c_dbl), ("ext_picard_tol", c_dbl),
        ("ext_graphs", c_int), ("ext_elements", c_int), ("ext_rp_scheme", c_int), ("ext_rp_tol", c_dbl),
        ("ext_grid_z", c_int), ("ext_grid_lz", c_dbl), ("ext_pml_z0", c_int), ("ext_pml_z1", c_int),
        ("ext_array_elements", c_int), ("ext_array_radius", c_dbl), ("ext_array_focus_dx", c_dbl),
        ("ext_array_seed", ctypes.c_uint64), ("ext_array_phases", c_int), ("ext_rp_reuse", c_int),
    ]


class Dims(ctypes.Structure):
    _fields_ = [("i1m", c_int), ("j1m", c_int), ("i2m", c_int), ("j2m", c_int), ("i2n", c_int),
                ("j2n", c_int), ("num_bubbles", c_int), ("dx", c_dbl), ("dy", c_dbl), ("dt", c_dbl)]


class Dims3(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int), ("num_bubbles", c_int), ("dx", c_dbl), ("dy", c_dbl),
                ("dz", c_dbl), ("dt", c_dbl), ("source_cells", c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("fdtd_rows", c_int), ("rp_blocks", c_int), ("rp_blocks_max", c_int)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("mode", c_int), ("threads", c_int), ("blocking", c_int), ("fdtd_rows", c_int),
                ("rp_bubbles_per_lane", c_int), ("ms_per_step", c_dbl)]

    def as_dict(self) -> dict:
        return {"mode": ["threads", "graphs"][self.mode], "threads": self.threads, "blocking": self.blocking,
                "fdtd_rows": self.fdtd_rows, "rp_bubbles_per_lane": self.rp_bubbles_per_lane,
                "ms_per_step": self.ms_per_step}


BATCH_THREADS, BATCH_GRAPHS = 0, 1


class Stats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("time", c_dbl), ("picard_total", ctypes.c_int64),
                ("picard_last", c_int), ("picard_max", c_int), ("rp_substeps_max", ctypes.c_int64),
                ("residual_last", c_dbl), ("kernel_launches", ctypes.c_int64), ("fdtd_launches", ctypes.c_int64),
                ("rp_launches", ctypes.c_int64), ("couple_launches", ctypes.c_int64),
                ("ms_fdtd", c_dbl), ("ms_rp", c_dbl), ("ms_couple", c_dbl), ("ms_other", c_dbl),
                ("picard_stalls", ctypes.c_int64), ("rp_reused", ctypes.c_int64)]


PROGRESS = ctypes.CFUNCTYPE(None, ctypes.c_int64, c_dbl, ctypes.c_void_p)


class Objective(ctypes.Structure):
    """crp_objective: steps to run and differentiate over, focal radius [m]."""
    _fields_ = [("steps", c_int), ("focal_radius", c_dbl)]


class FocusState(ctypes.Structure):
    _fields_ = [("control_x", c_dbl), ("control_y", c_dbl), ("err_total_x", c_dbl), ("err_total_y", c_dbl),
                ("d_err_x", c_dbl), ("d_err_y", c_dbl), ("filter_in", c_dbl * 5), ("filter_out", c_dbl * 5)]


class OutputPlan(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int64), ("t_max", c_dbl), ("save_interval", c_int),
                ("dir", ctypes.c_char_p), ("sph", c_int), ("progress", PROGRESS), ("user", ctypes.c_void_p)]


class BubblesIn(ctypes.Structure):
    _fields_ = [("n", c_int), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("r0", ctypes.c_void_p),
                ("n_b", ctypes.c_void_p), ("z", ctypes.c_void_p)]


FIELDS = {"p0": 0, "px": 1, "py": 2, "pnx": 3, "pny": 4, "vx": 5, "vy": 6, "f_g": 7, "f_gn": 8, "T": 11,
          "f_gm": 9, "rho_m": 10, "vz": 12, "pz": 13}
BUBBLE_FIELDS = {"x": 0, "y": 1, "R_t": 2, "R_p": 3, "R_n": 4, "d1_R_p": 5, "PG_p": 6, "PL_p": 7,
                 "PL_n": 8, "PL_m": 9, "dt": 10, "re": 11, "Q_B": 12, "n_B": 13, "R0": 14, "v_x": 15,
                 "v_y": 16, "ibm_x": 17, "ibm_y": 18, "ibn_x": 19, "ibn_y": 20, "substeps": 21,
                 "z": 22, "v_z": 23, "ibm_z": 24, "ibn_z": 25}


class CrpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"crp status {status}: {msg}")
        self.status = status


def field_shape(dims, name: str) -> tuple[int, int]:
    """(height, width) of a field's dense array in the reference's layout."""
    if name in ("p0", "px", "py", "pnx", "pny", "rho_m"):
        return dims.j1m, dims.i1m
    if name == "vx":
        return dims.j2m, dims.i2n
    if name == "vy":
        return dims.j2n, dims.i2m
    return dims.j2m, dims.i2m


def field_shape3(d3, name: str) -> tuple[int, int, int]:
    """(depth, height, width) of a 3-D field's dense array (x fastest)."""
    nz, ny, nx = d3.nz, d3.ny, d3.nx
    return {"vx": (nz, ny, nx + 1), "vy": (nz, ny + 1, nx), "vz": (nz + 1, ny, nx)}.get(name, (nz, ny, nx))


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return a.ctypes.data_as(ctypes.c_void_p)


_lib = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Load libcrp.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"libcrp.so not built at {path}; run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sigs = {
        "crp_config_defaults": (c_int, [P(Config)]),
        "crp_config_parse_file": (c_int, [ctypes.c_char_p, P(Config), ctypes.c_char_p, ctypes.c_size_t]),
        "crp_config_parse_string": (c_int, [ctypes.c_char_p, P(Config), ctypes.c_char_p, ctypes.c_size_t]),
        "crp_seed_bubbles": (c_int, [P(Config), vp, vp, vp, vp]),
        "crp_seed_bubbles3": (c_int, [P(Config), vp, vp, vp, vp, vp]),
        "crp_get_dims3": (c_int, [vp, P(Dims3)]),
        "crp_create": (c_int, [P(Config), P(BubblesIn), vp, P(vp)]),
        "crp_step": (c_int, [vp, c_int]),
        "crp_get_dims": (c_int, [vp, P(Dims)]),
        "crp_get_stats": (c_int, [vp, P(Stats)]),
        "crp_read_field": (c_int, [vp, c_int, vp]),
        "crp_read_bubbles": (c_int, [vp, c_int, vp]),
        "crp_write_rawdata": (c_int, [vp, ctypes.c_char_p]),
        "crp_write_sph": (c_int, [vp, ctypes.c_char_p]),
        "crp_stream": (vp, [vp]),
        "crp_set_profiling": (c_int, [vp, c_int]),
        "crp_minmax": (c_int, [vp, P(c_dbl), P(c_dbl), P(c_dbl), P(c_dbl)]),
        "crp_last_error": (ctypes.c_char_p, [vp]),
        "crp_status_string": (ctypes.c_char_p, [c_int]),
        "crp_destroy": (None, [vp]),
        "crp_void_fraction_noalloc_scratch": (ctypes.c_size_t, [c_int, c_int, c_int]),
        "crp_void_fraction_noalloc": (c_int, [P(Config), c_int, vp, vp, vp, vp, vp, vp]),
        "crp_run": (c_int, [vp, P(OutputPlan), P(Config)]),
        "crp_focus_history": (ctypes.c_int64, [vp, c_int, vp, ctypes.c_int64]),
        "crp_get_focus_state": (c_int, [vp, P(FocusState)]),
        "crp_set_focus_state": (c_int, [vp, P(FocusState)]),
        "crp_set_source_elements": (c_int, [vp, c_int, vp, vp]),
        "crp_adjoint": (c_int, [vp, P(Objective), P(c_dbl), vp, vp]),
        "crp_batch_create": (c_int, [c_int, P(Config), P(BubblesIn), P(vp)]),
        "crp_batch_run": (c_int, [vp, P(c_int), c_int, P(c_int)]),
        "crp_batch_count": (c_int, [vp]),
        "crp_batch_sim": (vp, [vp, c_int]),
        "crp_batch_destroy": (None, [vp]),
        "crp_state_bytes": (ctypes.c_size_t, [vp]),
        "crp_save_state": (c_int, [vp, P(vp)]),
        "crp_load_state": (c_int, [vp, vp]),
        "crp_state_free": (None, [vp]),
        "crp_get_tuning": (c_int, [vp, P(Tuning)]),
        "crp_set_tuning": (c_int, [vp, P(Tuning)]),
        "crp_batch_get_tuning": (c_int, [vp, P(BatchTuning)]),
        "crp_batch_set_tuning": (c_int, [vp, P(BatchTuning)]),
        "crp_batch_tune": (c_int, [vp, c_int, P(BatchTuning), P(BatchTuning), c_int, P(c_int)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def defaults() -> Config:
    cfg = Config()
    load().crp_config_defaults(ctypes.byref(cfg))
    return cfg


def parse_string(text: str, cfg: Config | None = None) -> Config:
    cfg = cfg if cfg is not None else defaults()
    err = ctypes.create_string_buffer(512)
    st = load().crp_config_parse_string(text.encode(), ctypes.byref(cfg), err, 512)
    if st:
        raise CrpError(st, err.value.decode())
    return cfg


def parse_file(path: str, cfg: Config | None = None) -> Config:
    cfg = cfg if cfg is not None else defaults()
    err = ctypes.create_string_buffer(512)
    st = load().crp_config_parse_file(path.encode(), ctypes.byref(cfg), err, 512)
    if st:
        raise CrpError(st, err.value.decode())
    return cfg


@dataclass
class Bubbles:
    x: np.ndarray
    y: np.ndarray
    r0: np.ndarray
    n_b: np.ndarray
    z: np.ndarray | None = None  # 3-D grids only

    def as_c(self) -> BubblesIn:
        arrays = (self.x, self.y, self.r0, self.n_b) + ((self.z,) if self.z is not None else ())
        for a in arrays:
            assert a.dtype == np.float64 and a.flags.c_contiguous
        return BubblesIn(len(self.x), _ptr(self.x), _ptr(self.y), _ptr(self.r0), _ptr(self.n_b),
                         _ptr(self.z) if self.z is not None else None)


def seed_bubbles(cfg: Config) -> Bubbles:
    n = cfg.ext_bubble_count
    arrs = [np.zeros(n) for _ in range(4)]
    st = load().crp_seed_bubbles(ctypes.byref(cfg), *[_ptr(a) for a in arrs])
    if st:
        raise CrpError(st, "crp_seed_bubbles")
    return Bubbles(*arrs)


def seed_bubbles3(cfg: Config) -> Bubbles:
    n = cfg.ext_bubble_count
    x, y, z, r0, nb = (np.zeros(n) for _ in range(5))
    st = load().crp_seed_bubbles3(ctypes.byref(cfg), _ptr(x), _ptr(y), _ptr(z), _ptr(r0), _ptr(nb))
    if st:
        raise CrpError(st, "crp_seed_bubbles3")
    return Bubbles(x, y, r0, nb, z)


class Sim:
    """A simulation on the current CUDA device (one crp_sim handle)."""

    def __init__(self, cfg: Config, bubbles: Bubbles | None = None, stream: int | None = None):
        self.lib = load()
        self._keep = (cfg, bubbles)
        h = ctypes.c_void_p()
        bin_ = bubbles.as_c() if bubbles is not None else None
        st = self.lib.crp_create(ctypes.byref(cfg), ctypes.byref(bin_) if bin_ is not None else None,
                                 ctypes.c_void_p(stream) if stream else None, ctypes.byref(h))
        if st:
            raise CrpError(st, self.lib.crp_status_string(st).decode())
        self.h = h
        self.dims = Dims()
        self._check(self.lib.crp_get_dims(self.h, ctypes.byref(self.dims)))
        self.dims3 = None
        if cfg.ext_grid_z > 0:
            self.dims3 = Dims3()
            self._check(self.lib.crp_get_dims3(self.h, ctypes.byref(self.dims3)))

    def _check(self, st: int):
        if st:
            msg = self.lib.crp_last_error(self.h)
            raise CrpError(st, (msg or b"").decode() or self.lib.crp_status_string(st).decode())

    def step(self, n: int = 1):
        self._check(self.lib.crp_step(self.h, n))

    def stats(self) -> Stats:
        s = Stats()
        self._check(self.lib.crp_get_stats(self.h, ctypes.byref(s)))
        return s

    def save_state(self, into: "State | None" = None) -> "State":
        """Snapshot of the whole simulation state (crp_save_state); `into`, a
        snapshot of this simulation, is overwritten instead of allocating."""
        st = into if into is not None else State(self.lib)
        self._check(self.lib.crp_save_state(self.h, ctypes.byref(st.h)))
        return st

    def load_state(self, st: "State"):
        self._check(self.lib.crp_load_state(self.h, st.h))

    @property
    def tuning(self) -> Tuning:
        t = Tuning()
        self._check(self.lib.crp_get_tuning(self.h, ctypes.byref(t)))
        return t

    @tuning.setter
    def tuning(self, t: Tuning):
        self._check(self.lib.crp_set_tuning(self.h, ctypes.byref(t)))

    def field(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Dense copy of a field; into `out` (float64, C-contiguous, the field's
        shape) when given, e.g. a pinned host buffer."""
        shape = field_shape3(self.dims3, name) if self.dims3 is not None else field_shape(self.dims, name)
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        assert out.shape == shape and out.dtype == np.float64 and out.flags.c_contiguous
        self._check(self.lib.crp_read_field(self.h, FIELDS[name], _ptr(out)))
        return out

    def bubbles(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """One bubble quantity; into `out` (float64, num_bubbles) when given."""
        if out is None:
            out = np.empty(self.dims.num_bubbles, dtype=np.float64)
        assert out.shape == (self.dims.num_bubbles,) and out.dtype == np.float64 and out.flags.c_contiguous
        self._check(self.lib.crp_read_bubbles(self.h, BUBBLE_FIELDS[name], _ptr(out)))
        return out

    def run(self, n_steps: int = 0, t_max: float = 0.0, save_interval: int = 0, directory: str | None = None,
            progress=None):
        """crp_run: step to the limits (config's n_step_max/t_step_max when both
        are 0), writing rawdata every save_interval steps into directory."""
        cb = PROGRESS(lambda step, t, user: progress(step, t)) if progress else PROGRESS()
        plan = OutputPlan(n_steps, t_max, save_interval, directory.encode() if directory else None, 0, cb, None)
        cfg = self._keep[0]
        self._check(self.lib.crp_run(self.h, ctypes.byref(plan), ctypes.byref(cfg) if cfg is not None else None))

    def focus_history(self, which: str = "actual") -> np.ndarray:
        """Tracked focal depths ("actual") or control depths ("control")."""
        w = 0 if which == "actual" else 1
        n = self.lib.crp_focus_history(self.h, w, None, 0)
        out = np.zeros(max(n, 0))
        if n > 0:
            self.lib.crp_focus_history(self.h, w, _ptr(out), n)
        return out

    def focus_state(self) -> FocusState:
        st = FocusState()
        self._check(self.lib.crp_get_focus_state(self.h, ctypes.byref(st)))
        return st

    def set_focus_state(self, st: FocusState):
        self._check(self.lib.crp_set_focus_state(self.h, ctypes.byref(st)))

    def set_source_elements(self, amp, phase):
        """Amplitude factors and phase offsets of the cfg.ext_elements source elements."""
        a = np.ascontiguousarray(amp, dtype=np.float64)
        p = np.ascontiguousarray(phase, dtype=np.float64)
        assert a.shape == p.shape and a.ndim == 1
        self._check(self.lib.crp_set_source_elements(self.h, int(a.size), _ptr(a), _ptr(p)))

    def adjoint(self, steps: int, focal_radius: float, n_elements: int = 0):
        """Advance `steps` steps and return (J, dJ/d amplitudes, dJ/d phases) of
        the focal objective (crp_adjoint); the gradients are None without elements."""
        obj = Objective(int(steps), float(focal_radius))
        J = c_dbl(0.0)
        ga = np.zeros(n_elements) if n_elements > 0 else None
        gp = np.zeros(n_elements) if n_elements > 0 else None
        self._check(self.lib.crp_adjoint(self.h, ctypes.byref(obj), ctypes.byref(J),
                                         _ptr(ga) if ga is not None else None,
                                         _ptr(gp) if gp is not None else None))
        return J.value, ga, gp

    def write_sph(self, directory: str):
        self._check(self.lib.crp_write_sph(self.h, directory.encode()))

    def write_rawdata(self, directory: str):
        self._check(self.lib.crp_write_rawdata(self.h, directory.encode()))

    def set_profiling(self, on: bool):
        self._check(self.lib.crp_set_profiling(self.h, 1 if on else 0))

    @property
    def stream(self) -> int:
        return self.lib.crp_stream(self.h) or 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.crp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class State:
    """A snapshot taken by Sim.save_state (device memory, freed with the object)."""

    def __init__(self, lib):
        self.lib = lib
        self.h = ctypes.c_void_p()

    def free(self):
        if getattr(self, "h", None):
            self.lib.crp_state_free(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        self.free()


class _BatchSim(Sim):
    """A simulation owned by a Batch (not destroyed on its own)."""

    def __init__(self, lib, h, keep):
        self.lib = lib
        self._keep = keep
        self.h = ctypes.c_void_p(h)
        self.dims = Dims()
        self._check(self.lib.crp_get_dims(self.h, ctypes.byref(self.dims)))
        self.dims3 = None
        if keep[0].ext_grid_z > 0:
            self.dims3 = Dims3()
            self._check(self.lib.crp_get_dims3(self.h, ctypes.byref(self.dims3)))

    def close(self):
        self.h = None


class Batch:
    """Independent simulations advanced concurrently (crp_batch)."""

    def __init__(self, cfgs: list[Config], bubbles: list[Bubbles | None] | None = None):
        self.lib = load()
        n = len(cfgs)
        self._cfgs = (Config * n)(*cfgs)
        bubbles = bubbles or [None] * n
        self._bub = bubbles
        self._bin = (BubblesIn * n)(*[b.as_c() if b is not None else BubblesIn() for b in bubbles])
        h = ctypes.c_void_p()
        st = self.lib.crp_batch_create(n, self._cfgs, self._bin, ctypes.byref(h))
        if st:
            raise CrpError(st, self.lib.crp_status_string(st).decode())
        self.h = h
        self.sims = [_BatchSim(self.lib, self.lib.crp_batch_sim(self.h, k), (cfgs[k], bubbles[k])) for k in range(n)]

    def run(self, steps: list[int], threads: int = 0) -> list[int]:
        n = len(self.sims)
        st_arr = (c_int * n)()
        st = self.lib.crp_batch_run(self.h, (c_int * n)(*steps), threads, st_arr)
        per = list(st_arr)
        if st:
            bad = [k for k, v in enumerate(per) if v]
            raise CrpError(st, f"simulations {bad} failed: {self.lib.crp_status_string(st).decode()}")
        return per

    @property
    def tuning(self) -> BatchTuning:
        t = BatchTuning()
        self._check(self.lib.crp_batch_get_tuning(self.h, ctypes.byref(t)))
        return t

    @tuning.setter
    def tuning(self, t: BatchTuning):
        self._check(self.lib.crp_batch_set_tuning(self.h, ctypes.byref(t)))

    def tune(self, trial_steps: int = 10) -> tuple[BatchTuning, list[BatchTuning]]:
        """crp_batch_tune: the fastest setting (applied) and every setting timed."""
        best, tried, n = BatchTuning(), (BatchTuning * 16)(), c_int()
        self._check(self.lib.crp_batch_tune(self.h, trial_steps, ctypes.byref(best), tried, 16, ctypes.byref(n)))
        return best, [tried[k] for k in range(min(n.value, 16))]

    def _check(self, st: int):
        if st:
            raise CrpError(st, self.lib.crp_status_string(st).decode())

    def close(self):
        if getattr(self, "h", None):
            for s in self.sims:
                s.close()
            self.lib.crp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
