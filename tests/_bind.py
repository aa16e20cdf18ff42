"""Test-side bindings: the CPU oracle (oracle/liboracle.so) and the reference
harness built from the reference's own sources (oracle/_ref/libcrp_ref.so).

Test infrastructure only — the product package never imports this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import crp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libcrp_ref.so")

P = ctypes.POINTER
vp = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(vp)


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(ORACLE_LIB)
        sig = {
            "crpo_create": (ctypes.c_int32, [P(crp.Config), P(crp.BubblesIn), P(vp)]),
            "crpo_step": (ctypes.c_int32, [vp, ctypes.c_int32]),
            "crpo_set_source_elements": (ctypes.c_int32, [vp, ctypes.c_int32, vp, vp]),
            "crpo_get_dims": (ctypes.c_int32, [vp, P(crp.Dims)]),
            "crpo_get_stats": (ctypes.c_int32, [vp, P(crp.Stats)]),
            "crpo_read_field": (ctypes.c_int32, [vp, ctypes.c_int32, vp]),
            "crpo_focus_history": (ctypes.c_int64, [vp, ctypes.c_int32, vp, ctypes.c_int64]),
            "crpo_read_bubbles": (ctypes.c_int32, [vp, ctypes.c_int32, vp]),
            "crpo_set_threads": (None, [ctypes.c_int32]),
            "crpo_get_threads": (ctypes.c_int32, []),
            "crpo_destroy": (None, [vp]),
            "crpo_rp_step": (None, [vp, vp, ctypes.c_double, ctypes.c_double]),
            "crpo_omega_n": (ctypes.c_double, [vp, ctypes.c_double, ctypes.c_double, vp]),
            "crpo_upsilon_lp": (None, [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, vp]),
            "crpo_solve_pg": (ctypes.c_double, [vp] + [ctypes.c_double] * 7),
            "crpo_host_scalars": (None, [P(crp.Config), vp]),
            "crpo_host_sigma": (ctypes.c_int32, [P(crp.Config), vp, vp, vp, vp, vp, vp]),
            "crpo_config_defaults": (ctypes.c_int32, [P(crp.Config)]),
            "crpo_config_parse_file": (ctypes.c_int32, [ctypes.c_char_p, P(crp.Config), ctypes.c_char_p,
                                                        ctypes.c_size_t]),
            "crpo_seed_bubbles": (ctypes.c_int32, [P(crp.Config), vp, vp, vp, vp]),
            "crpo_seed_bubbles3": (ctypes.c_int32, [P(crp.Config), vp, vp, vp, vp, vp]),
            "crpo3_create": (ctypes.c_int32, [P(crp.Config), P(crp.BubblesIn), P(vp)]),
            "crpo3_step": (ctypes.c_int32, [vp, ctypes.c_int32]),
            "crpo3_set_source_elements": (ctypes.c_int32, [vp, ctypes.c_int32, vp, vp]),
            "crpo3_get_stats": (ctypes.c_int32, [vp, P(crp.Stats)]),
            "crpo3_num_bubbles": (ctypes.c_int32, [vp]),
            "crpo3_num_source_cells": (ctypes.c_int32, [vp]),
            "crpo3_read_field": (ctypes.c_int32, [vp, ctypes.c_int32, vp]),
            "crpo3_read_bubbles": (ctypes.c_int32, [vp, ctypes.c_int32, vp]),
            "crpo3_destroy": (None, [vp]),
        }
        for n, (r, a) in sig.items():
            f = getattr(lib, n)
            f.restype = r
            f.argtypes = a
        _oracle = lib
    return _oracle


def oracle_parse_file(path: str) -> crp.Config:
    """A configuration file parsed by the oracle's own parser on the oracle's
    defaults (oracle/workload.cpp): no product library involved."""
    lib = oracle_lib()
    cfg = crp.Config()
    lib.crpo_config_defaults(ctypes.byref(cfg))
    err = ctypes.create_string_buffer(512)
    st = lib.crpo_config_parse_file(path.encode(), ctypes.byref(cfg), err, 512)
    if st:
        raise crp.CrpError(st, err.value.decode())
    return cfg


def oracle_seed_bubbles(cfg: crp.Config) -> crp.Bubbles:
    """The seeded [ext] bubble population drawn by the oracle's own Philox."""
    n = cfg.ext_bubble_count
    arrs = [np.zeros(n) for _ in range(4)]
    st = oracle_lib().crpo_seed_bubbles(ctypes.byref(cfg), *[_ptr(a) for a in arrs])
    if st:
        raise crp.CrpError(st, "crpo_seed_bubbles")
    return crp.Bubbles(*arrs)


def oracle_seed_bubbles3(cfg: crp.Config) -> crp.Bubbles:
    """The seeded 3-D bubble population drawn by the oracle's own Philox."""
    n = cfg.ext_bubble_count
    x, y, z, r0, nb = (np.zeros(n) for _ in range(5))
    st = oracle_lib().crpo_seed_bubbles3(ctypes.byref(cfg), *[_ptr(a) for a in (x, y, z, r0, nb)])
    if st:
        raise crp.CrpError(st, "crpo_seed_bubbles3")
    return crp.Bubbles(x, y, r0, nb, z)


class OracleSim3:
    """The 3-D oracle (ext_grid_z > 0) with the surface of crp.Sim."""

    def __init__(self, cfg: crp.Config, bubbles: crp.Bubbles | None = None, threads: int = 0):
        self.lib = oracle_lib()
        if threads:
            self.lib.crpo_set_threads(threads)
        self._keep = (cfg, bubbles)
        h = vp()
        bin_ = bubbles.as_c() if bubbles is not None else None
        st = self.lib.crpo3_create(ctypes.byref(cfg), ctypes.byref(bin_) if bin_ is not None else None,
                                   ctypes.byref(h))
        if st:
            raise crp.CrpError(st, "crpo3_create")
        self.h = h
        self.dims3 = crp.Dims3()
        self.dims3.nx, self.dims3.ny, self.dims3.nz = cfg.grid_x + 2, cfg.grid_y + 2, cfg.ext_grid_z + 2
        self.dims3.num_bubbles = self.lib.crpo3_num_bubbles(self.h)
        self.dims3.source_cells = self.lib.crpo3_num_source_cells(self.h)

    def step(self, n=1):
        st = self.lib.crpo3_step(self.h, n)
        if st:
            raise crp.CrpError(st, "crpo3_step")

    def set_source_elements(self, amp, phase):
        a = np.ascontiguousarray(amp, dtype=np.float64)
        p = np.ascontiguousarray(phase, dtype=np.float64)
        st = self.lib.crpo3_set_source_elements(self.h, int(a.size), _ptr(a), _ptr(p))
        if st:
            raise crp.CrpError(st, "crpo3_set_source_elements")

    def stats(self):
        s = crp.Stats()
        self.lib.crpo3_get_stats(self.h, ctypes.byref(s))
        return s

    def field(self, name):
        out = np.empty(crp.field_shape3(self.dims3, name))
        st = self.lib.crpo3_read_field(self.h, crp.FIELDS[name], _ptr(out))
        assert st == 0, st
        return out

    def bubbles(self, name):
        out = np.empty(self.dims3.num_bubbles)
        st = self.lib.crpo3_read_bubbles(self.h, crp.BUBBLE_FIELDS[name], _ptr(out))
        assert st == 0, st
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.crpo3_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class OracleSim:
    """The CPU oracle with the same surface as crp.Sim."""

    def __init__(self, cfg: crp.Config, bubbles: crp.Bubbles | None = None, threads: int = 0):
        self.lib = oracle_lib()
        if threads:
            self.lib.crpo_set_threads(threads)
        self._keep = (cfg, bubbles)
        h = vp()
        bin_ = bubbles.as_c() if bubbles is not None else None
        st = self.lib.crpo_create(ctypes.byref(cfg), ctypes.byref(bin_) if bin_ is not None else None, ctypes.byref(h))
        if st:
            raise crp.CrpError(st, "crpo_create")
        self.h = h
        self.dims = crp.Dims()
        self.lib.crpo_get_dims(self.h, ctypes.byref(self.dims))

    def step(self, n=1):
        st = self.lib.crpo_step(self.h, n)
        if st:
            raise crp.CrpError(st, "crpo_step")

    def set_source_elements(self, amp, phase):
        a = np.ascontiguousarray(amp, dtype=np.float64)
        p = np.ascontiguousarray(phase, dtype=np.float64)
        st = self.lib.crpo_set_source_elements(self.h, int(a.size), _ptr(a), _ptr(p))
        if st:
            raise crp.CrpError(st, "crpo_set_source_elements")

    def stats(self):
        s = crp.Stats()
        self.lib.crpo_get_stats(self.h, ctypes.byref(s))
        return s

    def field(self, name):
        out = np.empty(crp.field_shape(self.dims, name))
        st = self.lib.crpo_read_field(self.h, crp.FIELDS[name], _ptr(out))
        assert st == 0
        return out

    def focus_history(self, which="actual"):
        w = 0 if which == "actual" else 1
        n = self.lib.crpo_focus_history(self.h, w, None, 0)
        out = np.zeros(max(n, 0))
        if n > 0:
            self.lib.crpo_focus_history(self.h, w, _ptr(out), n)
        return out

    def bubbles(self, name):
        out = np.empty(self.dims.num_bubbles)
        st = self.lib.crpo_read_bubbles(self.h, crp.BUBBLE_FIELDS[name], _ptr(out))
        assert st == 0
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.crpo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


# ---------------------------------------------------------------------------
# Reference harness (oracle/ref_harness.inc).

REF_FIELDS = [
    ("grid_x", "i"), ("grid_y", "i"), ("grid_lx", "d"), ("grid_ly", "d"), ("pml_x0", "i"), ("pml_x1", "i"),
    ("pml_y0", "i"), ("pml_y1", "i"), ("pml_grid_number", "i"), ("pml_sigma", "d"), ("pml_order", "i"),
    ("sim_cfl", "d"), ("sim_dt0", "d"), ("sim_n_step_max", "i"), ("sim_t_step_max", "d"),
    ("sim_save_interval", "i"), ("sim_order", "i"), ("sim_smooth_delta_band", "i"), ("tr_amp", "d"),
    ("tr_freq", "d"), ("tr_focal_dist", "d"), ("tr_pid", "i"), ("tr_pid_start_step", "i"),
    ("tr_init_control", "d"), ("tr_box_size", "d"), ("tr_cylindrical", "i"), ("tr_on_wave", "i"),
    ("tr_off_wave", "i"), ("tr_plane_v", "i"), ("tr_plane_p", "i"), ("tr_focused_v", "i"), ("tr_focused_p", "i"),
    ("bub_enable", "i"), ("bub_fg0", "d"), ("bub_R0", "d"), ("bub_P0", "d"), ("bub_T0", "d"), ("bub_gamma", "d"),
    ("bub_sigma", "d"), ("bub_mu", "d"), ("bub_rho", "d"), ("bub_K0", "d"), ("dbg_display", "i"), ("dbg_fg", "i"),
    ("dbg_T", "i"), ("dbg_p", "i"), ("dbg_v", "i"), ("dbg_bubbles", "i"),
]


class RefParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int if t == "i" else ctypes.c_double) for n, t in REF_FIELDS]


def ref_params(cfg: crp.Config) -> RefParams:
    p = RefParams()
    for n, _ in REF_FIELDS:
        src = {"dbg_display": "dbg_display"}.get(n, n)
        setattr(p, n, getattr(cfg, src))
    return p


_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_LIB)
        sig = {
            "crp_ref_host_scalars": (ctypes.c_int, [P(RefParams), vp]),
            "crp_ref_host_array_index": (ctypes.c_int, [P(RefParams), vp]),
            "crp_ref_host_sigma": (ctypes.c_int, [P(RefParams), vp, vp, vp, vp, vp, vp]),
            "crp_ref_host_bubbles": (ctypes.c_int, [P(RefParams), vp, ctypes.c_int]),
            "crp_ref_rp_step": (ctypes.c_int, [vp, vp, ctypes.c_double, ctypes.c_double]),
            "crp_ref_omega_n": (ctypes.c_double, [vp, ctypes.c_double, ctypes.c_double, vp]),
            "crp_ref_upsilon_lp": (ctypes.c_int, [ctypes.c_double] * 4 + [vp]),
            "crp_ref_solve_pg": (ctypes.c_double, [vp] + [ctypes.c_double] * 7),
            "crp_ref_setup": (ctypes.c_int, [P(RefParams), vp]),
            "crp_ref_run": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp]),
            "crp_ref_read_field": (ctypes.c_int, [ctypes.c_char_p, vp]),
            "crp_ref_read_bubbles": (ctypes.c_int, [ctypes.c_char_p, vp]),
            "crp_ref_save_ascii": (ctypes.c_int, [ctypes.c_char_p]),
            "crp_ref_save_sph": (ctypes.c_int, [ctypes.c_char_p]),
            "crp_ref_time": (ctypes.c_double, []),
            "crp_ref_teardown": (ctypes.c_int, []),
        }
        for n, (r, a) in sig.items():
            f = getattr(lib, n)
            f.restype = r
            f.argtypes = a
        _ref = lib
    return _ref


SMALL_CONF = os.path.join(ROOT, "tests", "golden", "small.conf")


def small_config(**over) -> crp.Config:
    """tests/golden/small.conf with overrides."""
    text = open(SMALL_CONF).read()
    cfg = crp.parse_string(text)
    for k, v in over.items():
        setattr(cfg, k, v)
    return cfg


def focal_weights(cfg: crp.Config, radius: float) -> np.ndarray:
    """Cell weights of the focal objective of crp_adjoint on the dense p0 layout
    [j][i] (i in 0..X+1, j in 0..Y+1): the cell volume (2 pi r dx dy in the
    axisymmetric geometry, dx dy otherwise) for interior cells whose centre lies
    within `radius` of the source's focus, 0 elsewhere and on the source row."""
    X, Y = cfg.grid_x, cfg.grid_y
    dx, dy = cfg.grid_lx / X, cfg.grid_ly / Y
    cx = 0.0
    cy = cfg.tr_focal_dist * 0.5 * np.sqrt(3.0) if cfg.tr_focal_dist else cfg.grid_ly * 0.5
    xm = (np.arange(X + 2) - 0.5) * dx
    ym = (np.arange(Y + 2) - 0.5) * dy
    ii, jj = np.meshgrid(np.arange(X + 2), np.arange(Y + 2))
    xx, yy = np.meshgrid(xm, ym)
    inside = (ii >= 1) & (ii <= X) & (jj >= 1) & (jj <= Y) & ((xx - cx) * (xx - cx) + (yy - cy) * (yy - cy) <= radius * radius)
    if cfg.ext_source_row > 0:
        inside &= jj != cfg.ext_source_row
    vol = 2.0 * np.pi * xx * dx * dy if cfg.tr_cylindrical else np.full_like(xx, dx * dy)
    return np.where(inside, vol, 0.0)


def oracle_focal_objective(cfg: crp.Config, amp, phase, steps: int, radius: float) -> float:
    """J = sum over `steps` steps from t = 0 of dt sum w p0^2 (focal_weights), on the oracle."""
    sim = OracleSim(cfg)
    try:
        if amp is not None:
            sim.set_source_elements(amp, phase)
        w = focal_weights(cfg, radius)
        dt = cfg.sim_cfl * min(cfg.grid_lx / cfg.grid_x, cfg.grid_ly / cfg.grid_y) / cfg.ext_c_inf
        J = 0.0
        for _ in range(steps):
            sim.step(1)
            p0 = sim.field("p0")
            assert p0.shape == w.shape
            J += dt * float(np.sum(w * p0 * p0))
        return J
    finally:
        sim.close()
