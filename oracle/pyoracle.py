"""ctypes binding of the C oracle (oracle/_build/liboracle.so) -- TEST
INFRASTRUCTURE, used only by tests/, __graft_entry__.smoke() and the CPU
baseline of bench.py as the checker.

The oracle reads the tables exported by an mcpet scene (same reference
layout); those tables are themselves pinned bit for bit against the
reference loaders by tests/test_tables.py.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
M = 15
P = C.c_void_p


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("inv_vx", C.c_float), ("inv_vy", C.c_float), ("inv_vz", C.c_float),
        ("bbx", C.c_float), ("bby", C.c_float), ("bbz", C.c_float),
        ("n_e", C.c_int), ("e0", C.c_float), ("ide", C.c_float),
        ("cx", C.c_float), ("cy", C.c_float), ("cz", C.c_float), ("radius", C.c_float), ("height", C.c_float),
        ("psf_capacity", C.c_int), ("tally_psf_sinogram", C.c_int), ("tally_type", C.c_int),
        ("acq_ps", C.c_ulonglong), ("mean_life", C.c_float),
        ("e_resol", C.c_float), ("e_low", C.c_float), ("e_high", C.c_float), ("fovz", C.c_float),
        ("nrows", C.c_int), ("ncrystals", C.c_int), ("nangles", C.c_int), ("nrad", C.c_int), ("nzs", C.c_int),
        ("ne", C.c_int), ("mrd", C.c_int), ("span", C.c_int), ("nsinos", C.c_int),
        ("nbins", C.c_longlong),
        ("tpb", C.c_int), ("seed", C.c_int), ("background", C.c_int),
        ("dose_roi", C.c_int * 6),
        ("prompt_energy", C.c_float), ("prompt_yield", C.c_float),
    ]


class Tables(C.Structure):
    _fields_ = [(n, P) for n in ["woodcock", "mfp_a", "mfp_b", "pmax", "fco", "uico", "fj0", "noscco", "xco",
                                 "pco", "aco", "bco", "itlco", "ituco"]]


class Outputs(C.Structure):
    _fields_ = [("trues", P), ("scatter", P), ("image_trues", P), ("image_scatter", P), ("spectrum", P),
                ("psf", P), ("psf_count", C.c_int32), ("histories", C.c_ulonglong),
                ("counters", C.c_ulonglong * 9), ("material_dose", P), ("voxel_dose", P)]


COUNTER_NAMES = ["woodcock_steps_inside", "table_refreshes", "majorant_refreshes", "tally_increments", "photons",
                 "compton", "rayleigh", "photoelectric", "lanes"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(f"{LIB} missing: run `make -C {HERE}` or __graft_entry__.build()")
        L = C.CDLL(LIB)
        L.orc_run.argtypes = [P, P, P, P, P, P, C.c_longlong, C.c_int, P]
        L.orc_run.restype = C.c_int
        L.orc_rng.argtypes = [C.c_int, P, C.c_int, C.c_int, P, P, P]
        L.orc_detector.argtypes = [P, C.c_int] + [P] * 10
        L.orc_sinogram_bin.argtypes = [P, C.c_float, C.c_float, C.c_float, C.c_float]
        L.orc_sinogram_bin.restype = C.c_longlong
        L.orc_compton.argtypes = [P, C.c_int, P, P, P, P, P, P]
        L.orc_rayleigh.argtypes = [P, C.c_int, P, P, P, P, P, P]
        L.orc_source.argtypes = [C.c_int, C.c_int, C.c_int, P, C.c_int, P, P, P]
        L.orc_sinogram_sizes.argtypes = [C.c_int, C.c_int, C.c_int, P, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class OracleScene:
    """Parameters and tables of an mcpet scene, in the oracle's layout."""

    def __init__(self, scene, seed=None, background=False, tables=None):
        cfg, info = scene.config, scene.info
        self.t = tables if tables is not None else scene.export_tables()
        vox = self.t["voxels"]
        self.mat0 = np.ascontiguousarray((vox[:, 0] - 1).astype(np.int32))
        self.rho = np.ascontiguousarray(vox[:, 1])
        self.act = np.ascontiguousarray(vox[:, 2])
        p = Params()
        p.nx, p.ny, p.nz = info.nx, info.ny, info.nz
        p.inv_vx, p.inv_vy, p.inv_vz = [np.float32(1.0) / np.float32(v) for v in info.voxel_size]
        p.bbx, p.bby, p.bbz = list(info.bbox)
        p.n_e, p.e0, p.ide = info.n_energy, info.e0, info.inv_de
        p.cx, p.cy, p.cz = list(cfg.detector_center)
        p.radius, p.height = cfg.detector_radius, cfg.detector_height
        p.psf_capacity, p.tally_psf_sinogram, p.tally_type = cfg.psf_size, cfg.tally_psf_sinogram, cfg.tally_type
        p.acq_ps, p.mean_life = cfg.acquisition_time_ps, cfg.mean_life
        p.e_resol, p.e_low, p.e_high, p.fovz = (cfg.energy_resolution, cfg.energy_window_low,
                                                cfg.energy_window_high, cfg.fov_z)
        p.nrows, p.ncrystals, p.nangles, p.nrad, p.nzs = (cfg.n_rows, cfg.n_crystals, cfg.n_angles, cfg.n_radial,
                                                          cfg.n_z_slices)
        p.ne, p.mrd, p.span, p.nsinos, p.nbins = (cfg.n_energy_bins, cfg.max_ring_difference, cfg.span,
                                                  cfg.n_sinograms, cfg.n_bins)
        p.tpb = cfg.threads_per_block
        p.seed = cfg.seed if seed is None else seed
        p.background = int(bool(background))
        roi = list(cfg.dose_roi) if cfg.tally_voxel_dose else [0, -1, 0, -1, 0, -1]
        for k in range(6):
            p.dose_roi[k] = int(roi[k])
        if cfg.prompt_gamma_energy > 0:
            p.prompt_energy, p.prompt_yield = cfg.prompt_gamma_energy, cfg.prompt_gamma_yield
        self.material_dose = bool(cfg.tally_material_dose)
        self.n_dose = int(info.n_dose_voxels)
        self.p = p
        self._tab = Tables()
        for n, _ in Tables._fields_:
            setattr(self._tab, n, _p(self.t[n]))
        self.n_voxels = int(info.n_voxels)

    def run(self, voxel_list=None, n_threads: int = 0, psf_capacity=None) -> dict:
        p = Params.from_buffer_copy(self.p)
        if psf_capacity is not None:
            p.psf_capacity = psf_capacity
        want_sino = p.tally_psf_sinogram in (0, 2)
        nb = int(p.nbins) if want_sino else 1
        out = {
            "trues": np.zeros(nb, np.int32), "scatter": np.zeros(nb, np.int32),
            "image_trues": np.zeros(self.n_voxels, np.int32), "image_scatter": np.zeros(self.n_voxels, np.int32),
            "spectrum": np.zeros(max(p.ne, 1), np.int32),
        }
        psf = np.zeros(max(p.psf_capacity, 1) * 44, np.uint8) if p.tally_psf_sinogram in (0, 1) else None
        o = Outputs()
        for k in ["trues", "scatter", "image_trues", "image_scatter", "spectrum"]:
            setattr(o, k, _p(out[k]))
        o.psf = _p(psf)
        md = np.zeros((M, 2), np.uint64) if self.material_dose else None
        vd = np.zeros((self.n_dose, 2), np.uint64) if self.n_dose > 0 else None
        o.material_dose, o.voxel_dose = _p(md), _p(vd)
        vl = None if voxel_list is None else np.ascontiguousarray(voxel_list, np.int32)
        rc = lib().orc_run(C.byref(p), C.byref(self._tab), _p(self.mat0), _p(self.rho), _p(self.act), _p(vl),
                           0 if vl is None else len(vl), int(n_threads), C.byref(o))
        assert rc == 0
        out["total_histories"] = int(o.histories)
        out["psf_count"] = int(o.psf_count)
        n = max(0, min(o.psf_count, p.psf_capacity))
        out["psf_raw"] = None if psf is None else psf[: n * 44]
        out["counters"] = {k: int(o.counters[i]) for i, k in enumerate(COUNTER_NAMES)}
        out["material_dose"], out["voxel_dose"] = md, vd
        return out


def run_scene(scene, n_threads: int = 0, **kw) -> dict:
    return OracleScene(scene, **{k: v for k, v in kw.items() if k in ("seed", "background")}).run(
        n_threads=n_threads, voxel_list=kw.get("voxel_list"))


def rng(seed: int, stream_ids, ndraw: int):
    ids = np.ascontiguousarray(stream_ids, np.int64)
    n = len(ids)
    s = np.zeros((n, 2), np.int32)
    f = np.zeros((n, ndraw), np.float32)
    d = np.zeros((n, ndraw), np.float64)
    lib().orc_rng(int(seed), _p(ids), n, ndraw, _p(s), _p(f), _p(d))
    return s, f, d


def detector(osc: OracleScene, ev: dict) -> np.ndarray:
    n = len(ev["e2"])
    a = {k: np.ascontiguousarray(ev[k], dtype=(np.int8 if k.startswith("st") else
                                               np.int32 if k == "seeds" else np.float32))
         for k in ["e2", "e1", "pos2", "pos1", "dir2", "dir1", "st2", "st1", "seeds"]}
    out = np.zeros((n, 6), np.int32)
    lib().orc_detector(C.byref(osc.p), n, _p(a["e2"]), _p(a["e1"]), _p(a["pos2"]), _p(a["pos1"]), _p(a["dir2"]),
                       _p(a["dir1"]), _p(a["st2"]), _p(a["st1"]), _p(a["seeds"]), _p(out))
    return out


def compton(osc: OracleScene, energy, mat, seeds):
    e = np.ascontiguousarray(energy, np.float32)
    m = np.ascontiguousarray(mat, np.int32)
    s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
    n = len(e)
    eo, co, so = np.zeros(n, np.float32), np.zeros(n, np.float64), np.zeros((n, 2), np.int32)
    lib().orc_compton(C.byref(osc._tab), n, _p(e), _p(m), _p(s), _p(eo), _p(co), _p(so))
    return eo, co, so


def rayleigh(osc: OracleScene, energy, mat, pmax, seeds):
    e = np.ascontiguousarray(energy, np.float32)
    m = np.ascontiguousarray(mat, np.int32)
    pm = np.ascontiguousarray(pmax, np.float32)
    s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
    n = len(e)
    co, so = np.zeros(n, np.float64), np.zeros((n, 2), np.int32)
    lib().orc_rayleigh(C.byref(osc._tab), n, _p(e), _p(m), _p(pm), _p(s), _p(co), _p(so))
    return co, so


def source(shape, inv_voxel_size, seeds, background=False):
    nz, ny, nx = shape
    inv = np.ascontiguousarray(inv_voxel_size, np.float32)
    s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
    out = np.zeros((nx * ny * nz, 4, 3), np.float32)
    so = np.zeros_like(s)
    lib().orc_source(nx, ny, nz, _p(inv), int(bool(background)), _p(s), _p(out), _p(so))
    return out, so


def sinogram_sizes(mrd: int, span: int, nzs: int):
    a, b = C.c_int(0), C.c_int(0)
    lib().orc_sinogram_sizes(mrd, span, nzs, C.addressof(a), C.addressof(b))
    return a.value, b.value


def total_zscore(res, ref: dict) -> float:
    """z-score of the difference of two independent Poisson-like totals of
    detected coincidences (GPU result object vs. oracle dict)."""
    a = float(res.coincidences)
    b = float(ref["trues"].sum(dtype=np.int64) + ref["scatter"].sum(dtype=np.int64))
    return (a - b) / math.sqrt(max(a + b, 1.0))
