"""Bindings of the reference builds under oracle/_ref (test infrastructure).

* ``RefIO``   -- the reference parser/loaders (host code of libref_prog.so);
* ``RefProg`` -- the reference transport run as its main() performs it, with
                 the kernel timed by CUDA events (libref_prog.so, needs a GPU);
* ``RefGPU``  -- GPU harnesses running the reference's own device functions
                 (libref_cuda.so, needs a GPU);
* ``RefCPU``  -- the reference transport kernel compiled for the host
                 (libref_cpu.so, OpenMP);
* ``run_reference_program`` -- the unmodified reference program
                 (mcgpu_pet_ref.x, needs a GPU).

The libraries are built from the reference sources by oracle/ref/Makefile.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import gzip
import os
import subprocess
from typing import Optional

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
M, S, R, NE_RAY = 15, 30, 128, 25005

P = C.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data


def available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, name))


class Params(C.Structure):
    """refc_params / the head of refio_config (same leading layout)."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("inv_vx", C.c_float), ("inv_vy", C.c_float), ("inv_vz", C.c_float),
        ("bbx", C.c_float), ("bby", C.c_float), ("bbz", C.c_float),
        ("n_e", C.c_int), ("e0", C.c_float), ("ide", C.c_float),
        ("cx", C.c_float), ("cy", C.c_float), ("cz", C.c_float), ("radius", C.c_float), ("height", C.c_float),
        ("psf_size", C.c_int), ("tally_psf_sino", C.c_int), ("tally_type", C.c_int),
        ("acq_ps", C.c_ulonglong), ("mean_life", C.c_float),
        ("e_resol", C.c_float), ("e_low", C.c_float), ("e_high", C.c_float), ("fovz", C.c_float),
        ("nrows", C.c_int), ("ncrystals", C.c_int), ("nangles", C.c_int), ("nrad", C.c_int), ("nzs", C.c_int),
        ("nbins", C.c_int), ("res", C.c_int), ("nvoxs", C.c_int), ("ne", C.c_int), ("mrd", C.c_int),
        ("span", C.c_int), ("nsinos", C.c_int),
        ("tpb", C.c_int), ("seed", C.c_int), ("peta", C.c_int),
    ]


class IOConfig(C.Structure):
    _fields_ = Params._fields_ + [
        ("gpu_id", C.c_int), ("nseg", C.c_int), ("flag_material_dose", C.c_int), ("fact_object", C.c_float),
        ("roi", C.c_short * 6), ("activity", C.c_float * M), ("density_max", C.c_float * M),
        ("density_nominal", C.c_float * M), ("voxel_file", C.c_char * 250), ("psf_file", C.c_char * 250),
        ("dose_file", C.c_char * 250), ("materials", (C.c_char * 250) * M),
    ]


class Tables(C.Structure):
    _fields_ = [(n, P) for n in ["fco", "uico", "fj0", "noscco", "xco", "pco", "aco", "bco", "pmax", "itlco",
                                 "ituco"]]


@contextlib.contextmanager
def _chdir(path: Optional[str]):
    old = os.getcwd()
    if path:
        os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


def _quiet_call(fn, *args):
    """Run a reference function while discarding what it prints on stdout."""
    import sys
    sys.stdout.flush()
    fd = os.dup(1)
    with open(os.devnull, "w") as dn:
        os.dup2(dn.fileno(), 1)
        try:
            return fn(*args)
        finally:
            C.CDLL(None).fflush(None)
            os.dup2(fd, 1)
            os.close(fd)


class RefTables:
    """Reference tables as numpy arrays (flat, reference layout)."""

    def __init__(self, n_e: int):
        self.woodcock = np.zeros((n_e, 2), np.float32)
        self.mfp_a = np.zeros((n_e, M, 3), np.float32)
        self.mfp_b = np.zeros((n_e, M, 3), np.float32)
        self.fco = np.zeros(S * M, np.float32)
        self.uico = np.zeros(S * M, np.float32)
        self.fj0 = np.zeros(S * M, np.float32)
        self.noscco = np.zeros(M, np.int32)
        self.xco = np.zeros(M * R, np.float32)
        self.pco = np.zeros(M * R, np.float32)
        self.aco = np.zeros(M * R, np.float32)
        self.bco = np.zeros(M * R, np.float32)
        self.pmax = np.zeros((NE_RAY, M), np.float32)
        self.itlco = np.zeros(M * R, np.uint8)
        self.ituco = np.zeros(M * R, np.uint8)

    def c_struct(self) -> Tables:
        t = Tables()
        for n, _ in Tables._fields_:
            setattr(t, n, _p(getattr(self, n)))
        return t

    @classmethod
    def from_scene_export(cls, t: dict) -> "RefTables":
        """Wrap tables exported by mcpet (same layout) for the reference kernel."""
        ne = t["woodcock"].shape[0]
        r = cls(ne)
        r.woodcock[:] = t["woodcock"]
        r.mfp_a[:] = t["mfp_a"]
        r.mfp_b[:] = t["mfp_b"]
        for k in ["fco", "uico", "fj0", "noscco", "xco", "pco", "aco", "bco", "itlco", "ituco"]:
            getattr(r, k)[:] = t[k]
        r.pmax[:ne] = t["pmax"]
        return r


class RefIO:
    """read_input + load_voxels + load_material of the reference (host only)."""

    def __init__(self):
        self.L = C.CDLL(os.path.join(REF_DIR, "libref_prog.so"))
        self.L.refio_open.restype = P
        self.L.refio_open.argtypes = [C.c_char_p]
        for n in ["refio_get_config", "refio_get_voxels", "refio_close"]:
            getattr(self.L, n).argtypes = [P, P]
        self.L.refio_close.argtypes = [P]
        self.L.refio_get_tables.argtypes = [P] * 15

    def load(self, in_path: str, cwd: Optional[str] = None):
        with _chdir(cwd):
            h = _quiet_call(self.L.refio_open, os.fsencode(in_path))
        try:
            cfg = IOConfig()
            self.L.refio_get_config(h, C.byref(cfg))
            nv = cfg.nx * cfg.ny * cfg.nz
            vox = np.zeros((nv, 3), np.float32)
            self.L.refio_get_voxels(h, _p(vox))
            t = RefTables(cfg.n_e)
            self.L.refio_get_tables(h, _p(t.woodcock), _p(t.mfp_a), _p(t.mfp_b), _p(t.fco), _p(t.uico), _p(t.fj0),
                                    _p(t.noscco), _p(t.xco), _p(t.pco), _p(t.aco), _p(t.bco), _p(t.pmax),
                                    _p(t.itlco), _p(t.ituco))
        finally:
            self.L.refio_close(h)
        return cfg, vox, t


def params_from_scene(scene, seed: Optional[int] = None, peta: int = 1) -> Params:
    """Reference parameter block from an mcpet scene's configuration."""
    cfg, info = scene.config, scene.info
    p = Params()
    p.nx, p.ny, p.nz = info.nx, info.ny, info.nz
    p.inv_vx, p.inv_vy, p.inv_vz = [np.float32(1.0) / np.float32(v) for v in info.voxel_size]
    p.bbx, p.bby, p.bbz = list(info.bbox)
    p.n_e, p.e0, p.ide = info.n_energy, info.e0, info.inv_de
    p.cx, p.cy, p.cz = list(cfg.detector_center)
    p.radius, p.height = cfg.detector_radius, cfg.detector_height
    p.psf_size, p.tally_psf_sino, p.tally_type = cfg.psf_size, cfg.tally_psf_sinogram, cfg.tally_type
    p.acq_ps, p.mean_life = cfg.acquisition_time_ps, cfg.mean_life
    p.e_resol, p.e_low, p.e_high, p.fovz = (cfg.energy_resolution, cfg.energy_window_low, cfg.energy_window_high,
                                            cfg.fov_z)
    p.nrows, p.ncrystals, p.nangles, p.nrad, p.nzs = cfg.n_rows, cfg.n_crystals, cfg.n_angles, cfg.n_radial, \
        cfg.n_z_slices
    p.nbins, p.res, p.ne, p.mrd, p.span, p.nsinos = (int(cfg.n_bins), cfg.image_res, cfg.n_energy_bins,
                                                     cfg.max_ring_difference, cfg.span, cfg.n_sinograms)
    p.nvoxs = cfg.image_res * cfg.image_res * cfg.n_z_slices
    p.tpb = cfg.threads_per_block
    p.seed = cfg.seed if seed is None else seed
    p.peta = peta
    return p


class RefCPU:
    """The reference transport kernel compiled for the host (libref_cpu.so)."""

    def __init__(self):
        self.L = C.CDLL(os.path.join(REF_DIR, "libref_cpu.so"))
        self.L.refc_run.argtypes = [P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, C.c_longlong, C.c_int]
        self.L.refc_run.restype = C.c_int
        self.L.refc_run2.argtypes = self.L.refc_run.argtypes + [P, P, P]
        self.L.refc_run2.restype = C.c_int
        self.L.refc_prng.argtypes = [C.c_int, C.c_int, P, C.c_int, P, P, P]
        self.L.refc_sinogram_events.argtypes = [P, C.c_int] + [P] * 15
        self.L.refc_gcoa.argtypes = [C.c_int, P, P, P, P, P, P, P]
        self.L.refc_graa.argtypes = [C.c_int, P, P, P, P, P, P, P]
        self.L.refc_abmodm.argtypes = [C.c_int, C.c_int, C.c_int]
        self.L.refc_abmodm.restype = C.c_int

    def run(self, p: Params, voxels: np.ndarray, t: RefTables, block_list=None, n_threads: int = 0,
            psf_capacity: int = 0, material_dose: bool = False, dose_roi=None):
        """dose_roi: 0-based (x0, x1, y0, y1, z0, z1) enables the voxel dose tally;
        the reference's host dose tallies are not atomic, so n_threads must be 1."""
        nv = p.nx * p.ny * p.nz
        out = {
            "trues": np.zeros(p.nbins, np.int32), "scatter": np.zeros(p.nbins, np.int32),
            "image_trues": np.zeros(nv, np.int32), "image_scatter": np.zeros(nv, np.int32),
            "spectrum": np.zeros(max(p.ne, 1), np.int32),
        }
        psf = np.zeros(max(psf_capacity, 1) * 44, np.uint8)
        idx = C.c_int(0)
        hist = C.c_ulonglong(0)
        tab = t.c_struct()
        bl = None if block_list is None else np.ascontiguousarray(block_list, np.int32)
        p2 = Params.from_buffer_copy(p)
        p2.psf_size = psf_capacity
        md = np.zeros((15, 2), np.uint64) if material_dose else None
        vd, roi = None, None
        if dose_roi is not None:
            roi = np.ascontiguousarray(dose_roi, np.int16)
            nd = int(roi[1] - roi[0] + 1) * int(roi[3] - roi[2] + 1) * int(roi[5] - roi[4] + 1)
            vd = np.zeros((nd, 2), np.uint64)
        if (md is not None or vd is not None) and n_threads != 1:
            raise ValueError("the reference's host dose tallies need n_threads=1")
        rc = self.L.refc_run2(C.byref(p2), _p(np.ascontiguousarray(voxels, np.float32)), _p(t.woodcock),
                              _p(t.mfp_a), _p(t.mfp_b), C.byref(tab), _p(out["trues"]), _p(out["scatter"]),
                              _p(out["image_trues"]), _p(out["image_scatter"]), _p(out["spectrum"]), _p(psf),
                              C.addressof(idx), C.addressof(hist), _p(bl), 0 if bl is None else len(bl),
                              int(n_threads), _p(md), _p(vd), _p(roi))
        assert rc == 0
        out["material_dose"], out["voxel_dose"] = md, vd
        out["psf_count"] = idx.value
        out["total_histories"] = hist.value
        n = max(0, min(idx.value, psf_capacity))
        out["psf_raw"] = psf[: n * 44]
        return out

    def prng(self, seed: int, tids, ndraw: int):
        tids = np.ascontiguousarray(tids, np.int32)
        n = len(tids)
        s = np.zeros((n, 2), np.int32)
        f = np.zeros((n, ndraw), np.float32)
        d = np.zeros((n, ndraw), np.float64)
        self.L.refc_prng(n, seed, _p(tids), ndraw, _p(s), _p(f), _p(d))
        return s, f, d

    def sinogram_events(self, p: Params, ev: dict) -> np.ndarray:
        n = len(ev["e2"])
        a = _event_arrays(ev)
        nv = p.nx * p.ny * p.nz
        tr = np.zeros(p.nbins, np.int32)
        sc = np.zeros(p.nbins, np.int32)
        it = np.zeros(max(nv, 1), np.int32)
        isc = np.zeros(max(nv, 1), np.int32)
        sp = np.zeros(max(p.ne, 1), np.int32)
        out = np.zeros((n, 6), np.int32)
        self.L.refc_sinogram_events(C.byref(p), n, _p(a["e2"]), _p(a["e1"]), _p(a["pos2"]), _p(a["pos1"]),
                                    _p(a["dir2"]), _p(a["dir1"]), _p(a["st2"]), _p(a["st1"]), _p(a["seeds"]),
                                    _p(tr), _p(sc), _p(it), _p(isc), _p(sp), _p(out))
        return out

    def gcoa(self, t: RefTables, energy, mat, seeds):
        e = np.ascontiguousarray(energy, np.float32)
        m = np.ascontiguousarray(mat, np.int32)
        s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
        n = len(e)
        eo = np.zeros(n, np.float32)
        co = np.zeros(n, np.float64)
        so = np.zeros((n, 2), np.int32)
        tab = t.c_struct()
        self.L.refc_gcoa(n, _p(e), _p(m), _p(s), C.byref(tab), _p(eo), _p(co), _p(so))
        return eo, co, so

    def graa(self, t: RefTables, energy, mat, pmax, seeds):
        e = np.ascontiguousarray(energy, np.float32)
        m = np.ascontiguousarray(mat, np.int32)
        pm = np.ascontiguousarray(pmax, np.float32)
        s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
        n = len(e)
        co = np.zeros(n, np.float64)
        so = np.zeros((n, 2), np.int32)
        tab = t.c_struct()
        self.L.refc_graa(n, _p(e), _p(m), _p(pm), _p(s), C.byref(tab), _p(co), _p(so))
        return co, so


def _event_arrays(ev: dict) -> dict:
    return {k: np.ascontiguousarray(ev[k], dtype=(np.int8 if k.startswith("st") else
                                                  np.int32 if k == "seeds" else np.float32))
            for k in ["e2", "e1", "pos2", "pos1", "dir2", "dir1", "st2", "st1", "seeds"]}


class ProgOutputs(C.Structure):
    _fields_ = [("trues", P), ("scatter", P), ("image_trues", P), ("image_scatter", P), ("spectrum", P),
                ("psf", P), ("psf_capacity", C.c_longlong), ("psf_count", C.c_int),
                ("total_histories", C.c_ulonglong), ("kernel_ms", C.c_float), ("nbins", C.c_int),
                ("nvox", C.c_int), ("ne", C.c_int), ("material_dose", P), ("voxel_dose", P),
                ("voxel_dose_capacity", C.c_longlong), ("roi", C.c_short * 6), ("n_roi", C.c_longlong)]


class RefProg:
    """The reference's own transport run (read_input .. track_particles) on the GPU."""

    def __init__(self):
        self.L = C.CDLL(os.path.join(REF_DIR, "libref_prog.so"))
        self.L.refp_run.argtypes = [C.c_char_p, C.c_int, P]
        self.L.refp_run.restype = C.c_int

    def run(self, in_path: str, nbins: int, nvox: int, ne: int, background: bool = False, psf_capacity: int = 0,
            cwd: Optional[str] = None, dose_voxels: int = 0) -> dict:
        out = {"trues": np.zeros(nbins, np.int32), "scatter": np.zeros(nbins, np.int32),
               "image_trues": np.zeros(nvox, np.int32), "image_scatter": np.zeros(nvox, np.int32),
               "spectrum": np.zeros(max(ne, 1), np.int32)}
        psf = np.zeros(max(psf_capacity, 1) * 44, np.uint8)
        o = ProgOutputs()
        for k in ["trues", "scatter", "image_trues", "image_scatter", "spectrum"]:
            setattr(o, k, _p(out[k]))
        o.psf = _p(psf)
        o.psf_capacity = psf_capacity
        md = np.zeros((15, 2), np.uint64)
        vd = np.zeros((max(dose_voxels, 1), 2), np.uint64)
        o.material_dose, o.voxel_dose, o.voxel_dose_capacity = _p(md), _p(vd), dose_voxels
        out["material_dose"], out["voxel_dose"] = md, vd[:dose_voxels]
        with _chdir(cwd):
            rc = _quiet_call(self.L.refp_run, os.fsencode(in_path), int(bool(background)), C.byref(o))
        if rc != 0:
            raise RuntimeError(f"reference run failed with CUDA error {rc}")
        assert (o.nbins, o.nvox) == (nbins, nvox)
        out["psf_count"] = o.psf_count
        out["total_histories"] = int(o.total_histories)
        out["kernel_ms"] = float(o.kernel_ms)
        out["roi"] = [int(v) for v in o.roi]
        out["n_roi"] = int(o.n_roi)
        n = max(0, min(o.psf_count, psf_capacity))
        out["psf_raw"] = psf[: n * 44]
        return out


class RefGPU:
    """Reference device functions on the GPU (libref_cuda.so harnesses)."""

    def __init__(self):
        self.L = C.CDLL(os.path.join(REF_DIR, "libref_cuda.so"))
        self.L.refh_prng.argtypes = [C.c_int, C.c_int, P, C.c_int, P, P, P]
        self.L.refh_sinogram_events.argtypes = [P, C.c_int] + [P] * 10
        self.L.refh_gcoa.argtypes = [C.c_int, P, P, P, P, P, P, P, P, P, P]
        self.L.refh_graa.argtypes = [C.c_int, P, P, P, P, P, P, P, P, P, P, P, P]
        self.L.refh_source.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int, P, P,
                                       P]
        for n in ["refh_prng", "refh_sinogram_events", "refh_gcoa", "refh_graa", "refh_source"]:
            getattr(self.L, n).restype = C.c_int

    def prng(self, seed: int, tids, ndraw: int):
        tids = np.ascontiguousarray(tids, np.int32)
        n = len(tids)
        s = np.zeros((n, 2), np.int32)
        f = np.zeros((n, ndraw), np.float32)
        d = np.zeros((n, ndraw), np.float64)
        assert self.L.refh_prng(n, seed, _p(tids), ndraw, _p(s), _p(f), _p(d)) == 0
        return s, f, d

    def sinogram_events(self, p: Params, ev: dict) -> np.ndarray:
        n = len(ev["e2"])
        a = _event_arrays(ev)
        out = np.zeros((n, 6), np.int32)
        assert self.L.refh_sinogram_events(C.byref(p), n, _p(a["e2"]), _p(a["e1"]), _p(a["pos2"]),
                                           _p(a["pos1"]), _p(a["dir2"]), _p(a["dir1"]), _p(a["st2"]),
                                           _p(a["st1"]), _p(a["seeds"]), _p(out)) == 0
        return out

    def gcoa(self, t: RefTables, energy, mat, seeds):
        e = np.ascontiguousarray(energy, np.float32)
        m = np.ascontiguousarray(mat, np.int32)
        s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
        n = len(e)
        eo = np.zeros(n, np.float32)
        co = np.zeros(n, np.float64)
        so = np.zeros((n, 2), np.int32)
        assert self.L.refh_gcoa(n, _p(e), _p(m), _p(s), _p(t.fco), _p(t.uico), _p(t.fj0), _p(t.noscco), _p(eo),
                                _p(co), _p(so)) == 0
        return eo, co, so

    def graa(self, t: RefTables, energy, mat, pmax, seeds):
        e = np.ascontiguousarray(energy, np.float32)
        m = np.ascontiguousarray(mat, np.int32)
        pm = np.ascontiguousarray(pmax, np.float32)
        s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
        n = len(e)
        co = np.zeros(n, np.float64)
        so = np.zeros((n, 2), np.int32)
        assert self.L.refh_graa(n, _p(e), _p(m), _p(pm), _p(s), _p(t.xco), _p(t.pco), _p(t.aco), _p(t.bco),
                                _p(t.itlco), _p(t.ituco), _p(co), _p(so)) == 0
        return co, so

    def source(self, shape, inv_voxel_size, seeds, background: bool = False):
        nz, ny, nx = shape
        s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
        out = np.zeros((nx * ny * nz, 4, 3), np.float32)
        so = np.zeros_like(s)
        assert self.L.refh_source(nx, ny, nz, float(inv_voxel_size[0]), float(inv_voxel_size[1]),
                                  float(inv_voxel_size[2]), 0 if background else 1, _p(s), _p(out), _p(so)) == 0
        return out, so


def run_reference_program(in_path: str, workdir: str, background: bool = False, timeout: int = 600) -> dict:
    """Run the unmodified reference program (GPU) in workdir; return its outputs."""
    exe = os.path.join(REF_DIR, "mcgpu_pet_ref.x")
    args = [exe, in_path] + (["bg"] if background else [])
    proc = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"reference program failed ({proc.returncode}):\n{proc.stdout[-3000:]}\n{proc.stderr}")
    out = {"stdout": proc.stdout}
    names = (("trues", "sinogram_BG_Trues.raw.gz" if background else "sinogram_Trues.raw.gz"),
             ("scatter", "sinogram_BG_Scatter.raw.gz" if background else "sinogram_Scatter.raw.gz"),
             ("image_trues", "BG_image_True.raw.gz" if background else "image_Trues.raw.gz"),
             ("image_scatter", "BG_image_Scatter.raw.gz" if background else "image_Scatter.raw.gz"))
    for key, name in names:
        p = os.path.join(workdir, name)
        if os.path.exists(p):
            with gzip.open(p, "rb") as f:
                out[key] = np.frombuffer(f.read(), np.int32).copy()
    spec = os.path.join(workdir, "Energy_Sinogram_Spectrum.dat")
    if os.path.exists(spec):
        out["spectrum"] = np.loadtxt(spec, dtype=np.int64)[:, 1].astype(np.int32)
    for line in proc.stdout.splitlines():
        if "Total number of histories simulated" in line:
            out["total_histories"] = int(line.split("=")[1].split()[0])
        if "Time spent in the Monte Carlo transport only" in line:
            out["mc_seconds"] = float(line.split(":")[1].split()[0])
    return out
