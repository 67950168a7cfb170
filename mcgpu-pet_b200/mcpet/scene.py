"""Python view of the C ABI: scenes, runs, outputs and verification probes.

This is the thin test/benchmark binding over ``libmcpet.so``; every call goes
through the C ABI of include/mcpet.h.  Host results come back as numpy
arrays; device runs take torch CUDA tensors (used for device-resident timing).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return a.ctypes.data


@dataclass
class RunOptions:
    """Options of one transport run (mcpet_run_opts)."""

    lane_mode: int = _abi.LANES_REFERENCE
    background_mode: bool = False
    histories_per_lane: int = 0
    block_threads: int = 0
    blocks_per_sm: int = 0
    collect_counters: bool = False
    seed_override: int = 0
    stream: int = 0
    algorithm: int = _abi.ALGORITHM_AUTO
    max_woodcock_steps: int = 0     # device loop guards (<= 0: defaults 2^20 / 2^16)
    max_rejections: int = 0

    def to_c(self) -> _abi.RunOpts:
        o = _abi.RunOpts()
        o.lane_mode = int(self.lane_mode)
        o.background_mode = int(bool(self.background_mode))
        o.histories_per_lane = int(self.histories_per_lane)
        o.block_threads = int(self.block_threads)
        o.blocks_per_sm = int(self.blocks_per_sm)
        o.collect_counters = int(bool(self.collect_counters))
        o.seed_override = int(self.seed_override)
        o.stream = self.stream or None
        o.algorithm = int(self.algorithm)
        o.max_woodcock_steps = int(self.max_woodcock_steps)
        o.max_rejections = int(self.max_rejections)
        return o


@dataclass
class RunResult:
    trues: Optional[np.ndarray]
    scatter: Optional[np.ndarray]
    image_trues: Optional[np.ndarray]
    image_scatter: Optional[np.ndarray]
    spectrum: np.ndarray
    psf: Optional[np.ndarray]          # structured array of PSF records
    psf_count: int
    total_histories: int
    transport_ms: float
    counters: dict = field(default_factory=dict)
    detected: int = 0                  # coincidences counted by the kernel
    material_dose: Optional[np.ndarray] = None   # uint64 [15, 2]: sum Edep (eV), sum Edep^2
    voxel_dose: Optional[np.ndarray] = None      # uint64 [n_dose_voxels, 2] over the dose ROI

    @property
    def coincidences(self) -> int:
        t = 0 if self.trues is None else int(self.trues.sum(dtype=np.int64))
        s = 0 if self.scatter is None else int(self.scatter.sum(dtype=np.int64))
        return t + s


PSF_DTYPE = np.dtype(
    [
        ("emission_time_ps", "<u8"),
        ("travel_time_ps", "<f4"),
        ("emission_absvox", "<i4"),
        ("energy", "<f4"),
        ("z", "<f4"),
        ("phi", "<f4"),
        ("vx", "<f4"),
        ("vy", "<f4"),
        ("vz", "<f4"),
        ("index1", "<i2"),
        ("index2", "<i2"),
    ]
)
assert PSF_DTYPE.itemsize == _abi.PSF_RECORD_BYTES


def _device_tallies(tallies: dict) -> _abi.Tallies:
    """mcpet_tallies over a dict of torch CUDA tensors (see Scene.run_device)."""
    def p(name):
        x = tallies.get(name)
        return None if x is None else x.data_ptr()

    t = _abi.Tallies()
    t.trues, t.scatter = p("trues"), p("scatter")
    t.image_trues, t.image_scatter = p("image_trues"), p("image_scatter")
    t.spectrum = p("spectrum")
    t.psf = p("psf")
    t.psf_capacity = 0 if tallies.get("psf") is None else tallies["psf"].numel() // _abi.PSF_RECORD_BYTES
    t.psf_count = p("psf_count")
    t.total_histories = p("histories")
    t.coincidences = p("coincidences")
    t.counters = p("counters")
    t.material_dose = p("material_dose")
    t.voxel_dose = p("voxel_dose")
    return t


def device_tallies_for(scene: "Scene", device=None, psf_capacity: int = 0) -> dict:
    """Fresh torch CUDA tensors for one scene's device tallies."""
    import torch
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    cfg, info = scene.config, scene.info
    nb, nv, ne = int(cfg.n_bins), int(info.n_voxels), int(cfg.n_energy_bins)
    t = {
        "trues": torch.empty(nb, dtype=torch.int32, device=dev),
        "scatter": torch.empty(nb, dtype=torch.int32, device=dev),
        "image_trues": torch.empty(nv, dtype=torch.int32, device=dev),
        "image_scatter": torch.empty(nv, dtype=torch.int32, device=dev),
        "spectrum": torch.empty(ne, dtype=torch.int32, device=dev),
        "psf_count": torch.zeros(1, dtype=torch.int32, device=dev),
        "histories": torch.zeros(1, dtype=torch.int64, device=dev),
        "coincidences": torch.zeros(1, dtype=torch.int64, device=dev),
    }
    if psf_capacity > 0:
        t["psf"] = torch.empty(psf_capacity * _abi.PSF_RECORD_BYTES, dtype=torch.uint8, device=dev)
    return t


def autotune(scenes: list, tallies: list, opts: Optional[RunOptions] = None,
             sample_decays: float = 2.0e8) -> tuple:
    """Pick histories_per_lane and block_threads for these scenes
    (mcpet_autotune): returns (RunOptions with the chosen values, dict with
    the sample times).  ``tallies[k]`` are scene k's device tallies (as for
    Scene.run_device); they are overwritten."""
    import dataclasses
    opts = opts or RunOptions(lane_mode=_abi.LANES_BALANCED)
    arr = (_abi.Tallies * len(scenes))(*[_device_tallies(t) for t in tallies])
    ptrs = (C.c_void_p * max(len(scenes), 1))(*[sc._h.value for sc in scenes])
    co = opts.to_c()
    r = _abi.TuneResult()
    check(lib().mcpet_autotune(ptrs, len(scenes), C.byref(co), arr, float(sample_decays), C.byref(r)))
    tuned = dataclasses.replace(opts, block_threads=r.block_threads,
                                histories_per_lane=r.histories_per_lane or opts.histories_per_lane)
    return tuned, {"block_threads": r.block_threads, "histories_per_lane": r.histories_per_lane,
                   "best_ms": r.best_ms, "auto_ms": r.auto_ms, "sample_fraction": r.sample_fraction,
                   "candidates": r.candidates}


class BatchGraph:
    """A batched run captured in a CUDA graph (mcpet_batch_graph_*): every
    launch() regenerates all scenes' histories with the next seeds (seed_k +
    r * seed_step) into ``tallies[k]`` (torch CUDA tensors, as for
    Scene.run_device), with one graph launch and no host work."""

    def __init__(self, scenes: list, tallies: list, opts: Optional[RunOptions] = None, seed_step: int = 1):
        opts = opts or RunOptions(lane_mode=_abi.LANES_BALANCED)
        self._scenes = list(scenes)          # the graph reads their device data
        self._tallies = list(tallies)
        arr = (_abi.Tallies * len(scenes))(*[_device_tallies(t) for t in tallies])
        ptrs = (C.c_void_p * max(len(scenes), 1))(*[sc._h.value for sc in scenes])
        co = opts.to_c()
        h = C.c_void_p()
        check(lib().mcpet_batch_graph_create(ptrs, len(scenes), C.byref(co), arr, int(seed_step), C.byref(h)))
        self._h = h

    def launch(self, stream=None) -> None:
        check(lib().mcpet_batch_graph_launch(self._h, stream))

    def set_seeds(self, seeds, stream=None) -> None:
        a = (C.c_int * len(self._scenes))(*[int(x) for x in seeds])
        check(lib().mcpet_batch_graph_set_seeds(self._h, C.cast(a, C.c_void_p), stream))

    def guard_trips(self) -> int:
        v = C.c_ulonglong(0)
        check(lib().mcpet_batch_graph_guard_trips(self._h, C.byref(v)))
        return int(v.value)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().mcpet_batch_graph_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_config(in_path: str) -> _abi.Config:
    cfg = _abi.Config()
    check(lib().mcpet_config_read(os.fsencode(in_path), C.byref(cfg)))
    return cfg


class _HostRun:
    """Host (numpy) buffers of one run and the mcpet_tallies pointing at them."""

    def __init__(self, scene: "Scene", psf_capacity: Optional[int]):
        cfg, info = scene.config, scene.info
        sino = cfg.tally_psf_sinogram in (0, 2)
        want_psf = cfg.tally_psf_sinogram in (0, 1)
        nb, nv = int(cfg.n_bins), int(info.n_voxels)
        self.trues = np.zeros(nb, np.int32) if sino else None
        self.scatter = np.zeros(nb, np.int32) if sino else None
        self.img_t = np.zeros(nv, np.int32) if sino else None
        self.img_s = np.zeros(nv, np.int32) if sino else None
        self.spec = np.zeros(max(cfg.n_energy_bins, 1), np.int32)
        self.cap = int(cfg.psf_size if psf_capacity is None else psf_capacity) if want_psf else 0
        self.psf = np.zeros(self.cap, PSF_DTYPE) if self.cap > 0 else None
        self.psf_count = C.c_int32(0)
        self.hist = C.c_ulonglong(0)
        self.det = C.c_ulonglong(0)
        self.ms = C.c_double(0)
        self.cnt = _abi.Counters()
        t = _abi.Tallies()
        t.trues, t.scatter = _ptr(self.trues), _ptr(self.scatter)
        t.image_trues, t.image_scatter = _ptr(self.img_t), _ptr(self.img_s)
        t.spectrum = _ptr(self.spec)
        t.psf = _ptr(self.psf) if self.psf is not None else None
        t.psf_capacity = self.cap
        t.psf_count = C.addressof(self.psf_count)
        t.total_histories = C.addressof(self.hist)
        t.coincidences = C.addressof(self.det)
        t.counters = C.addressof(self.cnt)
        t.transport_ms = C.addressof(self.ms)
        self.mdose = np.zeros((_abi.MAX_MATERIALS, 2), np.uint64) if cfg.tally_material_dose else None
        nd = int(info.n_dose_voxels)
        self.vdose = np.zeros((nd, 2), np.uint64) if nd > 0 else None
        t.material_dose = _ptr(self.mdose) if self.mdose is not None else None
        t.voxel_dose = _ptr(self.vdose) if self.vdose is not None else None
        self.t = t

    def result(self) -> RunResult:
        n = self.psf_count.value
        counters = {name: int(getattr(self.cnt, name)) for name, _ in _abi.Counters._fields_}
        psf = self.psf[: max(0, min(n, self.cap))] if self.psf is not None else None
        return RunResult(self.trues, self.scatter, self.img_t, self.img_s, self.spec, psf, n, int(self.hist.value),
                         float(self.ms.value), counters, int(self.det.value), self.mdose, self.vdose)


class Scene:
    """A loaded phantom + material tables (+ its device copy)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    # -- construction ------------------------------------------------------
    @classmethod
    def load(cls, in_path: str) -> "Scene":
        h = C.c_void_p()
        check(lib().mcpet_scene_load(os.fsencode(in_path), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, cfg: _abi.Config, material: np.ndarray, density: np.ndarray, activity: np.ndarray,
                    voxel_size_cm) -> "Scene":
        """Arrays shaped (nz, ny, nx) (x fastest in memory), material 1-based."""
        material = np.ascontiguousarray(material, dtype=np.int32)
        density = np.ascontiguousarray(density, dtype=np.float32)
        activity = np.ascontiguousarray(activity, dtype=np.float32)
        nz, ny, nx = material.shape
        vs = np.ascontiguousarray(voxel_size_cm, dtype=np.float32)
        h = C.c_void_p()
        check(lib().mcpet_scene_from_arrays(C.byref(cfg), nx, ny, nz, _ptr(vs), _ptr(material), _ptr(density),
                                            _ptr(activity), C.byref(h)))
        return cls(h.value)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().mcpet_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- queries -----------------------------------------------------------
    @property
    def config(self) -> _abi.Config:
        cfg = _abi.Config()
        check(lib().mcpet_scene_get_config(self._h, C.byref(cfg)))
        return cfg

    @property
    def info(self) -> _abi.SceneInfo:
        info = _abi.SceneInfo()
        check(lib().mcpet_scene_get_info(self._h, C.byref(info)))
        return info

    def set_activity(self, activity: np.ndarray) -> None:
        a = np.ascontiguousarray(activity, dtype=np.float32).ravel()
        assert a.size == self.info.n_voxels
        check(lib().mcpet_scene_set_activity(self._h, _ptr(a)))

    def export_tables(self) -> dict:
        """Host tables in the reference layout (for parity checks)."""
        info = self.info
        ne, nv = info.n_energy, info.n_voxels
        M, S, R = _abi.MAX_MATERIALS, _abi.MAX_SHELLS, _abi.NP_RAYLEIGH
        t = {
            "woodcock": np.zeros((ne, 2), np.float32),
            "mfp_a": np.zeros((ne, M, 3), np.float32),
            "mfp_b": np.zeros((ne, M, 3), np.float32),
            "voxels": np.zeros((nv, 3), np.float32),
            "fco": np.zeros(S * M, np.float32),
            "uico": np.zeros(S * M, np.float32),
            "fj0": np.zeros(S * M, np.float32),
            "noscco": np.zeros(M, np.int32),
            "xco": np.zeros(M * R, np.float32),
            "pco": np.zeros(M * R, np.float32),
            "aco": np.zeros(M * R, np.float32),
            "bco": np.zeros(M * R, np.float32),
            "pmax": np.zeros((ne, M), np.float32),
            "itlco": np.zeros(M * R, np.uint8),
            "ituco": np.zeros(M * R, np.uint8),
        }
        order = ["woodcock", "mfp_a", "mfp_b", "voxels", "fco", "uico", "fj0", "noscco", "xco", "pco", "aco", "bco",
                 "pmax", "itlco", "ituco"]
        check(lib().mcpet_scene_export_tables(self._h, *[_ptr(t[k]) for k in order]))
        return t

    # -- runs ----------------------------------------------------------------
    def to_device(self, device: int = -1) -> None:
        check(lib().mcpet_scene_to_device(self._h, device))

    def _host_run(self, psf_capacity: Optional[int] = None) -> "_HostRun":
        return _HostRun(self, psf_capacity)

    def run(self, opts: Optional[RunOptions] = None, psf_capacity: Optional[int] = None) -> RunResult:
        """End-to-end run into host (numpy) buffers (mcpet_run)."""
        opts = opts or RunOptions()
        h = self._host_run(psf_capacity)
        co = opts.to_c()
        check(lib().mcpet_run(self._h, C.byref(co), C.byref(h.t)))
        return h.result()

    def run_psf_stream(self, chunk_records: int, opts: Optional[RunOptions] = None, sink=None) -> RunResult:
        """Run with the PSF streamed in chunks (mcpet_run_psf_stream).  sink(records)
        receives each chunk as a PSF_DTYPE array; without a sink the chunks
        are concatenated into RunResult.psf."""
        opts = opts or RunOptions()
        h = self._host_run(0)
        chunks = []

        def _cb(ptr, n, _user):
            try:
                buf = (C.c_ubyte * (int(n) * _abi.PSF_RECORD_BYTES)).from_address(ptr)
                rec = np.frombuffer(bytes(buf), dtype=PSF_DTYPE)
                if sink is not None:
                    return 1 if sink(rec) is False else 0
                chunks.append(rec)
                return 0
            except Exception:       # never let an exception cross the C boundary
                return 1

        cb = _abi.PSF_SINK(_cb)
        co = opts.to_c()
        check(lib().mcpet_run_psf_stream(self._h, C.byref(co), int(chunk_records), C.cast(cb, C.c_void_p), None,
                                         C.byref(h.t)))
        r = h.result()
        r.psf = np.concatenate(chunks) if chunks else np.zeros(0, PSF_DTYPE)
        r.psf_count = int(h.psf_count.value)
        return r

    @staticmethod
    def run_batch(scenes: list, opts: Optional[RunOptions] = None,
                  psf_capacity: Optional[int] = None) -> list:
        """Several scenes in one batched run (mcpet_run_batch: small scenes in
        one launch, large ones in chained launches of their own); one
        RunResult per scene, each equal to scene.run(opts) on its own.
        transport_ms is the time of all the launches; counters (if requested)
        are their totals, reported on the first result."""
        opts = opts or RunOptions()
        hs = [sc._host_run(psf_capacity) for sc in scenes]
        arr = (_abi.Tallies * len(hs))(*[h.t for h in hs])
        ptrs = (C.c_void_p * max(len(scenes), 1))(*[sc._h.value for sc in scenes])
        co = opts.to_c()
        check(lib().mcpet_run_batch(ptrs, len(scenes), C.byref(co), arr))
        return [h.result() for h in hs]

    def run_into(self, host: dict, opts: Optional[RunOptions] = None) -> dict:
        """End-to-end run (mcpet_run) writing into caller-provided host buffers
        (numpy arrays or pinned torch CPU tensors): trues, scatter,
        image_trues, image_scatter, spectrum.  Returns the scalar results."""
        opts = opts or RunOptions()

        def p(name):
            x = host.get(name)
            if x is None:
                return None
            return x.data_ptr() if hasattr(x, "data_ptr") else _ptr(x)

        psf_count = C.c_int32(0)
        hist = C.c_ulonglong(0)
        det = C.c_ulonglong(0)
        ms = C.c_double(0)
        t = _abi.Tallies()
        t.trues, t.scatter = p("trues"), p("scatter")
        t.image_trues, t.image_scatter = p("image_trues"), p("image_scatter")
        t.spectrum = p("spectrum")
        t.psf_count = C.addressof(psf_count)
        t.total_histories = C.addressof(hist)
        t.coincidences = C.addressof(det)
        t.transport_ms = C.addressof(ms)
        co = opts.to_c()
        check(lib().mcpet_run(self._h, C.byref(co), C.byref(t)))
        return {"coincidences": int(det.value), "total_histories": int(hist.value), "transport_ms": ms.value,
                "psf_count": psf_count.value}

    def run_async(self, host: dict, opts: Optional[RunOptions] = None) -> dict:
        """mcpet_run_async into caller-provided host buffers (pinned torch CPU
        tensors for overlapping copies): trues, scatter, image_trues,
        image_scatter, spectrum.  Returns a dict of ctypes scalars
        (coincidences, total_histories, psf_count) that hold the results once
        wait() returned; keep it and the buffers alive until then."""
        opts = opts or RunOptions()

        def p(name):
            x = host.get(name)
            if x is None:
                return None
            return x.data_ptr() if hasattr(x, "data_ptr") else _ptr(x)

        res = {"coincidences": C.c_ulonglong(0), "total_histories": C.c_ulonglong(0), "psf_count": C.c_int32(0),
               "tallies": _abi.Tallies()}
        t = res["tallies"]
        t.trues, t.scatter = p("trues"), p("scatter")
        t.image_trues, t.image_scatter = p("image_trues"), p("image_scatter")
        t.spectrum = p("spectrum")
        t.psf_count = C.addressof(res["psf_count"])
        t.total_histories = C.addressof(res["total_histories"])
        t.coincidences = C.addressof(res["coincidences"])
        co = opts.to_c()
        check(lib().mcpet_run_async(self._h, C.byref(co), C.byref(t)))
        return res

    def lane_plan(self, lane_mode: int = _abi.LANES_BALANCED, histories_per_lane: int = 0) -> dict:
        """The lane plan a run with these settings uses (mcpet_scene_lane_plan;
        host only): arrays voxel, n_lanes, first_lane, stream_base, inv_rate in
        launch order, and the total lane count."""
        n = C.c_longlong(0)
        tot = C.c_ulonglong(0)
        L = lib()
        st = L.mcpet_scene_lane_plan(self._h, lane_mode, histories_per_lane, 0, None, None, None, None, None,
                                     C.byref(n), C.byref(tot))
        if st not in (0, 6):
            check(st)
        k = n.value
        out = {"voxel": np.zeros(k, np.uint32), "n_lanes": np.zeros(k, np.uint32),
               "first_lane": np.zeros(k, np.uint64), "stream_base": np.zeros(k, np.uint64),
               "inv_rate": np.zeros(k, np.float64)}
        check(L.mcpet_scene_lane_plan(self._h, lane_mode, histories_per_lane, k, *[_ptr(out[f]) for f in
                                      ("voxel", "n_lanes", "first_lane", "stream_base", "inv_rate")],
                                      C.byref(n), C.byref(tot)))
        out["total_lanes"] = int(tot.value)
        return out

    def wait(self) -> None:
        """mcpet_run_wait: block until the scene's asynchronous runs are done."""
        check(lib().mcpet_run_wait(self._h))

    def last_upload_bytes(self) -> int:
        return int(self.info.last_h2d_bytes)

    def run_device(self, tallies: dict, opts: Optional[RunOptions] = None, time_it: bool = False) -> float:
        """Run into caller-owned torch CUDA tensors (mcpet_run_device).

        ``tallies`` holds int32 tensors trues/scatter/image_trues/image_scatter/
        spectrum, an int32 psf_count[1] and an int64 histories[1] (optionally
        a uint8 psf[capacity*44] and int64 counters[10]).  Returns the
        transport time in ms when ``time_it`` (this synchronises)."""
        opts = opts or RunOptions()
        ms = C.c_double(0)
        t = _device_tallies(tallies)
        t.transport_ms = C.addressof(ms) if time_it else None
        co = opts.to_c()
        check(lib().mcpet_run_device(self._h, C.byref(co), C.byref(t)))
        return float(ms.value)

    @staticmethod
    def run_batch_device(scenes: list, tallies: list, opts: Optional[RunOptions] = None,
                         time_it: bool = False) -> float:
        """Several scenes in one batched run into device tallies
        (mcpet_run_batch_device); ``tallies[k]`` as for run_device.  Returns
        the run's transport time in ms when ``time_it``."""
        opts = opts or RunOptions()
        ms = C.c_double(0)
        arr = (_abi.Tallies * len(scenes))(*[_device_tallies(t) for t in tallies])
        if time_it:
            arr[0].transport_ms = C.addressof(ms)
        ptrs = (C.c_void_p * max(len(scenes), 1))(*[sc._h.value for sc in scenes])
        co = opts.to_c()
        check(lib().mcpet_run_batch_device(ptrs, len(scenes), C.byref(co), arr))
        return float(ms.value)

    def guard_trips(self) -> int:
        v = C.c_ulonglong(0)
        check(lib().mcpet_last_run_guard(self._h, C.byref(v)))
        return int(v.value)

    def write_outputs(self, result: RunResult, out_dir: Optional[str] = None, background_mode: bool = False) -> None:
        t = _abi.Tallies()
        t.trues, t.scatter = _ptr(result.trues), _ptr(result.scatter)
        t.image_trues, t.image_scatter = _ptr(result.image_trues), _ptr(result.image_scatter)
        t.spectrum = _ptr(result.spectrum)
        psf_count = C.c_int32(result.psf_count)
        hist = C.c_ulonglong(result.total_histories)
        if result.psf is not None:
            t.psf = _ptr(result.psf)
            t.psf_capacity = len(result.psf)
        t.psf_count = C.addressof(psf_count)
        t.total_histories = C.addressof(hist)
        if result.material_dose is not None:
            t.material_dose = _ptr(result.material_dose)
        if result.voxel_dose is not None:
            t.voxel_dose = _ptr(result.voxel_dose)
        check(lib().mcpet_write_outputs(self._h, C.byref(t), os.fsencode(out_dir) if out_dir else None,
                                        int(bool(background_mode)), result.transport_ms * 1e-3))


# -- verification probes (GPU) -----------------------------------------------

def probe_rng(seed: int, stream_ids, ndraw: int = 8):
    ids = np.ascontiguousarray(stream_ids, dtype=np.int64)
    n = len(ids)
    seeds = np.zeros((n, 2), np.int32)
    f = np.zeros((n, ndraw), np.float32)
    d = np.zeros((n, ndraw), np.float64)
    check(lib().mcpet_probe_rng(n, int(seed), _ptr(ids), ndraw, _ptr(seeds), _ptr(f), _ptr(d)))
    return seeds, f, d


def probe_detector(scene: Scene, ev: dict) -> np.ndarray:
    n = len(ev["e2"])
    a = {k: np.ascontiguousarray(ev[k], dtype=(np.int8 if k.startswith("st") else
                                               np.int32 if k == "seeds" else np.float32)) for k in
         ["e2", "e1", "pos2", "pos1", "dir2", "dir1", "st2", "st1", "seeds"]}
    out = np.zeros((n, 6), np.int32)
    check(lib().mcpet_probe_detector(scene.handle, n, _ptr(a["e2"]), _ptr(a["e1"]), _ptr(a["pos2"]),
                                     _ptr(a["pos1"]), _ptr(a["dir2"]), _ptr(a["dir1"]), _ptr(a["st2"]),
                                     _ptr(a["st1"]), _ptr(a["seeds"]), _ptr(out)))
    return out


def probe_compton(scene: Scene, energy, mat, seeds):
    e = np.ascontiguousarray(energy, np.float32)
    m = np.ascontiguousarray(mat, np.int32)
    s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
    n = len(e)
    e_out = np.zeros(n, np.float32)
    c_out = np.zeros(n, np.float64)
    s_out = np.zeros((n, 2), np.int32)
    check(lib().mcpet_probe_compton(scene.handle, n, _ptr(e), _ptr(m), _ptr(s), _ptr(e_out), _ptr(c_out),
                                    _ptr(s_out)))
    return e_out, c_out, s_out


def probe_rayleigh(scene: Scene, energy, mat, pmax, seeds):
    e = np.ascontiguousarray(energy, np.float32)
    m = np.ascontiguousarray(mat, np.int32)
    p = np.ascontiguousarray(pmax, np.float32)
    s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
    n = len(e)
    c_out = np.zeros(n, np.float64)
    s_out = np.zeros((n, 2), np.int32)
    check(lib().mcpet_probe_rayleigh(scene.handle, n, _ptr(e), _ptr(m), _ptr(p), _ptr(s), _ptr(c_out),
                                     _ptr(s_out)))
    return c_out, s_out


def probe_source(shape, inv_voxel_size, seeds, background: bool = False, balanced: bool = False):
    """Photon pairs of every voxel (mcpet_probe_source); balanced: the
    balanced lanes' photon-2 emission."""
    nz, ny, nx = shape
    inv = np.ascontiguousarray(inv_voxel_size, np.float32)
    s = np.ascontiguousarray(seeds, np.int32).reshape(-1, 2)
    out = np.zeros((nx * ny * nz, 4, 3), np.float32)
    s_out = np.zeros_like(s)
    mode = int(bool(background)) | (2 if balanced else 0)
    check(lib().mcpet_probe_source(nx, ny, nz, _ptr(inv), mode, _ptr(s), _ptr(out), _ptr(s_out)))
    return out, s_out
