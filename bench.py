#!/usr/bin/env python
"""Benchmark of the photon-transport path: detected coincidences per second.

Workload (one step): the head-like phantom -- 128x128x64 voxels of 2 mm, 8
water-equivalent tissues as seeded nested ellipsoids, FDG-like activity scaled
to 1e9 decays in a 1 s acquisition -- seen by a 41 cm radius, 64-ring scanner
binned into a 256 x 256 x 8065 (span 1) int32 sinogram pair.  A step zeroes
the tallies and runs the full transport of those 1e9 decays (2e9 photons).

Arms:
  default           this library on the GPU(s): device-resident timed steps
                    (value), plus end-to-end steps through the host-buffer
                    C-ABI call mcpet_run_async (e2e; the blocking mcpet_run is
                    timed beside it), the gradient of the sinogram
                    log-likelihood (gradient), the reference's own CUDA
                    build on the same input file and GPU (ref_cuda), and the
                    reference's own CPU implementation on a fixed voxel
                    sample (cpu_baseline).
                    --batch-scenes N adds the many-phantom batch, autotuner
                    and CUDA-graph measurements; --beds N the long-axial body
                    workload with N bed positions and its gradient.
  --impl reference  the reference's own CPU implementation (its loaders and
                    its transport kernel compiled for the host, all cores;
                    no part of this library is loaded) on the same fixed
                    voxel sample of the workload in every step.

Multi-GPU: one process per GPU (torchrun); every rank runs an independent
replica with its own seed (the transport has no exchange step); value = all
detected coincidences / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mcgpu-pet_b200"))

METRIC = "coincidences/s on 1 B200 vs ref CUDA (χ²-matched); gradient time/forward"
UNIT = "coincidences/s"
WORKLOAD = ("head-like phantom 128x128x64 voxels @ 2 mm, 8 tissues (seeded nested ellipsoids), FDG-like "
            "activity, 1e9 decays (511 keV pairs); scanner R=41 cm, 64 rings x 4 mm, sinogram 256 rad x 256 ang "
            "x 8065 planes (span 1, MRD 63) int32 trues+scatter, 12% energy resolution, 350-600 keV")
EMISSIONS = 1.0e9
PHANTOM_SEED = 2024


def bench_config(emissions: float, n_gpus: int) -> dict:
    """The workload as both arms report it."""
    return {"workload": WORKLOAD, "emissions_per_step_per_gpu": emissions, "parallelism": f"replicas x{n_gpus}",
            "l2": "each step zeroes 4.2 GB of sinograms (> 126 MB L2) before the transport"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_workload(workdir: str, emissions: float, scanner: str = "head"):
    from mcpet import inputs
    mat, rho, act, vs, used, scan = inputs.head_workload(emissions, scanner)
    spec = inputs.spec_for(inputs.tissue_materials(used), "unused.vox", **scan)
    cfg = inputs.config_from_spec(spec, workdir)
    return cfg, mat, rho, act, vs


def write_workload_files(workdir: str, emissions: float) -> str:
    """The head workload as the reference reads it: a .vox phantom and a .in
    input file (written by the pure-Python writers of mcpet.inputs, which
    load no library).  Returns the .in path."""
    from mcpet import inputs
    mat, rho, act, vs, used, scan = inputs.head_workload(emissions)
    vox = inputs.write_vox(os.path.join(workdir, "head_workload.vox"), mat, rho, act, vs)
    spec = inputs.spec_for(inputs.tissue_materials(used), vox, **scan)
    return inputs.write_input(os.path.join(workdir, "head_workload.in"), spec)


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(counters: dict) -> int:
    """B_alg = 8 S + 24 M + 8 W + 8 T: voxel material+density per Woodcock step
    inside the phantom, interaction-table refresh (2 x float3), majorant
    refresh (float2), int32 tally increment (read + write)."""
    return (8 * counters["woodcock_steps_inside"] + 24 * counters["table_refreshes"] +
            8 * counters["majorant_refreshes"] + 8 * counters["tally_increments"])


class ReferenceCPU:
    """The reference's own CPU path for the workload: its input file, voxel
    file and material tables loaded by its own read_input / load_voxels /
    load_material (MCGPU-PET.cu:866-1831, the host code of
    oracle/_ref/libref_prog.so), and its transport kernel compiled for the
    host (oracle/_ref/libref_cpu.so, OpenMP over voxel blocks, all host
    threads).  Nothing of this library is loaded."""

    def __init__(self, in_path: str, workdir: str):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import refbind
        self.refbind = refbind
        cfg, self.voxels, self.tables = refbind.RefIO().load(in_path, cwd=workdir)
        self.params = refbind.Params.from_buffer_copy(cfg)
        self.cpu = refbind.RefCPU()
        self.cores = os.cpu_count() or 1
        emit = np.nonzero(self.voxels[:, 2] > 1e-7)[0]
        self.n_emitting = len(emit)
        self.order = np.random.default_rng(7).permutation(emit).astype(np.int32)
        self.cum = np.cumsum(self.voxels[self.order, 2].astype(np.float64)) * (self.params.acq_ps * 1e-12)
        self.total_decays = float(self.cum[-1])

    def sample(self, decays: float) -> np.ndarray:
        """The first voxels of a fixed seeded permutation of the emitting
        voxels whose expected decays reach `decays`: the same sample in
        every leg and every step."""
        n = int(np.searchsorted(self.cum, decays)) + 1
        return self.order[:min(n, len(self.order))]

    def run(self, blocks: np.ndarray):
        t0 = time.perf_counter()
        r = self.cpu.run(self.params, self.voxels, self.tables, block_list=blocks, n_threads=self.cores)
        dt = time.perf_counter() - t0
        return int(r["trues"].sum(dtype=np.int64) + r["scatter"].sum(dtype=np.int64)), dt

    def describe(self, blocks: np.ndarray, coinc: int, secs: float) -> str:
        decays = float(self.cum[len(blocks) - 1])
        return (f"{len(blocks)} of {self.n_emitting} emitting voxels (a fixed seeded sample, {decays:.3g} of the "
                f"workload's {self.total_decays:.3g} expected decays), each with the reference's "
                f"{self.params.tpb} lanes over the full {self.params.acq_ps * 1e-12:g} s acquisition; {coinc} "
                f"coincidences in {secs:.1f} s on {self.cores} threads (the reference's read_input / load_voxels / "
                f"load_material and its MCGPU-PET_kernel.cu compiled for the host with OpenMP)")


CPU_SAMPLE_DECAYS = 6.0e7     # 6 % of the head workload per CPU step (~5 s on 16 host threads)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    with tempfile.TemporaryDirectory() as tmp:
        ref = ReferenceCPU(write_workload_files(tmp, args.emissions), tmp)
        small = ref.sample(CPU_SAMPLE_DECAYS / 25)
        for _ in range(args.warmup):
            ref.run(small)
        blocks = ref.sample(args.cpu_sample_decays)
        coinc, secs = 0, 0.0
        for _ in range(args.steps):
            c, s = ref.run(blocks)
            coinc += c
            secs += s
        desc = ref.describe(blocks, coinc // max(args.steps, 1), secs / max(args.steps, 1))
        cores = ref.cores
    value = coinc / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded phantom; a fixed voxel sample of the workload per step)",
            "config": bench_config(args.emissions, args.gpus),
            "impl_config": {"arm": "reference CPU implementation (its loaders and its kernel compiled for the host)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def measure_reference_cuda(workdir: str, emissions: float) -> dict:
    """The reference's own CUDA build on this GPU, same workload: its
    read_input / load_voxels / load_material / init_CUDA_device and one
    track_particles launch timed with CUDA events (MCGPU-PET.cu:228-535,
    oracle/_ref/libref_prog.so); coincidences = sum of its trues and
    scatter sinograms (MCGPU-PET.cu:793-794)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import refbind
    in_path = write_workload_files(workdir, emissions)
    cfg, vox, _ = refbind.RefIO().load(in_path, cwd=workdir)
    nvox = cfg.nx * cfg.ny * cfg.nz
    r = refbind.RefProg().run(in_path, cfg.nbins, nvox, cfg.ne, cwd=workdir)
    coinc = int(r["trues"].sum(dtype=np.int64) + r["scatter"].sum(dtype=np.int64))
    return {"kernel_ms": r["kernel_ms"], "coincidences": coinc, "value": coinc / (r["kernel_ms"] * 1e-3),
            "unit": UNIT, "histories": r["total_histories"],
            "what": "reference CUDA build (its own loaders and track_particles launch, reference lanes, seed 12345), "
                    "kernel time from CUDA events on this GPU"}


PROMPT_GAMMA_EV = 1157020.0   # the prompt gamma of the batched workload's second emitter


def measure_batch(n_scenes: int, workdir: str, emissions_each: float = 1.0e8, replays: int = 3) -> dict:
    """Batched many-phantom workload (config C3): n_scenes head-like phantoms
    of uneven size, each its own seed; the even ones a pure 511 keV positron
    emitter, the odd ones an emitter with a 1157 keV prompt gamma at 100 %
    yield (every scene on the material tables continued to 1250 keV, which
    leave 511 keV results unchanged).  Device-resident tallies throughout;
    times are CUDA events on the launch stream.

    * sequential: the scenes one after another through mcpet_run_device
      (one launch each), the plain form of the run;
    * batched: one mcpet_run_batch_device call over all scenes (small
      scenes share a launch, large ones get chained launches of their own);
    * autotuned: mcpet_autotune picks histories per lane and block size on a
      sample, then the batched launch with that choice;
    * graph: the tuned batch captured once (mcpet_batch_graph_create) and
      replayed; every replay regenerates all histories with new seeds.
    Also checks that the batched tallies equal the sequential ones."""
    import torch
    import mcpet
    from mcpet import inputs
    sc, sizes = [], []
    for k, (mat, rho, act, vs, used) in enumerate(inputs.batch_phantoms(n_scenes, emissions_each)):
        kw = dict(inputs.scanner_batch(), seed=1000 + k)
        if k % 2:
            kw.update(prompt_gamma_energy=PROMPT_GAMMA_EV, prompt_gamma_yield=1.0)
        spec = inputs.spec_for(inputs.tissue_materials(list(inputs.TISSUES)[:8], extended=True), "unused.vox",
                               **kw)
        cfg = inputs.config_from_spec(spec, workdir)
        sc.append(mcpet.Scene.from_arrays(cfg, mat, rho, act, vs))
        sizes.append(mat.shape[0])
    tal = [mcpet.device_tallies_for(s) for s in sc]
    stream = torch.cuda.current_stream()
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, stream=stream.cuda_stream)

    def coinc():
        return sum(int(t["coincidences"].item()) for t in tal)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), time.perf_counter() - t0

    # each configuration runs once untimed first: a scene caches one lane
    # plan, and a change of options (the tuned histories per lane) rebuilds
    # it on the host
    for s, t in zip(sc, tal):
        s.run_device(t, opts)
    seq_ms, seq_wall = timed(lambda: [s.run_device(t, opts) for s, t in zip(sc, tal)])
    seq_c = coinc()
    mcpet.Scene.run_batch_device(sc, tal, opts)
    bat_ms, bat_wall = timed(lambda: mcpet.Scene.run_batch_device(sc, tal, opts))
    bat_c = coinc()

    t0 = time.perf_counter()
    tuned, tune = mcpet.autotune(sc, tal, opts, sample_decays=2.0e8 * max(1.0, n_scenes / 8))
    tune["wall_s"] = time.perf_counter() - t0
    mcpet.Scene.run_batch_device(sc, tal, tuned)
    tun_ms, tun_wall = timed(lambda: mcpet.Scene.run_batch_device(sc, tal, tuned))
    tun_c = coinc()
    tun_trues = [t["trues"].clone() for t in tal[:4]]
    for s, t in zip(sc, tal):
        s.run_device(t, tuned)
    seqt_ms, seqt_wall = timed(lambda: [s.run_device(t, tuned) for s, t in zip(sc, tal)])
    seqt_c = coinc()
    # same explicit options: the batched tallies equal the one-by-one ones
    identical = tun_c == seqt_c and all(bool(torch.equal(a, t["trues"])) for a, t in zip(tun_trues, tal[:4]))

    g = mcpet.BatchGraph(sc, tal, tuned, seed_step=1)
    g.launch(stream.cuda_stream)                 # warm-up replay
    graph_c = 0
    graph_ms, graph_wall = 0.0, 0.0
    for _ in range(replays):
        ms, wall = timed(lambda: g.launch(stream.cuda_stream))
        graph_ms += ms
        graph_wall += wall
        graph_c += coinc()
    guard = g.guard_trips()
    g.close()
    for s in sc:
        s.close()
    rate = lambda c, ms: c / (ms * 1e-3)
    return {"workload": f"{n_scenes} head-like phantoms of m^3 voxels, m in [32,192] (min {min(sizes)}, max "
                        f"{max(sizes)}), 2-4 mm voxels, {emissions_each:.0e} decays each, own seed each; half "
                        "pure 511 keV emitters, half with a 1157 keV prompt gamma at 100 % yield (tables to 1250 "
                        "keV); scanner 32 rings, 128 rad x 128 ang x 1985 planes (span 1); device-resident tallies",
            "unit": UNIT, "tuned_batch_identical_to_tuned_sequential": identical,
            "sequential": {"ms": seq_ms, "wall_s": seq_wall, "value": rate(seq_c, seq_ms), "launches": n_scenes},
            "batched": {"ms": bat_ms, "wall_s": bat_wall, "value": rate(bat_c, bat_ms), "calls": 1},
            "sequential_tuned": {"ms": seqt_ms, "wall_s": seqt_wall, "value": rate(seqt_c, seqt_ms),
                                 "launches": n_scenes},
            "autotune": tune,
            "batched_tuned": {"ms": tun_ms, "wall_s": tun_wall, "value": rate(tun_c, tun_ms),
                              "histories_per_lane": tuned.histories_per_lane, "block_threads": tuned.block_threads},
            "graph": {"replays": replays, "ms_per_replay": graph_ms / replays, "wall_s_per_replay": graph_wall / replays,
                      "value": rate(graph_c, graph_ms), "guard_trips": guard},
            "graph_vs_sequential": rate(graph_c, graph_ms) / rate(seq_c, seq_ms),
            "batched_vs_sequential": rate(bat_c, bat_ms) / rate(seq_c, seq_ms)}


def measure_gradient(workdir: str, emissions: float = 2.0e8) -> dict:
    """Gradient of the sinogram log-likelihood on the head phantom (2e8
    decays): the measured sinogram is another seed's forward run with grey
    matter activity x1.5 plus 5 % uniform randoms.  Reports the device time
    of the gradient call (forward with event records + log-likelihood +
    replay) against a plain forward run of the same scene."""
    import torch
    import mcpet
    from mcpet import grad as G
    from mcpet import inputs
    mat, rho, act, vs, used = inputs.head_phantom(shape=(64, 128, 128), voxel_cm=0.2, seed=PHANTOM_SEED,
                                                  total_bq=emissions)
    spec = inputs.spec_for(inputs.tissue_materials(used), "unused.vox", seed=12345, **inputs.scanner_for_head())
    cfg = inputs.config_from_spec(spec, workdir)
    act_true = act.copy()
    act_true[mat == inputs.TISSUES["grey"][0]] *= 1.5
    sc_t = mcpet.Scene.from_arrays(cfg, mat, rho, act_true, vs)
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, seed_override=777)
    t = G._device_tallies(sc_t, torch, torch.device("cuda"))
    sc_t.run_device(t, opts)
    tot = (t["trues"] + t["scatter"]).to(torch.float32)
    bg = torch.full_like(tot, 0.05 * float(tot.sum()) / tot.numel())
    y = tot + torch.poisson(bg)
    sc_t.close()
    del t, tot
    sc = mcpet.Scene.from_arrays(cfg, mat, rho, act, vs)
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED)
    tall = G._device_tallies(sc, torch, torch.device("cuda"))
    r = G.grad(sc, y, bg, opts, tallies=tall)             # warm-up (event buffer, device activity)
    plain = [sc.run_device(tall, opts, time_it=True) for _ in range(3)]
    runs = [G.grad(sc, y, bg, opts, tallies=tall) for _ in range(3)]
    r = runs[-1]
    fwd = min(x.forward_ms for x in runs)
    gms = min(x.gradient_ms for x in runs)
    sc.close()
    return {"workload": f"head phantom 128x128x64 @ 2 mm, {emissions:.0e} decays, 64-ring scanner; measured "
                        "sinogram: another seed with grey-matter activity x1.5 plus 5% uniform randoms",
            "plain_forward_ms": min(plain), "forward_with_records_ms": fwd, "gradient_pass_ms": gms,
            "gradient_time_over_forward": (fwd + gms) / min(plain),
            "events": r.events, "replay_mismatches": r.mismatches, "loglik": r.loglik,
            "outputs": "dL/dA and dL/ds for every voxel"}


def measure_beds(n_beds: int, workdir: str, emissions_total: float = 5.0e9) -> dict:
    """Long-axial body workload (config C5 shapes): 256x256x400 body phantom
    at 2 mm with 10 tissues (lungs, bone, hot organ at 8x), 1 m scanner of
    256 rings, 384 x 384 x 12333-plane span-11 sinograms (1.82e9 bins, int32),
    n_beds bed positions 20 cm apart sharing emissions_total decays.  The beds
    run batched and one by one (mcpet_run_batch_device vs
    mcpet_run_device, device-resident tallies, CUDA events); then the
    activity and density-scale gradient of one bed's sinogram
    log-likelihood (mcpet_grad) against a plain forward of that bed."""
    import torch
    import mcpet
    from mcpet import grad as G
    from mcpet import inputs
    mat, rho, act, vs, used = inputs.body_phantom(seed=2025, total_bq=emissions_total / n_beds)
    size = tuple(n * v for n, v in zip(mat.shape[::-1], vs))
    scan = inputs.scanner_long_axial()
    scan["detector_radius"] = 39.0
    beds = []
    for k, c in enumerate(inputs.bed_centers(size, n_beds, 20.0)):
        spec = inputs.spec_for(inputs.tissue_materials(used), "unused.vox", seed=3000 + k, detector_center=c, **scan)
        beds.append(mcpet.Scene.from_arrays(inputs.config_from_spec(spec, workdir), mat, rho, act, vs))
    tal = [mcpet.device_tallies_for(b) for b in beds]
    stream = torch.cuda.current_stream()
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, stream=stream.cuda_stream)

    def coinc():
        return sum(int(t["coincidences"].item()) for t in tal)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # each configuration once untimed first (tables; the lane plans, which the
    # beds run alone and the batch size differently)
    for b, t in zip(beds, tal):
        b.run_device(t, opts)
    seq_ms = timed(lambda: [b.run_device(t, opts) for b, t in zip(beds, tal)])
    seq_c = coinc()
    mcpet.Scene.run_batch_device(beds, tal, opts)
    bat_ms = timed(lambda: mcpet.Scene.run_batch_device(beds, tal, opts))
    bat_c = coinc()
    per_bed = [int(t["coincidences"].item()) for t in tal]
    top = int(torch.nonzero(tal[0]["trues"]).max().item()) if bool(tal[0]["trues"].any()) else -1
    guard = beds[0].guard_trips()
    nbins = int(beds[0].config.n_bins)
    del tal
    torch.cuda.empty_cache()

    # gradient of bed 0: measured sinogram = another seed with the organ x1.5, plus 5 % randoms
    b0 = beds[0]
    act_t = act.copy()
    act_t[mat == inputs.TISSUES["organ"][0]] *= 1.5
    b0.set_activity(act_t)
    t = G._device_tallies(b0, torch, torch.device("cuda"))
    b0.run_device(t, mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, seed_override=4242))
    y = (t["trues"] + t["scatter"]).to(torch.float32)
    del t
    torch.cuda.empty_cache()
    bg = torch.full_like(y, 0.05 * float(y.sum()) / y.numel())
    y += torch.poisson(bg)
    b0.set_activity(act)
    tall = G._device_tallies(b0, torch, torch.device("cuda"))
    G.grad(b0, y, bg, opts, tallies=tall)                    # warm-up: event buffer, device activity
    plain = timed(lambda: b0.run_device(tall, opts))
    r = G.grad(b0, y, bg, opts, tallies=tall)
    for b in beds:
        b.close()
    rate = lambda c, ms: c / (ms * 1e-3)
    return {"workload": f"body phantom 256x256x400 @ 2 mm, 10 tissues (lung 0.3, bone 1.85, hot organ 8x), "
                        f"{emissions_total:.0e} decays over {n_beds} bed positions 20 cm apart; scanner R=39 cm, "
                        f"256 rings x 4 mm, 384 x 384 x 12333 span-11 sinograms ({nbins} bins, int32) per bed",
            "unit": UNIT, "batched": {"ms": bat_ms, "value": rate(bat_c, bat_ms), "calls": 1},
            "one_by_one": {"ms": seq_ms, "value": rate(seq_c, seq_ms), "launches": n_beds},
            "coincidences_per_bed": per_bed, "highest_bin_bed0": top, "guard_trips": guard,
            "gradient_bed0": {"plain_forward_ms": plain, "forward_with_records_ms": r.forward_ms,
                              "gradient_pass_ms": r.gradient_ms,
                              "gradient_time_over_forward": (r.forward_ms + r.gradient_ms) / plain,
                              "events": r.events, "replay_mismatches": r.mismatches}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mcpet", choices=["mcpet", "reference"])
    ap.add_argument("--emissions", type=float, default=EMISSIONS)
    ap.add_argument("--lanes", default="balanced", choices=["balanced", "reference"])
    ap.add_argument("--cpu-sample-decays", type=float, default=CPU_SAMPLE_DECAYS,
                    help="expected decays of the fixed voxel sample each CPU step runs")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip the reference CUDA build's run of the workload (ref_cuda)")
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--algorithm", default="auto", choices=["auto", "histories", "events"])
    ap.add_argument("--batch-scenes", type=int, default=32,
                    help="also time N phantoms of m^3 voxels (m in [32,192], 1e8 decays each) batched in one "
                         "launch against the same runs one by one (reported under 'batch'; 0: skip; one GPU only)")
    ap.add_argument("--batch-emissions", type=float, default=1.0e8, help="decays per phantom of --batch-scenes")
    ap.add_argument("--no-gradient", action="store_true", help="skip the gradient (mcpet_grad) measurement")
    ap.add_argument("--beds", type=int, default=0,
                    help="also measure the long-axial body workload with this many bed positions (not a bench line)")
    ap.add_argument("--block-threads", type=int, default=0, help="threads per block (0: automatic)")
    ap.add_argument("--histories-per-lane", type=int, default=0, help="balanced lanes: decays per lane (0: automatic)")
    ap.add_argument("--scanner", default="head", choices=["head", "head32"],
                    help="head32: smaller sinogram for profiler captures (not a bench line)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import mcpet

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lanes = mcpet.LANES_BALANCED if args.lanes == "balanced" else mcpet.LANES_REFERENCE

    tmp = tempfile.mkdtemp()
    cfg, mat, rho, act, vs = build_workload(tmp, args.emissions, args.scanner)
    scene = mcpet.Scene.from_arrays(cfg, mat, rho, act, vs)
    scene.to_device(local)
    nb, nv, ne = int(cfg.n_bins), int(scene.info.n_voxels), cfg.n_energy_bins
    tallies = {
        "trues": torch.empty(nb, dtype=torch.int32, device=dev),
        "scatter": torch.empty(nb, dtype=torch.int32, device=dev),
        "image_trues": torch.empty(nv, dtype=torch.int32, device=dev),
        "image_scatter": torch.empty(nv, dtype=torch.int32, device=dev),
        "spectrum": torch.empty(ne, dtype=torch.int32, device=dev),
        "psf_count": torch.zeros(1, dtype=torch.int32, device=dev),
        "histories": torch.zeros(1, dtype=torch.int64, device=dev),
        "coincidences": torch.zeros(1, dtype=torch.int64, device=dev),
        "counters": torch.zeros(10, dtype=torch.int64, device=dev),
    }
    stream = torch.cuda.current_stream(dev)
    base_seed = 12345 + 7919 * rank

    algorithm = {"auto": mcpet.ALGORITHM_AUTO, "histories": mcpet.ALGORITHM_HISTORIES,
                 "events": mcpet.ALGORITHM_EVENTS}[args.algorithm]

    def opts(step, counters=False):
        return mcpet.RunOptions(lane_mode=lanes, seed_override=base_seed + step, collect_counters=counters,
                                stream=stream.cuda_stream, algorithm=algorithm, block_threads=args.block_threads,
                                histories_per_lane=args.histories_per_lane)

    # algorithmic-byte counters of one launch (separate, untimed, same seed as step 0)
    scene.run_device(tallies, opts(0, counters=True))
    torch.cuda.synchronize()
    cvals = tallies["counters"].cpu().numpy().astype(np.int64)
    names = ["woodcock_steps_inside", "table_refreshes", "majorant_refreshes", "tally_increments", "photons",
             "compton", "rayleigh", "photoelectric", "lanes", "guard_trips"]
    counters = {n: int(v) for n, v in zip(names, cvals)}
    b_alg = algorithmic_bytes(counters)

    for w in range(args.warmup):
        scene.run_device(tallies, opts(1000 + w))
    torch.cuda.synchronize()

    coinc = torch.zeros(1, dtype=torch.int64, device=dev)
    kernel_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.steps):
        kernel_ms.append(scene.run_device(tallies, opts(k), time_it=True))
        coinc += tallies["coincidences"]
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    guard = scene.guard_trips()
    total = int(coinc.item())
    hist = int(tallies["histories"].item())
    if dist:
        t = torch.tensor([elapsed_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
        c = torch.tensor([total], device=dev, dtype=torch.int64)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        total = int(c.item())
    value = total / (elapsed_ms * 1e-3)
    avg_kernel_ms = sum(kernel_ms) / len(kernel_ms)

    # end to end through the host-buffer C-ABI call (inputs: the activity map,
    # turned into the lane plan and uploaded; outputs: sinograms, images,
    # spectrum downloaded into pinned host memory)
    e2e = None
    if args.e2e_steps > 0:
        # end to end through the host-buffer C-ABI: per step the activity map
        # goes in (lane plan built on the host and uploaded) and the sinograms,
        # images and spectrum come out into pinned host buffers.  Steps are
        # mcpet_run_async calls (two in flight: one step's downloads overlap
        # the next step's transport); the clock stops after mcpet_run_wait.
        # The blocking mcpet_run of the same step is timed too.
        # one pinned set: the downloads of consecutive steps are ordered on the
        # scene's copy stream, so they may land in the same host buffers
        names = (("trues", nb), ("scatter", nb), ("image_trues", nv), ("image_scatter", nv), ("spectrum", ne))
        pin = {k: torch.empty(n, dtype=torch.int32, pin_memory=True) for k, n in names}
        pins = [pin, pin]
        act_pinned = torch.from_numpy(np.ascontiguousarray(act.ravel())).pin_memory()

        def e2e_opts(k):
            return mcpet.RunOptions(lane_mode=lanes, seed_override=base_seed + 500 + k, algorithm=algorithm,
                                    block_threads=args.block_threads, histories_per_lane=args.histories_per_lane)

        for k in range(2):                         # warm-up: host plan builder, second tally set
            scene.set_activity(act_pinned.numpy())
            scene.run_async(pins[k], e2e_opts(k))
        scene.wait()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        res = []
        for k in range(args.e2e_steps):
            scene.set_activity(act_pinned.numpy())
            res.append(scene.run_async(pins[k % 2], e2e_opts(10 + k)))
        scene.wait()
        e2e_s = time.perf_counter() - t0
        e2e_coinc = sum(int(r["coincidences"].value) for r in res)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scene.set_activity(act_pinned.numpy())
        rb = scene.run_into(pins[0], e2e_opts(99))
        blocking_s = time.perf_counter() - t0
        h2d = scene.last_upload_bytes()
        d2h = 2 * nb * 4 + 2 * nv * 4 + ne * 4 + 16
        e2e_val = e2e_coinc / e2e_s
        if dist:
            t = torch.tensor([e2e_s / args.e2e_steps], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            c = torch.tensor([e2e_coinc], device=dev, dtype=torch.int64)
            dist.all_reduce(c, op=dist.ReduceOp.SUM)
            e2e_val = float(c.item()) / (float(t.item()) * args.e2e_steps)
        e2e = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps, "ms_per_step": 1e3 * e2e_s / args.e2e_steps, "api": "mcpet_run_async",
               "blocking_mcpet_run": {"value": rb["coincidences"] / blocking_s, "ms_per_step": 1e3 * blocking_s}}

    peak, peak_kind = load_peaks()
    achieved = b_alg / (avg_kernel_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "peak_kind": peak_kind,
            "kernel": "transport_kernel" if args.algorithm == "histories" else "transport_events_kernel",
            "kernel_ms": avg_kernel_ms, "algorithmic_bytes_per_launch": b_alg,
            "counters": counters}
    prof = os.path.join(ROOT, "profiles", "transport_traffic_head_1e9.md")
    if os.path.exists(prof):
        import re
        m = re.search(r"^dram_bytes_per_launch_full_workload:\s*(\d+)\s*$", open(prof).read(), re.M)
        if m:
            roof["traffic"] = int(m.group(1))

    gradient = None
    if rank == 0 and world == 1 and not args.no_gradient:
        gradient = measure_gradient(tmp)

    batch = None
    if args.batch_scenes > 0 and rank == 0 and world == 1:
        batch = measure_batch(args.batch_scenes, tmp, args.batch_emissions)

    beds = None
    if args.beds > 0 and rank == 0:
        scene.close()
        del tallies
        torch.cuda.empty_cache()
        beds = measure_beds(args.beds, tmp)

    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_ref_cuda and args.scanner == "head":
        ref_cuda = measure_reference_cuda(tmp, args.emissions)
        ref_cuda["this_library_kernel_ms"] = avg_kernel_ms
        ref_cuda["kernel_time_ratio"] = ref_cuda["kernel_ms"] / avg_kernel_ms

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = ReferenceCPU(write_workload_files(tmp, args.emissions), tmp)
        blocks = ref.sample(args.cpu_sample_decays)
        ref.run(ref.sample(args.cpu_sample_decays / 25))          # warm-up
        c, secs = ref.run(blocks)
        cpu = {"value": c / secs, "unit": UNIT, "cores": ref.cores, "kind": "reference",
               "sample": ref.describe(blocks, c, secs)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded head phantom; tissue densities on the reference's own air/water material tables)",
                "config": bench_config(args.emissions, world),
                "impl_config": {"lanes": args.lanes, "algorithm": args.algorithm,
                                "block_threads": args.block_threads or "auto",
                                "histories_per_lane": args.histories_per_lane or "auto"},
                "run": {"coincidences_per_step": total / args.steps / world, "histories_last_step": hist,
                        "guard_trips": guard},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps, "clocks": clocks}
        if ref_cuda is not None:
            line["ref_cuda"] = ref_cuda
        if gradient is not None:
            line["gradient"] = gradient
        if batch is not None:
            line["batch"] = batch
        if beds is not None:
            line["beds"] = beds
        print(json.dumps(line))
    scene.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
