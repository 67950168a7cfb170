"""Transport on the GPU through the C ABI.

* replay parity with the reference's own CUDA run (libref_prog.so, same GPU,
  same seed): histories, coincidences and >= 99.9% of detected events in the
  same sinogram bins and PSF records;
* statistical parity with the C oracle (independent seeds): chi^2/dof of the
  sinograms in [0.9, 1.1] and totals within 3 sigma;
* invariants and the device-buffer entry point.
"""
import math
import os

import numpy as np
import pytest

import mcpet
from mcpet import inputs
from oracle import pyoracle
import refbind
import scenes

pytestmark = pytest.mark.gpu
needs_ref_prog = pytest.mark.needs_ref("libref_prog.so")


def overlap(a: np.ndarray, b: np.ndarray) -> float:
    """Fraction of counts that sit in the same bins of two histograms."""
    tot = max(int(a.sum(dtype=np.int64)), int(b.sum(dtype=np.int64)), 1)
    return float(np.minimum(a, b).sum(dtype=np.int64)) / tot


def coarse(sino: np.ndarray, cfg, f=(1, 8, 8)) -> np.ndarray:
    s = sino.reshape(cfg.n_sinograms, cfg.n_angles, cfg.n_radial).astype(np.int64)
    pads = [(0, (-n) % k) for n, k in zip(s.shape, f)]
    s = np.pad(s, pads)
    a, b, c = (n // k for n, k in zip(s.shape, f))
    return s.reshape(a, f[0], b, f[1], c, f[2]).sum(axis=(1, 3, 5))


def replay(in_path: str, workdir: str, opts=None, background=False, psf_capacity=0):
    with mcpet.Scene.load(in_path) as sc:
        cfg, info = sc.config, sc.info
        mine = sc.run(opts or mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, background_mode=background),
                      psf_capacity=psf_capacity or None)
        assert sc.guard_trips() == 0
    ref = refbind.RefProg().run(in_path, int(cfg.n_bins), int(info.n_voxels), cfg.n_energy_bins,
                                background=background, psf_capacity=psf_capacity, cwd=workdir)
    return cfg, mine, ref


def assert_replay(cfg, mine, ref, min_overlap=0.999):
    assert mine.total_histories == ref["total_histories"] or \
        abs(mine.total_histories - ref["total_histories"]) <= 1e-4 * ref["total_histories"]
    n_ref = int(ref["trues"].sum() + ref["scatter"].sum())
    assert n_ref > 0
    assert abs(mine.coincidences - n_ref) <= max(2, 1e-3 * n_ref)
    for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
        a, b = getattr(mine, k), ref[k]
        if b.sum() > 50:
            assert overlap(a, b) >= min_overlap, (k, overlap(a, b))


@needs_ref_prog
def test_replay_sample_with_psf(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, "rp_sample", mat, rho, act, vs, tally_psf_sinogram=0, psf_size=200000,
                            seed=12345)
    cfg, mine, ref = replay(inp, workdir, psf_capacity=200000)
    assert_replay(cfg, mine, ref)
    np.testing.assert_array_equal(mine.trues, ref["trues"])
    a = scenes.psf_records(mine.psf)
    b = scenes.psf_records(ref["psf_raw"])
    assert len(a) == len(b) == mine.psf_count == ref["psf_count"]
    # discrete fields and the blurred energy identical; positions/directions/
    # times equal to FP32 rounding (a few ulp)
    for f in ("emission_time_ps", "emission_absvox", "index1", "index2", "energy"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)
    for f in ("travel_time_ps", "z", "phi", "vx", "vy", "vz"):
        np.testing.assert_allclose(a[f], b[f], rtol=2e-6, atol=2e-6, err_msg=f)


@needs_ref_prog
@pytest.mark.parametrize("algorithm", [mcpet.ALGORITHM_EVENTS, mcpet.ALGORITHM_HISTORIES])
def test_replay_head_both_algorithms(workdir, algorithm):
    mat, rho, act, vs, used = inputs.head_phantom(shape=(32, 64, 64), voxel_cm=0.4, seed=11, total_bq=1e6)
    inp = scenes.write_case(workdir, f"rp_alg{algorithm}", mat, rho, act, vs, tissues=used, seed=777,
                            **inputs.scanner_for_head())
    cfg, mine, ref = replay(inp, workdir, opts=mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE,
                                                                 algorithm=algorithm))
    assert_replay(cfg, mine, ref)


def test_algorithms_agree(workdir):
    """Same lanes and streams, two schedules: identical integer tallies."""
    sc = scenes.small_head_scene(workdir, total_bq=5.0e5, shape=(24, 48, 48), voxel_cm=0.5, tally_psf_sinogram=0,
                                 psf_size=300000)
    a = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, algorithm=mcpet.ALGORITHM_EVENTS))
    b = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, algorithm=mcpet.ALGORITHM_HISTORIES))
    assert a.total_histories == b.total_histories
    for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
        assert overlap(getattr(a, k), getattr(b, k)) >= 0.9999, k
    sc.close()


@needs_ref_prog
@pytest.mark.parametrize("case", ["water_cube", "background", "trues_only", "head_tissues", "span11"])
def test_replay_matches_reference_cuda_run(workdir, case):
    if case == "head_tissues":
        mat, rho, act, vs, used = inputs.head_phantom(shape=(24, 48, 48), voxel_cm=0.5, seed=3, total_bq=4e5)
        inp = scenes.write_case(workdir, f"rp_{case}", mat, rho, act, vs, tissues=used, seed=2024,
                                **inputs.scanner_for_head())
        cfg, mine, ref = replay(inp, workdir)
    else:
        mat, rho, act, vs = inputs.water_cube_phantom(1.0e6 if case == "water_cube" else 3.0e5)
        kw = dict(seed=31337)
        if case == "trues_only":
            kw["tally_type"] = 1
        if case == "span11":
            kw.update(fov_z=12.656, n_rows=80, n_z_slices=159, max_ring_difference=79, span=11,
                      detector_radius=-9.05, detector_height=12.656)
        inp = scenes.write_case(workdir, f"rp_{case}", mat, rho, act, vs, **kw)
        cfg, mine, ref = replay(inp, workdir, background=(case == "background"))
    assert_replay(cfg, mine, ref)
    if case == "trues_only":
        assert mine.scatter.sum() == 0


def _oracle_pair(sc, seed_gpu, seed_cpu, lane_mode):
    res = sc.run(mcpet.RunOptions(lane_mode=lane_mode, seed_override=seed_gpu))
    ref = pyoracle.OracleScene(sc, seed=seed_cpu).run(n_threads=0)
    return res, ref


@pytest.mark.parametrize("lane_mode", [mcpet.LANES_REFERENCE, mcpet.LANES_BALANCED])
def test_statistics_vs_oracle_water_cube(workdir, lane_mode):
    sc = scenes.water_cube_scene(workdir, 1.0e6)
    res, ref = _oracle_pair(sc, 1001, 2002, lane_mode)
    cfg = sc.config
    for k in ("trues", "scatter"):
        a, b = int(getattr(res, k).sum()), int(ref[k].sum())
        assert abs(a - b) <= 3 * math.sqrt(a + b) + 1, (k, a, b)
    chi, dof = scenes.chi2_per_dof(coarse(res.trues + res.scatter, cfg), coarse(ref["trues"] + ref["scatter"], cfg),
                                   min_count=20)
    assert dof > 1500 and 0.9 <= chi <= 1.1, (chi, dof)
    chi, dof = scenes.chi2_per_dof(res.image_trues, ref["image_trues"], min_count=20)
    assert 0.8 <= chi <= 1.2, (chi, dof)
    chi, dof = scenes.chi2_per_dof(res.spectrum, ref["spectrum"], min_count=20)
    assert 0.7 <= chi <= 1.3, (chi, dof)
    sc.close()


def test_statistics_vs_oracle_head(workdir):
    sc = scenes.small_head_scene(workdir, total_bq=2.0e6, shape=(24, 48, 48), voxel_cm=0.5)
    res, ref = _oracle_pair(sc, 77, 78, mcpet.LANES_BALANCED)
    cfg = sc.config
    for k in ("trues", "scatter"):
        a, b = int(getattr(res, k).sum()), int(ref[k].sum())
        assert abs(a - b) <= 3 * math.sqrt(a + b) + 1, (k, a, b)
    # 8065 x 256 x 256 sinogram -> 8 x 16 x 32 coarse bins
    f = (1009, 16, 8)
    chi, dof = scenes.chi2_per_dof(coarse(res.trues + res.scatter, cfg, f), coarse(ref["trues"] + ref["scatter"],
                                                                                   cfg, f), min_count=20)
    assert dof > 800 and 0.9 <= chi <= 1.1, (chi, dof)
    chi, dof = scenes.chi2_per_dof(res.image_trues + res.image_scatter, ref["image_trues"] + ref["image_scatter"],
                                   min_count=20)
    assert dof > 200 and 0.8 <= chi <= 1.2, (chi, dof)
    sc.close()


def test_invariants_and_determinism(workdir):
    sc = scenes.small_head_scene(workdir, total_bq=3.0e5, shape=(24, 48, 48), voxel_cm=0.5, tally_psf_sinogram=0,
                                 psf_size=400000)
    o = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, collect_counters=True)
    a = sc.run(o)
    b = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
    for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    assert a.total_histories == b.total_histories and a.total_histories % 2 == 0
    assert int(a.image_trues.sum()) == int(a.trues.sum())
    assert int(a.image_scatter.sum()) == int(a.scatter.sum())
    assert int(a.spectrum.sum()) >= 2 * a.coincidences
    assert a.counters["photons"] == a.total_histories
    assert a.counters["guard_trips"] == 0
    assert a.psf_count > 0 and len(a.psf) == min(a.psf_count, 400000)
    # the same kernel twice: identical PSF record sets (the counting variant of
    # run a is a different compilation, so only its integer tallies are compared)
    c = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
    assert {r.tobytes() for r in scenes.psf_records(b.psf)} == {r.tobytes() for r in scenes.psf_records(c.psf)}
    np.testing.assert_array_equal(b.psf["emission_time_ps"].sort(), c.psf["emission_time_ps"].sort())
    sc.close()


def test_device_entry_point_matches_host_entry_point(workdir):
    torch = pytest.importorskip("torch")
    sc = scenes.water_cube_scene(workdir, 2.0e5)
    cfg, info = sc.config, sc.info
    dev = torch.device("cuda:0")
    t = {
        "trues": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
        "scatter": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
        "image_trues": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
        "image_scatter": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
        "spectrum": torch.zeros(cfg.n_energy_bins, dtype=torch.int32, device=dev),
        "psf_count": torch.zeros(1, dtype=torch.int32, device=dev),
        "histories": torch.zeros(1, dtype=torch.int64, device=dev),
    }
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, stream=torch.cuda.current_stream().cuda_stream)
    ms = sc.run_device(t, opts, time_it=True)
    torch.cuda.synchronize()
    host = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
    assert ms > 0
    assert int(t["histories"].item()) == host.total_histories
    np.testing.assert_array_equal(t["trues"].cpu().numpy(), host.trues)
    np.testing.assert_array_equal(t["scatter"].cpu().numpy(), host.scatter)
    np.testing.assert_array_equal(t["spectrum"].cpu().numpy(), host.spectrum)
    sc.close()


def test_outputs_written_in_reference_formats(workdir):
    import gzip
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, "out_fmt", mat, rho, act, vs, tally_psf_sinogram=0, psf_size=50000)
    out_dir = os.path.join(workdir, "outputs")
    os.makedirs(out_dir, exist_ok=True)
    with mcpet.Scene.load(inp) as sc:
        r = sc.run()
        sc.write_outputs(r, out_dir)
        cfg = sc.config
    with gzip.open(os.path.join(out_dir, "sinogram_Trues.raw.gz")) as f:
        np.testing.assert_array_equal(np.frombuffer(f.read(), np.int32), r.trues)
    with gzip.open(os.path.join(out_dir, "image_Scatter.raw.gz")) as f:
        np.testing.assert_array_equal(np.frombuffer(f.read(), np.int32), r.image_scatter)
    spec = np.loadtxt(os.path.join(out_dir, "Energy_Sinogram_Spectrum.dat"), dtype=np.int64)
    np.testing.assert_array_equal(spec[:, 1], r.spectrum)
    raw = np.fromfile(os.path.join(out_dir, cfg.psf_file.decode() + ".raw"), dtype=mcpet.PSF_DTYPE)
    assert len(raw) == min(r.psf_count, 50000)
    assert open(os.path.join(out_dir, cfg.psf_file.decode())).read().count("\n") > min(r.psf_count, 5000)


def test_async_runs_equal_blocking_runs(workdir):
    """mcpet_run_async: three runs in flight on one stream with the activity
    changed between them (the plan upload is ordered after the run still
    reading the old plan) give the blocking runs' results."""
    torch = pytest.importorskip("torch")
    mat, rho, act, vs, used = inputs.head_phantom(shape=(24, 48, 48), voxel_cm=0.5, seed=3, total_bq=4e5)
    inp = scenes.write_case(workdir, "async", mat, rho, act, vs, tissues=used, seed=2024,
                            **inputs.scanner_batch())
    act2 = (act * np.linspace(0.5, 1.5, act.size, dtype=np.float32).reshape(act.shape)).astype(np.float32)
    plan = [(act, 11), (act2, 12), (act, 13)]
    with mcpet.Scene.load(inp) as sc:
        cfg, info = sc.config, sc.info
        want = []
        for a, seed in plan:
            sc.set_activity(a)
            want.append(sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, seed_override=seed)))
        bufs, res = [], []
        for a, seed in plan:
            b = {k: torch.zeros(n, dtype=torch.int32).pin_memory() for k, n in
                 (("trues", int(cfg.n_bins)), ("scatter", int(cfg.n_bins)), ("image_trues", int(info.n_voxels)),
                  ("image_scatter", int(info.n_voxels)), ("spectrum", cfg.n_energy_bins))}
            sc.set_activity(a)
            res.append(sc.run_async(b, mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, seed_override=seed)))
            bufs.append(b)
        # other runs share the scene's run words: refused until wait()
        with pytest.raises(mcpet.McpetError) as e:
            sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
        assert e.value.status == 1 and "mcpet_run_wait" in str(e.value)
        sc.wait()
        for k, (w, b, r) in enumerate(zip(want, bufs, res)):
            for key in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
                np.testing.assert_array_equal(b[key].numpy(), getattr(w, key), err_msg=f"run {k}: {key}")
            assert r["coincidences"].value == w.detected and r["total_histories"].value == w.total_histories
        assert want[0].detected != want[1].detected
