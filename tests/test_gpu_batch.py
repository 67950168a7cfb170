"""Batched runs (mcpet_run_batch / mcpet_run_batch_device): several phantoms of
uneven size, each with its own activity, seed, acquisition time and isotope
mean life, in one launch of the transport kernel (large scenes in chained
launches of their own).  Every scene keeps its own
lane plan and RANECU streams, so its tallies must equal those of the same
scene run alone: compared bit for bit, in both lane layouts."""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
import scenes

HEAD_TISSUES = ("air", "soft", "grey", "white", "bone", "fat", "blood", "csf")
KEYS = ("trues", "scatter", "image_trues", "image_scatter", "spectrum")


def _batch_scenes(tmp):
    out = []
    mat, rho, act, vs, _ = inputs.head_phantom(shape=(16, 32, 32), voxel_cm=0.8, seed=7, total_bq=2.0e5)
    out.append(scenes.scene_from_arrays(str(tmp), mat, rho, act, vs, tissues=HEAD_TISSUES,
                                        **inputs.scanner_batch()))
    mat, rho, act, vs, _ = inputs.head_phantom(shape=(24, 40, 40), voxel_cm=0.6, seed=11, total_bq=3.0e5)
    out.append(scenes.scene_from_arrays(str(tmp), mat, rho, act, vs, tissues=HEAD_TISSUES, seed=777,
                                        acquisition_s=0.5, mean_life_s=0.3, **inputs.scanner_batch()))
    mat, rho, act, vs = inputs.water_cube_phantom(1.5e5)
    out.append(scenes.scene_from_arrays(str(tmp), mat, rho, act, vs, tissues=HEAD_TISSUES, seed=4242,
                                        **inputs.scanner_batch()))
    return out


def _same(a, b, tag):
    for k in KEYS:
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=f"{tag}: {k}")
    assert a.total_histories == b.total_histories, tag
    assert a.detected == b.detected, tag
    assert a.psf_count == b.psf_count, tag


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [mcpet.LANES_REFERENCE, mcpet.LANES_BALANCED])
def test_batch_equals_runs_one_by_one(tmp_path, lanes):
    sc = _batch_scenes(tmp_path)
    opts = mcpet.RunOptions(lane_mode=lanes, histories_per_lane=4)
    alone = [s.run(opts) for s in sc]
    assert all(r.detected > 50 for r in alone)
    batch = mcpet.Scene.run_batch(sc, opts)
    for k, (a, b) in enumerate(zip(alone, batch)):
        _same(a, b, f"scene {k}")
    # a second batched call on the same scenes gives the same result again
    again = mcpet.Scene.run_batch(sc, opts)
    for k, (a, b) in enumerate(zip(batch, again)):
        _same(a, b, f"repeat scene {k}")
    for s in sc:
        s.close()


def _with_large_scenes(tmp):
    """The small scenes plus two heads of 2.5e7 and 3e7 decays: enough decays
    and lanes for launches of their own."""
    out = _batch_scenes(tmp)
    for k, (bq, seed) in enumerate(((2.5e7, 99), (3.0e7, 98))):
        mat, rho, act, vs, _ = inputs.head_phantom(shape=(40, 64, 64), voxel_cm=0.4, seed=20 + k, total_bq=bq)
        out.insert(1 + k, scenes.scene_from_arrays(str(tmp), mat, rho, act, vs, tissues=HEAD_TISSUES, seed=seed,
                                                   **inputs.scanner_batch()))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [mcpet.LANES_REFERENCE, mcpet.LANES_BALANCED])
def test_batch_with_chained_launches_equals_runs_one_by_one(tmp_path, lanes):
    """The two large scenes run as launches of their own, chained on the
    stream ahead of the launch the small scenes share; with automatic lanes
    every scene gets its own, so each equals its run alone; counters are the
    totals of all launches."""
    import dataclasses
    sc = _with_large_scenes(tmp_path)
    opts = mcpet.RunOptions(lane_mode=lanes)
    alone = [s.run(opts) for s in sc]
    batch = mcpet.Scene.run_batch(sc, opts)
    for k, (a, b) in enumerate(zip(alone, batch)):
        _same(a, b, f"scene {k}")
    copts = dataclasses.replace(opts, collect_counters=True)
    counts = [s.run(copts).counters for s in sc]
    first = mcpet.Scene.run_batch(sc, copts)[0]
    for key in ("photons", "compton", "rayleigh", "photoelectric", "tally_increments", "lanes", "guard_trips"):
        assert first.counters[key] == sum(c[key] for c in counts), key
    assert first.counters["guard_trips"] == 0
    for s in sc:
        s.close()


@pytest.mark.gpu
def test_batch_of_one_and_counters(tmp_path):
    sc = _batch_scenes(tmp_path)[:1]
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, collect_counters=True)
    a = sc[0].run(opts)
    (b,) = mcpet.Scene.run_batch(sc, opts)
    _same(a, b, "single")
    assert a.counters == b.counters
    assert b.counters["guard_trips"] == 0
    sc[0].close()


@pytest.mark.gpu
def test_batch_device_entry_point(tmp_path):
    torch = pytest.importorskip("torch")
    import ctypes as C
    from mcpet import _abi
    sc = _batch_scenes(tmp_path)
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=4)
    alone = [s.run(opts) for s in sc]
    dev = torch.device("cuda:0")
    bufs, arr = [], (_abi.Tallies * len(sc))()
    for k, s in enumerate(sc):
        cfg, info = s.config, s.info
        b = {"trues": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
             "scatter": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
             "image_trues": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
             "image_scatter": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
             "spectrum": torch.zeros(cfg.n_energy_bins, dtype=torch.int32, device=dev),
             "psf_count": torch.zeros(1, dtype=torch.int32, device=dev),
             "histories": torch.zeros(1, dtype=torch.int64, device=dev),
             "coincidences": torch.zeros(1, dtype=torch.int64, device=dev)}
        bufs.append(b)
        t = arr[k]
        t.trues, t.scatter = b["trues"].data_ptr(), b["scatter"].data_ptr()
        t.image_trues, t.image_scatter = b["image_trues"].data_ptr(), b["image_scatter"].data_ptr()
        t.spectrum = b["spectrum"].data_ptr()
        t.psf_count = b["psf_count"].data_ptr()
        t.total_histories = b["histories"].data_ptr()
        t.coincidences = b["coincidences"].data_ptr()
    ptrs = (C.c_void_p * len(sc))(*[s.handle for s in sc])
    co = opts.to_c()
    _abi.check(_abi.lib().mcpet_run_batch_device(ptrs, len(sc), C.byref(co), arr))
    torch.cuda.synchronize()
    for k, (a, b) in enumerate(zip(alone, bufs)):
        np.testing.assert_array_equal(b["trues"].cpu().numpy(), a.trues, err_msg=f"scene {k}")
        np.testing.assert_array_equal(b["scatter"].cpu().numpy(), a.scatter, err_msg=f"scene {k}")
        np.testing.assert_array_equal(b["image_trues"].cpu().numpy(), a.image_trues, err_msg=f"scene {k}")
        np.testing.assert_array_equal(b["spectrum"].cpu().numpy(), a.spectrum, err_msg=f"scene {k}")
        assert int(b["histories"].item()) == a.total_histories
        assert int(b["coincidences"].item()) == a.detected
    for s in sc:
        s.close()


def test_batch_rejects_invalid(tmp_path):
    """Host-side checks, no device needed: empty batch, tables that differ
    between scenes, the history-loop algorithm."""
    import ctypes as C
    from mcpet import _abi
    head = _batch_scenes(tmp_path)[0]
    # water in slot 1 and air in slot 2: the heads have air in slot 1
    mat, rho, act, vs = inputs.water_cube_phantom(1.0e4)
    spec = inputs.spec_for([inputs.material_path("water"), inputs.material_path("air")], "unused.vox",
                           **inputs.scanner_small())
    other = mcpet.Scene.from_arrays(inputs.config_from_spec(spec, str(tmp_path)), mat, rho, act, vs)
    with pytest.raises(mcpet.McpetError) as e:
        mcpet.Scene.run_batch([], mcpet.RunOptions())
    assert e.value.status == 1
    with pytest.raises(mcpet.McpetError) as e:
        mcpet.Scene.run_batch([head, other], mcpet.RunOptions())
    msg = str(e.value)
    assert e.value.status == 1 and ("material slot 1" in msg or "energy grid" in msg), msg
    with pytest.raises(mcpet.McpetError) as e:
        mcpet.Scene.run_batch([head], mcpet.RunOptions(algorithm=mcpet.ALGORITHM_HISTORIES))
    assert e.value.status == 1 and "event loop" in str(e.value)
    t = (_abi.Tallies * 1)()
    ptrs = (C.c_void_p * 1)(head.handle)
    with pytest.raises(mcpet.McpetError):
        _abi.check(_abi.lib().mcpet_run_batch_device(ptrs, 0, None, t))
    head.close()
    other.close()


needs_ref_prog = pytest.mark.needs_ref("libref_prog.so")


@needs_ref_prog
@pytest.mark.gpu
def test_batched_many_phantom_workload_replays_reference_runs(tmp_path, capsys):
    """The first four phantoms of the many-phantom workload (uneven cubes at
    2-4 mm, 1e8 decays each, 32-ring scanner), batched with the reference's
    lane layout, replay the reference's CUDA runs of the same input files one
    phantom at a time (its only way to run them)."""
    import refbind
    from test_gpu_transport import assert_replay
    ins = []
    for k, (mat, rho, act, vs, used) in enumerate(inputs.batch_phantoms(4, 1.0e8)):
        ins.append(scenes.write_case(str(tmp_path), f"many{k}", mat, rho, act, vs, tissues=HEAD_TISSUES,
                                     seed=1000 + k, **inputs.scanner_batch()))
    sc = [mcpet.Scene.load(p) for p in ins]
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE)
    batch = mcpet.Scene.run_batch(sc, opts)
    ref_ms = []
    for k, (p, s, r) in enumerate(zip(ins, sc, batch)):
        cfg, info = s.config, s.info
        ref = refbind.RefProg().run(p, int(cfg.n_bins), int(info.n_voxels), cfg.n_energy_bins, cwd=str(tmp_path))
        assert_replay(cfg, r, ref)
        ref_ms.append(ref["kernel_ms"])
    with capsys.disabled():
        print(f"\nreference kernels {[round(x, 1) for x in ref_ms]} ms (sum {sum(ref_ms):.1f}); batched "
              f"{batch[0].transport_ms:.1f} ms; coincidences {[r.detected for r in batch]}")
    for s in sc:
        s.close()
