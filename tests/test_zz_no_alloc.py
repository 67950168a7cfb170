"""Allocation-free transport entry point, mcpet_run_device_noalloc.

Some callers may not allocate device memory while they run: plugin and
custom-call hooks inside a host framework get every device buffer from that
framework's pool, and multi-stream pipelines cannot take the device-wide
synchronisation that cudaMalloc/cudaFree imply.  For them the library keeps
the lane plan and the work-queue words of a run in a fixed static device
array instead of buffers it allocates.  These tests call the entry point
through the C ABI, twice in a row, and check it against mcpet_run_device on
the same scene, activity map and seed.  With the reference lane layout the
two entry points run the same lanes on the same random streams, so the integer
tallies must be identical.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import mcpet
from mcpet import _abi, inputs
import scenes

pytestmark = pytest.mark.gpu


def _alloc(torch, cfg, info):
    dev = torch.device("cuda:0")
    return {
        "trues": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
        "scatter": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
        "image_trues": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
        "image_scatter": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
        "spectrum": torch.zeros(cfg.n_energy_bins, dtype=torch.int32, device=dev),
        "psf_count": torch.zeros(1, dtype=torch.int32, device=dev),
        "histories": torch.zeros(1, dtype=torch.int64, device=dev),
        "coincidences": torch.zeros(1, dtype=torch.int64, device=dev),
        "counters": torch.zeros(10, dtype=torch.int64, device=dev),
    }


def _run_noalloc(scene, activity, tallies, opts):
    t = _abi.Tallies()
    t.trues, t.scatter = tallies["trues"].data_ptr(), tallies["scatter"].data_ptr()
    t.image_trues, t.image_scatter = tallies["image_trues"].data_ptr(), tallies["image_scatter"].data_ptr()
    t.spectrum = tallies["spectrum"].data_ptr()
    t.psf_count = tallies["psf_count"].data_ptr()
    t.total_histories = tallies["histories"].data_ptr()
    t.coincidences = tallies["coincidences"].data_ptr()
    t.counters = tallies["counters"].data_ptr()
    co = opts.to_c()
    _abi.check(_abi.lib().mcpet_run_device_noalloc(scene.handle, C.c_void_p(activity.data_ptr()), C.byref(co),
                                                    C.byref(t)))


def _host(t):
    return {k: v.cpu().numpy() for k, v in t.items()}


def test_noalloc_matches_device_entry_point(tmp_path):
    torch = pytest.importorskip("torch")
    sc = scenes.small_head_scene(str(tmp_path), total_bq=4.0e5, shape=(24, 48, 48), voxel_cm=0.5)
    sc.to_device(0)
    cfg, info = sc.config, sc.info
    activity = torch.from_numpy(np.ascontiguousarray(sc.export_tables()["voxels"][:, 2])).cuda()
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, collect_counters=True)

    ref = _alloc(torch, cfg, info)
    sc.run_device(ref, opts)
    torch.cuda.synchronize()
    ref = _host(ref)
    assert ref["coincidences"][0] > 100

    for call in range(2):
        out = _alloc(torch, cfg, info)
        _run_noalloc(sc, activity, out, opts)
        torch.cuda.synchronize()
        got = _host(out)
        for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum", "histories", "coincidences",
                  "psf_count"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"call {call}: {k}")
        # counters: same work, and no guard trips
        np.testing.assert_array_equal(got["counters"], ref["counters"], err_msg=f"call {call}: counters")
        assert got["counters"][9] == 0
    # the second call (after the first one warmed up the module) allocated nothing
    out = _alloc(torch, cfg, info)
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    _run_noalloc(sc, activity, out, opts)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == before
    sc.close()


def test_noalloc_balanced_lanes_repeatable(tmp_path):
    torch = pytest.importorskip("torch")
    sc = scenes.water_cube_scene(str(tmp_path), 1.0e6)
    sc.to_device(0)
    cfg, info = sc.config, sc.info
    activity = torch.from_numpy(np.ascontiguousarray(sc.export_tables()["voxels"][:, 2])).cuda()
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=8)
    runs = []
    for _ in range(2):
        out = _alloc(torch, cfg, info)
        _run_noalloc(sc, activity, out, opts)
        torch.cuda.synchronize()
        runs.append(_host(out))
    for k in ("trues", "scatter", "spectrum", "histories", "coincidences"):
        np.testing.assert_array_equal(runs[0][k], runs[1][k], err_msg=k)
    host = sc.run(opts)
    a, b = int(runs[0]["coincidences"][0]), host.coincidences
    assert abs(a - b) <= 5 * np.sqrt(a + b), (a, b)
    assert int(runs[0]["trues"].sum() + runs[0]["scatter"].sum()) == a
    sc.close()


def _ball_phantom(levels):
    """16x32x32 voxels of 5 mm: a water ball in air whose voxels cycle
    through the activity levels (Bq) in voxel order."""
    nz, ny, nx = 16, 32, 32
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    inside = ((x - 15.5) / 13) ** 2 + ((y - 15.5) / 13) ** 2 + ((z - 7.5) / 7) ** 2 <= 1.0
    mat = np.where(inside, 2, 1).astype(np.int32)
    rho = np.where(inside, 1.0, 0.0012).astype(np.float32)
    lv = np.asarray(levels, np.float32)
    act = np.zeros(inside.shape, np.float32)
    act[inside] = lv[np.arange(int(inside.sum())) % len(lv)]
    return mat, rho, act, (0.5, 0.5, 0.5)


@pytest.mark.parametrize("case", ["proportional_lanes", "automatic_lanes"])
def test_noalloc_balanced_plan_equals_host_plan(tmp_path, case):
    """Balanced lanes pinned exactly.  The device builds its plan in voxel
    order, the host sorts emitters by decreasing decays per lane with ties
    in voxel order.  When every emitter has the same lanes/activity the two
    orders coincide, so the two entry points must run identical lanes
    (first lane, stream, rate of every emitter) and give identical integer
    tallies: activities 1000/2000/3000 Bq with 100 decays per lane give
    10/20/30 lanes per voxel; a uniform 1000 Bq map with the automatic lane
    size also checks the size computed on the device from the activity
    map against the host's."""
    torch = pytest.importorskip("torch")
    levels, hpl = ((1000.0, 2000.0, 3000.0), 100) if case == "proportional_lanes" else ((1000.0,), 0)
    mat, rho, act, vs = _ball_phantom(levels)
    sc = scenes.scene_from_arrays(str(tmp_path), mat, rho, act, vs)
    sc.to_device(0)
    cfg, info = sc.config, sc.info
    plan = sc.lane_plan(mcpet.LANES_BALANCED, hpl)
    np.testing.assert_array_equal(plan["voxel"], np.sort(plan["voxel"]))   # host order is voxel order here
    activity = torch.from_numpy(np.ascontiguousarray(act.ravel())).cuda()
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=hpl, collect_counters=True)
    ref = _alloc(torch, cfg, info)
    sc.run_device(ref, opts)
    torch.cuda.synchronize()
    ref = _host(ref)
    assert ref["coincidences"][0] > 1000
    assert int(ref["counters"][8]) == int(plan["total_lanes"])
    for call in range(2):
        out = _alloc(torch, cfg, info)
        _run_noalloc(sc, activity, out, opts)
        torch.cuda.synchronize()
        got = _host(out)
        for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum", "histories", "coincidences",
                  "counters"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"call {call}: {k}")
    sc.close()


def test_noalloc_stream_limit_trip_reaches_the_caller(tmp_path):
    """A plan that would need RANECU stream ids >= 2^31 runs nothing, and
    says so: counters[9] and mcpet_last_run_guard report the trip.  A
    following call within the limit is clean again."""
    torch = pytest.importorskip("torch")
    mat, rho, _, vs = inputs.water_cube_phantom(1.0)
    act = np.full(mat.shape, 3.0e6, np.float32)   # 2.19e9 decays: one lane per decay needs more than 2^31 streams
    sc = scenes.scene_from_arrays(str(tmp_path), mat, rho, act, vs)
    sc.to_device(0)
    cfg, info = sc.config, sc.info
    activity = torch.from_numpy(np.ascontiguousarray(act.ravel())).cuda()
    out = _alloc(torch, cfg, info)
    _run_noalloc(sc, activity, out, mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=1,
                                                     collect_counters=True))
    torch.cuda.synchronize()
    got = _host(out)
    assert got["counters"][9] == 1 and got["histories"][0] == 0 and got["trues"].sum() == 0
    assert sc.guard_trips() == 1
    out = _alloc(torch, cfg, info)
    activity /= 1000.0
    _run_noalloc(sc, activity, out, mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=100))
    torch.cuda.synchronize()
    assert sc.guard_trips() == 0 and int(out["histories"].item()) > 0
    sc.close()


def test_noalloc_reference_lanes_stream_limit(tmp_path):
    """Reference lanes use stream voxel * threads_per_block + thread: with
    2048 threads per block an emitting voxel at index 2^20 - 1 needs stream
    ids up to 2^31 - 1 + 2048, beyond the reference's 31-bit thread ids.  The
    host entry point refuses the plan, the allocation-free one counts a trip."""
    torch = pytest.importorskip("torch")
    shape = (256, 64, 64)                      # 2^20 voxels
    mat = np.full(shape, 2, np.int32)
    rho = np.ones(shape, np.float32)
    act = np.zeros(shape, np.float32)
    act[-1, -1, -1] = 10.0
    sc = scenes.scene_from_arrays(str(tmp_path), mat, rho, act, (0.5, 0.5, 0.5), threads_per_block=2048)
    sc.to_device(0)
    cfg, info = sc.config, sc.info
    out = _alloc(torch, cfg, info)
    with pytest.raises(mcpet.McpetError) as e:
        sc.run_device(out, mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE))
    assert e.value.status == 6
    activity = torch.from_numpy(np.ascontiguousarray(act.ravel())).cuda()
    _run_noalloc(sc, activity, out, mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, collect_counters=True))
    torch.cuda.synchronize()
    assert int(out["counters"][9].item()) == 1 and int(out["histories"].item()) == 0
    assert sc.guard_trips() == 1
    sc.close()


def test_noalloc_rejects_oversized_phantom(tmp_path):
    nz = (1 << 20) // (64 * 64) + 1
    mat = np.full((nz, 64, 64), 2, np.int32)
    rho = np.ones((nz, 64, 64), np.float32)
    act = np.zeros((nz, 64, 64), np.float32)
    act[0, 0, 0] = 1.0
    sc = scenes.scene_from_arrays(str(tmp_path), mat, rho, act, (0.5, 0.5, 0.5))
    with pytest.raises(mcpet.McpetError) as e:
        t = _abi.Tallies()
        _abi.check(_abi.lib().mcpet_run_device_noalloc(sc.handle, C.c_void_p(1), C.byref(mcpet.RunOptions().to_c()),
                                                        C.byref(t)))
    assert e.value.status == 6 and "at most" in str(e.value)
    sc.close()
