"""The host lane plan (mcpet_scene_lane_plan, no device): built on several
host threads and merged, it must be exactly the plan of one stable sort of
the emitting voxels by lanes/activity (the launch order: longest lanes
first, ties in voxel order), in both lane layouts."""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
import scenes


def _scene(workdir, seed=4):
    rng = np.random.default_rng(seed)
    n = 64
    mat = np.full((n, n, n), 2, np.int32)
    rho = np.ones((n, n, n), np.float32)
    act = rng.choice(np.array([0.0, 5.0, 50.0, 120.0, 3000.0, 7e4], np.float32), size=(n, n, n),
                     p=[0.4, 0.2, 0.2, 0.1, 0.09, 0.01])          # many ties
    return scenes.scene_from_arrays(workdir, mat, rho, act, (0.5, 0.5, 0.5), tissues=("air", "soft")), act


@pytest.mark.parametrize("hpl", [7, 100, 4096])
def test_balanced_plan_is_one_stable_sort(workdir, hpl):
    sc, act = _scene(workdir)
    p = sc.lane_plan(mcpet.LANES_BALANCED, hpl)
    a = act.ravel()
    emit = np.flatnonzero(a > np.float32(1e-7))
    T = sc.config.acquisition_time_ps * 1e-12
    L = np.clip(np.ceil(a[emit].astype(np.float64) * T / hpl), 1, 1e8)
    rate = L / a[emit].astype(np.float64)
    order = np.argsort(rate, kind="stable")
    np.testing.assert_array_equal(p["voxel"], emit[order].astype(np.uint32))
    np.testing.assert_array_equal(p["n_lanes"], L[order].astype(np.uint32))
    np.testing.assert_array_equal(p["inv_rate"], rate[order])
    first = np.concatenate([[0], np.cumsum(L[order])[:-1]]).astype(np.uint64)
    np.testing.assert_array_equal(p["first_lane"], first)
    np.testing.assert_array_equal(p["stream_base"], first)
    assert p["total_lanes"] == int(L.sum())
    sc.close()


def test_reference_plan_keeps_the_reference_streams(workdir):
    sc, act = _scene(workdir, seed=5)
    tpb = sc.config.threads_per_block
    p = sc.lane_plan(mcpet.LANES_REFERENCE)
    a = act.ravel()
    emit = np.flatnonzero(a > np.float32(1e-7))
    rate = tpb / a[emit].astype(np.float64)
    order = np.argsort(rate, kind="stable")
    np.testing.assert_array_equal(p["voxel"], emit[order].astype(np.uint32))
    assert np.all(p["n_lanes"] == tpb)
    np.testing.assert_array_equal(p["stream_base"], emit[order].astype(np.uint64) * tpb)
    np.testing.assert_array_equal(p["first_lane"], np.arange(len(emit), dtype=np.uint64) * tpb)
    sc.close()


def test_plan_capacity_and_errors(workdir):
    import ctypes as C
    from mcpet import _abi
    sc, act = _scene(workdir)
    n, tot = C.c_longlong(0), C.c_ulonglong(0)
    st = _abi.lib().mcpet_scene_lane_plan(sc.handle, 1, 10, 5, None, None, None, None, None, C.byref(n), C.byref(tot))
    assert st == 6 and n.value == int((act > 0).sum()) and tot.value > 0
    with pytest.raises(mcpet.McpetError):
        _abi.check(_abi.lib().mcpet_scene_lane_plan(sc.handle, 7, 10, 0, None, None, None, None, None, C.byref(n),
                                                    None))
    sc.close()
