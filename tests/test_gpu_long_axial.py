"""Long-axial scanner (256 rings x 0.4 cm, 768 crystals, 384 x 384 bins, span
11; at MRD 255: 12333 sinogram planes, 1.82e9 bins, 7.3 GB per int32
sinogram).  The reference cannot run the full size: its byte counts NBINS*4
are 32-bit ints (MCGPU-PET.cu:294-295).  Here the sizes are 64-bit:

* the detector model bins events spread over the 102 cm axial FOV exactly as
  the oracle's restatement does, including bins above 1.5e9;
* a full transport run allocates, zeroes, fills and downloads both 7.3 GB
  sinograms, with counts in the top segments and no guard trips;
* at MRD 38 (3373 planes, 5.0e8 bins: within the reference's 32-bit sizes)
  a body phantom with lungs and bone replays the reference's CUDA run;
* bed positions (detector centres stepped along the body axis, one scene
  each) batched in one launch equal the beds run one by one.
"""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
from oracle import pyoracle
import refbind
import scenes
from test_gpu_transport import assert_replay, replay

needs_ref_prog = pytest.mark.needs_ref("libref_prog.so")

pytestmark = pytest.mark.gpu
LONG_AXIAL = dict(detector_radius=-39.0, detector_height=102.4, fov_z=102.4, n_rows=256, n_crystals=768,
                  n_angles=384, n_radial=384, n_z_slices=511, max_ring_difference=255, span=11)


def _long_phantom(total_bq):
    nz, n = 250, 10
    mat = np.full((nz, n, n), 2, np.int32)
    rho = np.ones((nz, n, n), np.float32)
    act = np.full((nz, n, n), total_bq / (nz * n * n), np.float32)
    return mat, rho, act, (0.4, 0.4, 0.4)


def test_long_axial_detector_bins_match_oracle(tmp_path):
    mat, rho, act, vs = _long_phantom(1.0e3)
    sc = scenes.scene_from_arrays(str(tmp_path), mat, rho, act, vs, **LONG_AXIAL)
    assert sc.config.n_sinograms == 12333 and sc.config.n_bins == 12333 * 384 * 384
    rng = np.random.default_rng(23)
    ev = scenes.random_events(200000, rng, box=(4.0, 4.0, 100.0))
    got = mcpet.probe_detector(sc, ev)
    want = pyoracle.detector(pyoracle.OracleScene(sc), ev)
    # integer bins exact except for events within float rounding of a bin edge
    # (CPU libm vs GPU intrinsics), as for the small scanners
    same = np.all(got[:, :4] == want[:, :4], axis=1)
    assert same.mean() >= 0.999, (~same).sum()
    assert got[:, 0].max() > 1_500_000_000
    sc.close()


def test_long_axial_full_transport(tmp_path):
    mat, rho, act, vs = _long_phantom(1.0e6)
    sc = scenes.scene_from_arrays(str(tmp_path), mat, rho, act, vs, **LONG_AXIAL)
    r = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
    assert sc.guard_trips() == 0
    assert r.detected > 1000
    assert int(r.trues.sum(dtype=np.int64) + r.scatter.sum(dtype=np.int64)) == r.detected
    nz_t = np.flatnonzero(r.trues)
    assert nz_t.max() > 1_000_000_000
    sc.close()


@needs_ref_prog
def test_long_axial_body_replays_reference_cuda_run(workdir):
    mat, rho, act, vs, used = inputs.body_phantom(shape=(50, 32, 32), voxel_cm=1.6, seed=5, total_bq=4.0e5)
    inp = scenes.write_case(workdir, "rp_long_axial", mat, rho, act, vs, tissues=used, seed=777,
                            **inputs.scanner_long_axial(max_ring_difference=38))
    cfg, mine, ref = replay(inp, workdir)
    assert cfg.n_sinograms == 3373 and cfg.n_bins < 2**31 // 4
    assert_replay(cfg, mine, ref)


def test_bed_positions_batched_equal_beds_one_by_one(tmp_path):
    mat, rho, act, vs, used = inputs.body_phantom(shape=(100, 64, 64), voxel_cm=0.8, seed=9, total_bq=2.0e6)
    size = (64 * 0.8, 64 * 0.8, 100 * 0.8)
    # the long-axial rings with a coarser crystal ring (192 crystals, 96 x 96
    # bins: the sinogram wants n_crystals / 2 angles) to keep four beds small
    scan = inputs.scanner_long_axial(max_ring_difference=38, n_angles=96, n_radial=96)
    scan["n_crystals"] = 192
    scan["detector_radius"] = 39.0            # explicit centres instead of the phantom's
    beds = []
    for k, c in enumerate(inputs.bed_centers(size, 4, 20.0)):
        beds.append(scenes.scene_from_arrays(str(tmp_path), mat, rho, act, vs, tissues=used, seed=500 + k,
                                             detector_center=c, **scan))
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=16)
    alone = [b.run(opts) for b in beds]
    batch = mcpet.Scene.run_batch(beds, opts)
    for k, (a, b) in enumerate(zip(alone, batch)):
        for key in ("trues", "scatter", "image_trues", "spectrum"):
            np.testing.assert_array_equal(getattr(a, key), getattr(b, key), err_msg=f"bed {k}: {key}")
        assert a.detected == b.detected and a.total_histories == b.total_histories
    # the beds see different parts of the body: the detected emission images differ
    det = [a.detected for a in alone]
    assert min(det) > 100 and len(set(det)) == 4
    z_mean = [np.average(np.arange(100), weights=a.image_trues.reshape(100, -1).sum(1)) for a in alone]
    assert all(z_mean[k] < z_mean[k + 1] for k in range(3)), z_mean
    for b in beds:
        b.close()


def test_long_axial_detector_bins_match_reference_fixture(tmp_path):
    """The GPU detector model against the reference's own tally_Sinogram on
    the long-axial scanner (fixture made by tests/golden/make_golden.py)."""
    from test_golden import _long_axial_cases
    for blur, sc, ev, want in _long_axial_cases(str(tmp_path)):
        got = mcpet.probe_detector(sc, ev)
        same = np.all(got[:, :4] == want[:, :4], axis=1)
        assert same.mean() >= 0.999, (blur, (~same).sum())
        assert (got[:, 0] >= 0).sum() > 500
        sc.close()
