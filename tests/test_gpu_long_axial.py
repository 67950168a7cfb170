"""Long-axial scanner at full size (256 rings x 0.4 cm, 768 crystals, 384 x 384
bins, span 11, MRD 255 -> 12333 sinogram planes, 1.82e9 bins, 7.3 GB per int32
sinogram).  The reference cannot run it: its byte counts NBINS*4 are 32-bit
ints (MCGPU-PET.cu:294-295).  Here the sizes are 64-bit:

* the detector model bins events spread over the 102 cm axial FOV exactly as
  the oracle's restatement does, including bins above 1.5e9;
* a full transport run allocates, zeroes, fills and downloads both 7.3 GB
  sinograms, with counts in the top segments and no guard trips.
"""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
from oracle import pyoracle
import scenes

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
