"""Synthetic workload generators (host only): the long-axial body phantom, the
long-axial scanner and bed positions, and the ellipsoid painter they share
with the head phantoms."""
import numpy as np

import mcpet
from mcpet import inputs


def test_body_phantom_tissues_densities_and_activity():
    mat, rho, act, vs, used = inputs.body_phantom(shape=(200, 128, 128), voxel_cm=0.4, seed=3, total_bq=1.0e8)
    assert mat.shape == rho.shape == act.shape == (200, 128, 128) and vs == (0.4, 0.4, 0.4)
    assert used == list(inputs.TISSUES)                       # all 10 tissues present
    assert np.isclose(act.sum(dtype=np.float64), 1.0e8, rtol=1e-5)
    slot = {n: inputs.TISSUES[n][0] for n in inputs.TISSUES}
    assert np.all(rho[mat == slot["lung"]] == np.float32(0.3))
    assert np.all(rho[mat == slot["bone"]] == np.float32(1.85))
    assert act[mat == slot["air"]].max() == 0
    organ = act[mat == slot["organ"]].mean()
    soft = act[mat == slot["soft"]].mean()
    assert np.isclose(organ / soft, 8.0, rtol=1e-5)
    # the head sits at high z, the lungs in the torso
    z_grey = np.nonzero(mat == slot["grey"])[0].mean()
    z_lung = np.nonzero(mat == slot["lung"])[0].mean()
    assert z_grey > 0.8 * 200 > z_lung
    again = inputs.body_phantom(shape=(200, 128, 128), voxel_cm=0.4, seed=3, total_bq=1.0e8)
    assert np.array_equal(again[0], mat) and np.array_equal(again[2], act)


def test_long_axial_scanner_sizes(workdir):
    for mrd, planes in ((255, 12333), (38, 3373)):
        spec = inputs.spec_for(["a"], "x.vox", **inputs.scanner_long_axial(max_ring_difference=mrd))
        cfg = mcpet.read_config(inputs.write_input(f"{workdir}/_la_{mrd}.in", spec))
        assert cfg.n_sinograms == planes and cfg.n_bins == planes * 384 * 384
    assert 12333 * 384 * 384 * 4 > 2**31        # beyond the reference's 32-bit byte counts


def test_bed_centers():
    c = inputs.bed_centers((51.2, 51.2, 80.0), 4, 20.0)
    assert c == [(25.6, 25.6, 10.0), (25.6, 25.6, 30.0), (25.6, 25.6, 50.0), (25.6, 25.6, 70.0)]
    assert inputs.bed_centers((10.0, 10.0, 10.0), 1, 20.0) == [(5.0, 5.0, 5.0)]


def test_ellipsoid_matches_pointwise_formula():
    shape, vs = (7, 9, 11), (0.5, 0.4, 0.3)
    c, r = (1.7, 1.9, 1.3), (1.1, 1.4, 0.9)
    got = inputs._ellipsoid(shape, c, r, vs)
    z, y, x = np.meshgrid(*[(np.arange(n) + 0.5) * v for n, v in zip(shape, vs[::-1])], indexing="ij")
    want = (((x - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((z - c[2]) / r[2]) ** 2) <= 1.0
    assert np.array_equal(got, want) and got.any() and not got.all()
