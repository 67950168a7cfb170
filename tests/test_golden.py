"""Oracle and library against the golden fixtures of tests/golden, which were
produced by the reference's own code (see tests/golden/make_golden.py)."""
import hashlib
import os

import numpy as np

from mcpet import inputs
from oracle import pyoracle
import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SPAN11 = dict(fov_z=12.656, n_rows=80, n_crystals=336, n_angles=168, n_radial=147, n_z_slices=159,
              max_ring_difference=79, span=11, detector_radius=-9.05, detector_height=12.656)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_oracle_rng_matches_golden_streams():
    g = np.load(os.path.join(GOLD, "rng_streams.npz"))
    s, f, d = pyoracle.rng(int(g["seed"]), g["ids"], g["draws"].shape[1])
    np.testing.assert_array_equal(s, g["seeds"])
    np.testing.assert_array_equal(f, g["draws"])
    np.testing.assert_array_equal(d, g["ddraws"])


def _kat_cases():
    g = np.load(os.path.join(GOLD, "detector_kat.npz"))
    for name, kw in (("span1", dict(inputs.scanner_small())), ("span11", SPAN11)):
        for blur in (0, 12):
            key = f"{name}_res{blur}"
            ev = {k: g[f"{key}_{k}"] for k in ["e2", "e1", "pos2", "pos1", "dir2", "dir1", "st2", "st1", "seeds"]}
            yield key, dict(kw, energy_resolution=blur / 100.0), ev, g[f"{key}_out"]


def test_oracle_detector_matches_golden_kat(workdir):
    for key, kw, ev, want in _kat_cases():
        sc = scenes.sample_scene(workdir, **kw)
        got = pyoracle.detector(pyoracle.OracleScene(sc), ev)
        np.testing.assert_array_equal(got, want, err_msg=key)
        assert (want[:, 0] >= 0).sum() > 100
        sc.close()


def test_oracle_sample_run_matches_golden(workdir):
    g = np.load(os.path.join(GOLD, "sample_run.npz"))
    sc = scenes.sample_scene(workdir, tally_psf_sinogram=0, psf_size=100000, seed=12345)
    o = pyoracle.OracleScene(sc).run(n_threads=4, psf_capacity=100000)
    assert o["total_histories"] == int(g["total_histories"])
    assert o["psf_count"] == int(g["psf_count"])
    for k in ["trues", "scatter", "image_trues", "image_scatter", "spectrum"]:
        nz = np.nonzero(o[k])[0]
        np.testing.assert_array_equal(nz, g[f"{k}_idx"], err_msg=k)
        np.testing.assert_array_equal(o[k][nz], g[f"{k}_val"], err_msg=k)
    assert _sha(scenes.psf_records(o["psf_raw"])) == str(g["psf_sha"])


def test_library_tables_match_golden_checksums(workdir):
    g = np.load(os.path.join(GOLD, "tables.npz"))
    sc = scenes.sample_scene(workdir)
    t = sc.export_tables()
    used = [0, 1]
    assert sc.info.n_energy == int(g["n_e"])
    assert sc.config.n_sinograms == 421
    assert _sha(t["woodcock"][:-1]) == str(g["woodcock"])
    assert _sha(t["mfp_a"][:, used]) == str(g["mfp_a"])
    assert _sha(t["mfp_b"][:, used]) == str(g["mfp_b"])
    assert _sha(t["pmax"][:, used]) == str(g["pmax"])
    assert _sha(np.concatenate([t["fco"], t["uico"], t["fj0"]])) == str(g["compton"])
    assert _sha(np.concatenate([t["xco"], t["pco"], t["aco"], t["bco"]])) == str(g["rayleigh"])
    assert _sha(t["voxels"]) == str(g["voxels"])
    sc.close()


def _long_axial_cases(workdir):
    g = np.load(os.path.join(GOLD, "detector_kat_long_axial.npz"))
    mat, rho, act, vs, used = inputs.body_phantom(shape=(50, 32, 32), voxel_cm=1.6, seed=5, total_bq=1.0e3)
    for blur in (0, 12):
        ev = {k: g[f"res{blur}_{k}"] for k in ["e2", "e1", "pos2", "pos1", "dir2", "dir1", "st2", "st1", "seeds"]}
        sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, energy_resolution=blur / 100.0,
                                      **inputs.scanner_long_axial())
        yield blur, sc, ev, g[f"res{blur}_out"]


def test_oracle_detector_matches_golden_long_axial(workdir):
    """The reference's tally_Sinogram on pairs spread over the 1 m scanner
    (span 11, MRD 255, bins up to 1.82e9): the oracle gives the same bins,
    classes, spectrum bins and RNG states."""
    for blur, sc, ev, want in _long_axial_cases(workdir):
        assert sc.config.n_bins == 12333 * 384 * 384
        got = pyoracle.detector(pyoracle.OracleScene(sc), ev)
        np.testing.assert_array_equal(got, want, err_msg=f"blur {blur}")
        assert (want[:, 0] >= 0).sum() > 500 and want[:, 0].max() > 1_500_000_000
        sc.close()
