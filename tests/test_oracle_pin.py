"""Pin of the C oracle: bit-identical to the reference transport kernel compiled
for the host (oracle/_ref/libref_cpu.so, built from MCGPU-PET_kernel.cu where it
lies).  Sinograms, images, spectrum, histories and PSF records must all match."""
import numpy as np
import pytest

from mcpet import inputs
from oracle import pyoracle
import refbind
import scenes

pytestmark = pytest.mark.skipif(not refbind.available("libref_cpu.so"), reason="reference host build not present")


def _run_both(sc, background=False, psf_capacity=0, voxel_list=None):
    osc = pyoracle.OracleScene(sc, background=background)
    o = osc.run(n_threads=4, psf_capacity=psf_capacity, voxel_list=voxel_list)
    p = refbind.params_from_scene(sc, peta=0 if background else 1)
    r = refbind.RefCPU().run(p, osc.t["voxels"], refbind.RefTables.from_scene_export(osc.t), n_threads=4,
                             psf_capacity=psf_capacity, block_list=voxel_list)
    return o, r


def _assert_same(o, r, sino=True):
    assert o["total_histories"] == r["total_histories"]
    assert o["psf_count"] == r["psf_count"]
    if sino:
        for k in ["trues", "scatter", "image_trues", "image_scatter", "spectrum"]:
            np.testing.assert_array_equal(o[k], r[k], err_msg=k)
    if o["psf_raw"] is not None and len(o["psf_raw"]):
        a, b = scenes.psf_records(o["psf_raw"]), scenes.psf_records(r["psf_raw"])
        assert len(a) == len(b)
        assert a.tobytes() == b.tobytes()


def test_pin_sample_psf_and_sinogram(workdir):
    sc = scenes.sample_scene(workdir, tally_psf_sinogram=0, psf_size=100000)
    o, r = _run_both(sc, psf_capacity=100000)
    assert o["trues"].sum() > 100 and o["psf_count"] > 100
    _assert_same(o, r)


def test_pin_background_mode(workdir):
    sc = scenes.sample_scene(workdir, seed=4242)
    o, r = _run_both(sc, background=True)
    assert o["trues"].sum() + o["scatter"].sum() > 50
    _assert_same(o, r)


@pytest.mark.parametrize("tally_type", [1, 2])
def test_pin_tally_type_filters(workdir, tally_type):
    sc = scenes.sample_scene(workdir, tally_type=tally_type, tally_psf_sinogram=0, psf_size=50000, seed=99)
    o, r = _run_both(sc, psf_capacity=50000)
    _assert_same(o, r)
    if tally_type == 1:
        assert o["scatter"].sum() == 0
    else:
        assert o["trues"].sum() == 0


def test_pin_psf_only_with_overflow(workdir):
    # capacity far below the number of detections: the counter keeps counting;
    # which pairs fill the first slots depends on thread timing, so the stored
    # records are checked against the complete set of an unbounded run
    sc = scenes.sample_scene(workdir, tally_psf_sinogram=1, psf_size=64, seed=5)
    o, r = _run_both(sc, psf_capacity=64)
    assert o["psf_count"] == r["psf_count"] > 64
    assert o["total_histories"] == r["total_histories"]
    full, _ = _run_both(sc, psf_capacity=o["psf_count"] + 2)
    everything = {rec.tobytes() for rec in scenes.psf_records(full["psf_raw"])}
    for part in (o, r):
        recs = scenes.psf_records(part["psf_raw"])
        assert len(recs) == 64
        assert all(rec.tobytes() in everything for rec in recs)


def test_pin_span11_scanner_with_decay(workdir):
    sc = scenes.water_cube_scene(workdir, 3.0e4, fov_z=12.656, n_rows=80, n_crystals=336, n_angles=168,
                                 n_radial=147, n_z_slices=159, max_ring_difference=79, span=11,
                                 detector_radius=-9.05, detector_height=12.656, mean_life_s=0.5, seed=31)
    o, r = _run_both(sc)
    assert o["trues"].sum() > 100
    _assert_same(o, r)


def test_pin_head_tissues_subset(workdir):
    sc = scenes.small_head_scene(workdir, total_bq=3.0e4, shape=(12, 24, 24), voxel_cm=1.0)
    voxels = np.nonzero(sc.export_tables()["voxels"][:, 2] > 0)[0][::3].astype(np.int32)
    o, r = _run_both(sc, voxel_list=voxels)
    assert o["trues"].sum() + o["scatter"].sum() > 50
    _assert_same(o, r)


def test_pin_rng_and_probes(workdir):
    ref = refbind.RefCPU()
    ids = np.concatenate([np.arange(0, 300), [5_000_000, 33_554_431, 838_860_799]])
    s1, f1, d1 = pyoracle.rng(12345, ids, 10)
    s2, f2, d2 = ref.prng(12345, ids, 10)
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(f1, f2)
    np.testing.assert_array_equal(d1, d2)
    sc = scenes.sample_scene(workdir)
    osc = pyoracle.OracleScene(sc)
    rt = refbind.RefTables.from_scene_export(osc.t)
    seeds = s1[:200]
    for m in (0, 1):
        for e in (510998.95, 200000.0, 30000.0, 6000.0):
            en = np.full(200, e, np.float32)
            mm = np.full(200, m, np.int32)
            a = pyoracle.compton(osc, en, mm, seeds)
            b = ref.gcoa(rt, en, mm, seeds)
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y)
            pm = np.full(200, osc.t["pmax"][int((e - 5000) * 0.02) + 1, m], np.float32)
            a = pyoracle.rayleigh(osc, en, mm, pm, seeds)
            b = ref.graa(rt, en, mm, pm, seeds)
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y)
    ev = scenes.random_events(5000, np.random.default_rng(11))
    p = refbind.params_from_scene(sc)
    np.testing.assert_array_equal(pyoracle.detector(osc, ev), ref.sinogram_events(p, ev))


def test_pin_dose_tallies(workdir):
    """Material and ROI voxel dose (tally_materials_dose, tally_voxel_energy_deposition):
    the oracle's sums equal the reference host build's, term by term rounding included;
    the ROI's upper corner beyond the phantom is clipped as load_voxels does."""
    sc = scenes.sample_scene(workdir, material_dose=True, voxel_dose=True, dose_roi=(2, 8, 1, 9, 4, 99), seed=777)
    cfg, info = sc.config, sc.info
    assert list(cfg.dose_roi) == [1, 7, 0, 8, 3, 8]          # 0-based, z clipped to the 9-voxel phantom
    assert info.n_dose_voxels == 7 * 9 * 6
    osc = pyoracle.OracleScene(sc)
    o = osc.run(n_threads=4)
    p = refbind.params_from_scene(sc, peta=1)
    r = refbind.RefCPU().run(p, osc.t["voxels"], refbind.RefTables.from_scene_export(osc.t), n_threads=1,
                             material_dose=True, dose_roi=list(cfg.dose_roi))
    _assert_same(o, r)
    assert o["material_dose"][:, 0].sum() > 0 and o["voxel_dose"][:, 0].sum() > 0
    np.testing.assert_array_equal(o["material_dose"], r["material_dose"])
    np.testing.assert_array_equal(o["voxel_dose"], r["voxel_dose"])
    sc.close()


def test_pin_long_axial_body_phantom(workdir):
    """The long-axial rings (256 x 4 mm, span 11, MRD 38; a 192-crystal ring with
    96 x 96 bins keeps the sinograms small) around the body phantom with lungs
    (0.3 g/cm^3) and bone (1.85 g/cm^3)."""
    mat, rho, act, vs, used = inputs.body_phantom(shape=(50, 32, 32), voxel_cm=1.6, seed=5, total_bq=2.0e4)
    scan = inputs.scanner_long_axial(max_ring_difference=38, n_angles=96, n_radial=96)
    scan["n_crystals"] = 192
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, seed=606, **scan)
    assert sc.config.n_sinograms == 3373
    o, r = _run_both(sc)
    assert o["trues"].sum() + o["scatter"].sum() > 200
    _assert_same(o, r)
    sc.close()


def test_pin_many_phantom_workload_geometry(workdir):
    """A phantom of the many-phantom workload (seeded head-like cube at 2-4 mm)
    in the 32-ring batch scanner, a subset of its emitting voxels."""
    mat, rho, act, vs, used = next(inputs.batch_phantoms(1, 2.0e5, seed=8))
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, seed=1000, **inputs.scanner_batch())
    voxels = np.nonzero(sc.export_tables()["voxels"][:, 2] > 0)[0][::5].astype(np.int32)
    o, r = _run_both(sc, voxel_list=voxels)
    assert o["trues"].sum() + o["scatter"].sum() > 100
    _assert_same(o, r)
    sc.close()


def test_batch_phantoms_shapes():
    shapes = [(p[0].shape, p[3]) for p in inputs.batch_phantoms(6, 1.0e6, seed=3)]
    again = [(p[0].shape, p[3]) for p in inputs.batch_phantoms(6, 1.0e6, seed=3)]
    assert shapes == again
    for (nz, ny, nx), vs in shapes:
        assert nz == ny == nx and 32 <= nx <= 192
        assert 0.0 < vs[0] <= 0.4 + 1e-12 and nx * vs[0] <= 40.0 + 1e-9
