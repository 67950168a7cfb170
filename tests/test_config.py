"""Input-file parsing: same values as the reference read_input (MCGPU-PET.cu:866-1280)."""
import os
import shutil

import numpy as np
import pytest

import mcpet
from mcpet import inputs
from oracle import pyoracle
import refbind
import scenes

needs_refio = pytest.mark.skipif(not refbind.available("libref_cuda.so"), reason="reference build not present")


def _spec_variants():
    yield "small", dict(inputs.scanner_small())
    yield "head", dict(inputs.scanner_for_head(), seed=777, tally_type=1, tally_psf_sinogram=0, psf_size=1000)
    yield "span11", dict(fov_z=12.656, n_rows=80, n_crystals=336, n_angles=168, n_radial=147, n_z_slices=159,
                         max_ring_difference=79, span=11, detector_radius=-9.05, detector_height=12.656,
                         energy_resolution=0.2, energy_low=400000.0, energy_high=650000.0, tally_type=2)
    yield "explicit_center", dict(inputs.scanner_small(), detector_center=(4.5, 4.0, 3.5), detector_radius=30.0,
                                  density_factor=0.5, mean_life_s=6586.2, acquisition_s=2.5, threads_per_block=64)
    yield "voxel_dose", dict(inputs.scanner_small(), voxel_dose=True, material_dose=True, tally_psf_sinogram=1,
                             psf_size=5000)


def _compare(mine, ref):
    assert mine.seed == ref.seed
    assert mine.gpu_id == ref.gpu_id
    assert mine.threads_per_block == ref.tpb
    assert np.float32(mine.density_factor) == np.float32(ref.fact_object)
    assert mine.acquisition_time_ps == ref.acq_ps
    assert np.float32(mine.mean_life) == np.float32(ref.mean_life)
    assert list(mine.detector_center) == [ref.cx, ref.cy, ref.cz]
    assert mine.detector_height == ref.height and mine.detector_radius == ref.radius
    assert mine.psf_size == ref.psf_size
    assert mine.tally_type == ref.tally_type and mine.tally_psf_sinogram == ref.tally_psf_sino
    assert mine.tally_material_dose == ref.flag_material_dose
    assert list(mine.dose_roi) == list(ref.roi)
    assert (mine.energy_resolution, mine.energy_window_low, mine.energy_window_high) == (ref.e_resol, ref.e_low,
                                                                                        ref.e_high)
    assert mine.fov_z == ref.fovz
    assert (mine.n_rows, mine.n_crystals, mine.n_angles, mine.n_radial, mine.n_z_slices, mine.image_res,
            mine.n_energy_bins, mine.max_ring_difference, mine.span) == (
        ref.nrows, ref.ncrystals, ref.nangles, ref.nrad, ref.nzs, ref.res, ref.ne, ref.mrd, ref.span)
    assert (mine.n_segments, mine.n_sinograms, mine.n_bins) == (ref.nseg, ref.nsinos, ref.nbins)
    assert mine.psf_file == ref.psf_file
    assert mine.voxel_file == ref.voxel_file
    for i in range(15):
        # the reference marks an absent slot with a lone newline, the library with ""
        assert mine.material_files[i].value == ref.materials[i].value.rstrip(b"\n")


@needs_refio
@pytest.mark.parametrize("name,kw", list(_spec_variants()), ids=[n for n, _ in _spec_variants()])
def test_scene_config_matches_reference_parser(workdir, name, kw):
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, f"cfg_{name}", mat, rho, act, vs, **kw)
    ref_cfg, _, _ = refbind.RefIO().load(inp)
    with mcpet.Scene.load(inp) as sc:
        _compare(sc.config, ref_cfg)


def test_sinogram_sizes_match_running_sum():
    # NSEG/NSINOS closed form in the library vs. the reference's running sum
    # restated in the oracle (MCGPU-PET.cu:1176-1187)
    cases = [(79, 11, 159), (14, 1, 29), (63, 1, 127), (31, 1, 63), (255, 11, 511), (0, 1, 1), (5, 3, 17),
             (20, 4, 41), (7, 7, 15), (100, 9, 201), (2, 5, 9)]
    rng = np.random.default_rng(3)
    for _ in range(40):
        span = int(rng.integers(1, 13))
        mrd = int(rng.integers(0, 300))
        rows = int(rng.integers(mrd + 1, mrd + 60))
        cases.append((mrd, span, 2 * rows - 1))
    spec = inputs.InputSpec(material_files=["a"])
    for mrd, span, nzs in cases:
        nseg, nsinos = pyoracle.sinogram_sizes(mrd, span, nzs)
        cfg = mcpet.read_config(inputs.write_input("/tmp/_mcpet_sizes.in", _with(spec, mrd, span, nzs)))
        assert (cfg.n_segments, cfg.n_sinograms) == (nseg, nsinos), (mrd, span, nzs)
        assert cfg.n_bins == cfg.n_radial * cfg.n_angles * nsinos


def _with(spec, mrd, span, nzs):
    spec.max_ring_difference, spec.span, spec.n_z_slices = mrd, span, nzs
    return spec


def test_known_geometries():
    spec = inputs.InputSpec(material_files=["a"])
    for (mrd, span, nzs), want in {(79, 11, 159): 1293, (14, 1, 29): 421, (63, 1, 127): 8065, (31, 1, 63): 1985,
                                   (255, 11, 511): 12333}.items():
        cfg = mcpet.read_config(inputs.write_input("/tmp/_mcpet_known.in", _with(spec, mrd, span, nzs)))
        assert cfg.n_sinograms == want


def test_reference_sample_input_parses(workdir):
    src = "/root/reference/sample_simulation/MCGPU-PET.in"
    if not os.path.exists(src):
        pytest.skip("reference sample not present")
    dst = os.path.join(workdir, "sample.in")
    shutil.copyfile(src, dst)
    cfg = mcpet.read_config(dst)
    assert cfg.seed != 0                      # 0 in the file: time-based seed
    assert cfg.threads_per_block == 32 and cfg.density_factor == 1.0
    assert cfg.acquisition_time_ps == 10 ** 12 and np.float32(cfg.mean_life) == np.float32(70000.0)
    assert cfg.psf_file == b"MCGPU_PET.psf" and cfg.psf_size == 150000000
    assert cfg.detector_radius == np.float32(-9.05) and cfg.detector_height == np.float32(12.656)
    assert cfg.tally_material_dose == 1 and cfg.tally_voxel_dose == 0
    assert (cfg.n_sinograms, cfg.n_segments) == (1293, 15)
    assert cfg.voxel_file == b"phantom_9x9x9cm.vox"
    assert cfg.material_files[0].value == b"./materials/air_5-515keV.mcgpu.gz"
    assert cfg.material_files[1].value == b"./materials/water_5-515keV.mcgpu.gz"
    assert cfg.material_files[2].value == b""


def test_quirks_of_value_lines(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, "quirks", mat, rho, act, vs, tally_type=7, tally_psf_sinogram=-3)
    text = open(inp).read().replace("#[SECTION SIMULATION CONFIG v.2016-07-05]\n",
                                    "#[SECTION SIMULATION CONFIG v.2016-07-05]\n\n   # a comment line\n\n")
    open(inp, "w").write(text)
    cfg = mcpet.read_config(inp)
    assert cfg.seed == 12345
    assert cfg.tally_type == 0 and cfg.tally_psf_sinogram == 0     # out-of-range -> 0
