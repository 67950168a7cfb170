"""The output writers (mcpet_write_outputs) on the host, fed with the C
oracle's tallies of the sample case: gzip'd int32 sinograms and images in the
reference's file names (standard and background mode), the spectrum table,
the PSF text and 44-byte binary records, and the dose reports."""
import gzip
import os

import numpy as np

import mcpet
from oracle import pyoracle
import scenes


def _oracle_result(workdir):
    sc = scenes.sample_scene(workdir, tally_psf_sinogram=0, psf_size=50000, material_dose=True, voxel_dose=True,
                             dose_roi=(2, 8, 1, 9, 4, 99), seed=777)
    o = pyoracle.OracleScene(sc).run(n_threads=4, psf_capacity=50000)
    n = min(int(o["psf_count"]), 50000)
    psf = np.frombuffer(bytes(o["psf_raw"][: n * 44]), dtype=mcpet.PSF_DTYPE).copy()
    r = mcpet.RunResult(trues=o["trues"], scatter=o["scatter"], image_trues=o["image_trues"],
                        image_scatter=o["image_scatter"], spectrum=o["spectrum"], psf=psf,
                        psf_count=int(o["psf_count"]), total_histories=int(o["total_histories"]), transport_ms=12.5,
                        material_dose=o["material_dose"], voxel_dose=o["voxel_dose"])
    return sc, r


def _gz(path):
    with gzip.open(path) as f:
        return np.frombuffer(f.read(), np.int32)


def test_writers_standard_outputs(workdir):
    sc, r = _oracle_result(workdir)
    out = os.path.join(workdir, "writers_std")
    os.makedirs(out, exist_ok=True)
    sc.write_outputs(r, out)
    np.testing.assert_array_equal(_gz(os.path.join(out, "sinogram_Trues.raw.gz")), r.trues)
    np.testing.assert_array_equal(_gz(os.path.join(out, "sinogram_Scatter.raw.gz")), r.scatter)
    np.testing.assert_array_equal(_gz(os.path.join(out, "image_Trues.raw.gz")), r.image_trues)
    np.testing.assert_array_equal(_gz(os.path.join(out, "image_Scatter.raw.gz")), r.image_scatter)
    spec = np.loadtxt(os.path.join(out, "Energy_Sinogram_Spectrum.dat"), dtype=np.int64)
    np.testing.assert_array_equal(spec[:, 1], r.spectrum)
    psf_name = sc.config.psf_file.decode()
    raw = np.fromfile(os.path.join(out, psf_name + ".raw"), dtype=mcpet.PSF_DTYPE)
    assert len(raw) == len(r.psf) > 100
    assert raw.tobytes() == r.psf.tobytes()
    assert open(os.path.join(out, psf_name)).read().count("\n") > min(r.psf_count, 5000)
    n = sc.info.n_dose_voxels
    dose = np.fromfile(os.path.join(out, "mc-gpu_dose.dat.raw"), np.float32)
    err = np.fromfile(os.path.join(out, "mc-gpu_dose.dat_PercentRelError2sigma.raw"), np.float32)
    assert dose.size == err.size == n and dose.max() > 0
    assert "Total energy absorved inside the dose ROI" in open(os.path.join(out, "mc-gpu_dose.dat")).read()
    mats = open(os.path.join(out, "materials_dose.txt")).read()
    assert "MATERIALS TOTAL DOSE TALLY REPORT" in mats and "water_5-515keV" in mats
    sc.close()


def test_writers_background_mode_names(workdir):
    sc, r = _oracle_result(workdir)
    out = os.path.join(workdir, "writers_bg")
    os.makedirs(out, exist_ok=True)
    sc.write_outputs(r, out, background_mode=True)
    np.testing.assert_array_equal(_gz(os.path.join(out, "sinogram_BG_Trues.raw.gz")), r.trues)
    np.testing.assert_array_equal(_gz(os.path.join(out, "sinogram_BG_Scatter.raw.gz")), r.scatter)
    np.testing.assert_array_equal(_gz(os.path.join(out, "BG_image_True.raw.gz")), r.image_trues)
    np.testing.assert_array_equal(_gz(os.path.join(out, "BG_image_Scatter.raw.gz")), r.image_scatter)
    assert not os.path.exists(os.path.join(out, "sinogram_Trues.raw.gz"))
    sc.close()
