"""Phantom and interpolation tables: bit-identical to the reference loaders
(load_voxels MCGPU-PET.cu:1381-1533, load_material :1565-1831)."""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
import refbind
import scenes

pytestmark = pytest.mark.skipif(not refbind.available("libref_cuda.so"), reason="reference build not present")


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _cases():
    yield "sample", inputs.sample_phantom() + (("air", "soft"),), {}
    m, r, a, v = inputs.water_cube_phantom(1.0e5)
    yield "water_cube_gz", (m, r, a, v, ("air", "soft")), {"gz": True}
    m, r, a, v = inputs.sample_phantom()
    yield "density_factor", (m, r, a, v, ("air", "soft")), {"density_factor": 0.37}
    m, r, a, v, used = inputs.head_phantom(shape=(12, 24, 24), voxel_cm=1.0, seed=5, total_bq=1e4)
    yield "head_tissues", (m, r, a, v, tuple(used)), dict(inputs.scanner_for_head())
    # tables continued to 1250 keV (mcpet.tables), read by both loaders
    yield "extended_tables", (m, r, a, v, tuple(used)), dict(inputs.scanner_for_head(), extended=True,
                                                             prompt_gamma_energy=1157020.0)


@pytest.mark.parametrize("name,arrays,kw", list(_cases()), ids=[c[0] for c in _cases()])
def test_tables_bit_identical_to_reference_loader(workdir, name, arrays, kw):
    mat, rho, act, vs, tissues = arrays
    kw = dict(kw)
    gz = kw.pop("gz", False)
    ext = kw.pop("extended", False)
    inp = scenes.write_case(workdir, f"tab_{name}", mat, rho, act, vs, tissues=tissues, gz=gz, extended=ext, **kw)
    ref_cfg, ref_vox, ref_t = refbind.RefIO().load(inp)
    with mcpet.Scene.load(inp) as sc:
        t = sc.export_tables()
        info = sc.info
        used = [m for m in range(15) if ref_cfg.density_max[m] > 0]
        assert used, "no material used"
        assert info.n_energy == ref_cfg.n_e
        assert np.float32(info.e0) == np.float32(ref_cfg.e0) and np.float32(info.inv_de) == np.float32(ref_cfg.ide)
        np.testing.assert_array_equal(_bits(t["voxels"]), _bits(ref_vox))
        # the reference leaves the slope of the last Woodcock row uninitialised
        np.testing.assert_array_equal(_bits(t["woodcock"][:-1]), _bits(ref_t.woodcock[:-1]))
        np.testing.assert_array_equal(_bits(t["mfp_a"][:, used]), _bits(ref_t.mfp_a[:, used]))
        np.testing.assert_array_equal(_bits(t["mfp_b"][:, used]), _bits(ref_t.mfp_b[:, used]))
        np.testing.assert_array_equal(_bits(t["pmax"][:, used]), _bits(ref_t.pmax[: info.n_energy, used]))
        for k in ["fco", "uico", "fj0", "noscco", "xco", "pco", "aco", "bco", "itlco", "ituco"]:
            np.testing.assert_array_equal(t[k], getattr(ref_t, k), err_msg=k)
        for m in used:
            assert np.float32(info.density_max[m]) == np.float32(ref_cfg.density_max[m])
            assert np.float32(info.density_nominal[m]) == np.float32(ref_cfg.density_nominal[m])


def test_palette_is_lossless(workdir):
    mat, rho, act, vs, used = inputs.head_phantom(shape=(12, 24, 24), voxel_cm=1.0, seed=5, total_bq=1e4)
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, **inputs.scanner_for_head())
    t = sc.export_tables()
    assert sc.info.n_palette == len(set(zip(mat.ravel().tolist(), rho.ravel().tolist())))
    np.testing.assert_array_equal(t["voxels"][:, 1], rho.ravel())
    np.testing.assert_array_equal((t["voxels"][:, 0] - 1).astype(np.int32), mat.ravel() - 1)
    sc.close()
