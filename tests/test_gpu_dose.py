"""Dose tallies (material dose and ROI voxel dose) on the GPU.

* Replay against the reference's own CUDA build (same input, seed and lanes):
  material and voxel energy sums agree (integer sums of per-interaction
  rounded terms; the rare history that diverges by FP32 rounding moves a
  few interactions, so sums are compared to 1e-4 and voxels to >= 99.9 %).
* The dose tallies draw no random numbers: sinograms are unchanged.
* History and event schedules give identical sums; so do batched runs.
* The writers produce the reference's files.
"""
import os

import numpy as np
import pytest

import mcpet
from mcpet import inputs
import refbind
import scenes

pytestmark = pytest.mark.gpu
needs_ref_prog = pytest.mark.needs_ref("libref_prog.so")
ROI = (2, 40, 3, 60, 5, 28)                    # 1-based, inside a 32x64x64 head


def _head_case(workdir, name, **kw):
    mat, rho, act, vs, used = inputs.head_phantom(shape=(32, 64, 64), voxel_cm=0.4, seed=11, total_bq=1e6)
    return scenes.write_case(workdir, name, mat, rho, act, vs, tissues=used, seed=777, material_dose=True,
                             voxel_dose=True, dose_roi=ROI, dose_file="head_dose.dat", **inputs.scanner_batch(), **kw)


@needs_ref_prog
def test_dose_replays_reference_cuda_build(workdir):
    inp = _head_case(workdir, "dose_rp")
    with mcpet.Scene.load(inp) as sc:
        cfg, info = sc.config, sc.info
        mine = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE))
    ref = refbind.RefProg().run(inp, int(cfg.n_bins), int(info.n_voxels), cfg.n_energy_bins, cwd=workdir,
                                dose_voxels=int(info.n_dose_voxels))
    assert ref["n_roi"] == info.n_dose_voxels
    assert list(ref["roi"]) == list(cfg.dose_roi)
    md, rd = mine.material_dose.astype(np.float64), ref["material_dose"].astype(np.float64)
    assert md[:, 0].sum() > 0
    np.testing.assert_allclose(md, rd, rtol=1e-4)
    vm, vr = mine.voxel_dose, ref["voxel_dose"]
    assert vm.shape == vr.shape and vr[:, 0].sum() > 0
    same = np.all(vm == vr, axis=1)
    assert same.mean() >= 0.999, same.mean()
    np.testing.assert_allclose(vm[:, 0].sum(dtype=np.float64), vr[:, 0].sum(dtype=np.float64), rtol=1e-4)


def test_dose_leaves_transport_unchanged_and_schedules_agree(workdir):
    inp = _head_case(workdir, "dose_on")
    off = scenes.write_case(workdir, "dose_off", *inputs.head_phantom(shape=(32, 64, 64), voxel_cm=0.4, seed=11,
                                                                      total_bq=1e6)[:4],
                            tissues=inputs.head_phantom(shape=(32, 64, 64), voxel_cm=0.4, seed=11,
                                                        total_bq=1e6)[4], seed=777, **inputs.scanner_batch())
    opts = {a: mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, algorithm=a)
            for a in (mcpet.ALGORITHM_EVENTS, mcpet.ALGORITHM_HISTORIES)}
    with mcpet.Scene.load(inp) as sc, mcpet.Scene.load(off) as sc_off:
        ev = sc.run(opts[mcpet.ALGORITHM_EVENTS])
        hi = sc.run(opts[mcpet.ALGORITHM_HISTORIES])
        plain = sc_off.run(opts[mcpet.ALGORITHM_EVENTS])
        assert plain.material_dose is None
    for k in ("trues", "scatter", "spectrum", "image_trues"):
        np.testing.assert_array_equal(getattr(ev, k), getattr(plain, k), err_msg=k)
    np.testing.assert_array_equal(ev.material_dose, hi.material_dose)
    np.testing.assert_array_equal(ev.voxel_dose, hi.voxel_dose)


def test_dose_in_batches_and_outputs(workdir):
    inp = _head_case(workdir, "dose_b")
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=8)
    with mcpet.Scene.load(inp) as a, mcpet.Scene.load(inp) as b:
        alone = a.run(opts)
        ba, bb = mcpet.Scene.run_batch([a, b], opts)
        np.testing.assert_array_equal(ba.material_dose, alone.material_dose)
        np.testing.assert_array_equal(bb.voxel_dose, alone.voxel_dose)
        out = os.path.join(workdir, "dose_out")
        os.makedirs(out, exist_ok=True)
        a.write_outputs(alone, out_dir=out)
        n = a.info.n_dose_voxels
    raw = np.fromfile(os.path.join(out, "head_dose.dat.raw"), np.float32)
    err = np.fromfile(os.path.join(out, "head_dose.dat_PercentRelError2sigma.raw"), np.float32)
    assert raw.size == err.size == n and raw.max() > 0
    txt = open(os.path.join(out, "head_dose.dat")).read()
    assert "Total energy absorved inside the dose ROI" in txt
    mats = open(os.path.join(out, "materials_dose.txt")).read()
    assert "MATERIALS TOTAL DOSE TALLY REPORT" in mats and "water_5-515keV" in mats
