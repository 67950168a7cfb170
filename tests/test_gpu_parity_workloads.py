"""Parity at the stated workloads, against the reference's own CUDA build on
the same GPU and the same input files.

* The head workload exactly as the benchmark times it (128x128x64 voxels of
  2 mm, 1e9 decays, 64-ring scanner, 256 x 256 x 8065 sinograms; balanced
  lanes, the default event kernel) against the reference's run of the same
  .in file (its own read_input / load_voxels / load_material /
  track_particles, MCGPU-PET.cu:228-535).  The two runs use different lanes
  and random streams, so the check is statistical: trues, scatter and their
  sum within 3 sigma, chi^2/dof of coarse-binned sinograms in [0.9, 1.1],
  and chi^2 of the emission images and the energy spectrum.
* The plain small workload at its stated size (9^3 water cube, 1e7 decays,
  147 x 168 x 421 sinogram): reference lanes replay the reference's run, so
  >= 99.9 % of the counts sit in identical bins.

Both kernel times (CUDA events) are printed for the record.
"""
import math

import numpy as np
import pytest

import mcpet
from mcpet import inputs
import refbind
import scenes
from test_gpu_transport import assert_replay, replay

pytestmark = [pytest.mark.gpu, pytest.mark.needs_ref("libref_prog.so")]


def coarse_sum(trues: np.ndarray, scatter: np.ndarray, cfg, f) -> np.ndarray:
    """trues + scatter summed over blocks of f = (planes, angles, radial)
    bins; the sinogram dimensions must be multiples of f."""
    shape = (cfg.n_sinograms, cfg.n_angles, cfg.n_radial)
    assert all(n % k == 0 for n, k in zip(shape, f)), (shape, f)
    s = trues.reshape(shape) + scatter.reshape(shape)
    a, b, c = (n // k for n, k in zip(shape, f))
    return s.reshape(a, f[0], b, f[1], c, f[2]).sum(axis=(1, 3, 5), dtype=np.int64)


def within_3_sigma(a: int, b: int) -> bool:
    return abs(a - b) <= 3.0 * math.sqrt(a + b) + 1


def test_head_workload_as_timed_matches_reference_cuda_run(workdir):
    mat, rho, act, vs, used, scan = inputs.head_workload(1.0e9)
    inp = scenes.write_case(workdir, "timed_head", mat, rho, act, vs, tissues=used, **scan)
    with mcpet.Scene.load(inp) as sc:
        cfg, info = sc.config, sc.info
        mine = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
        assert sc.guard_trips() == 0
    ref = refbind.RefProg().run(inp, int(cfg.n_bins), int(info.n_voxels), cfg.n_energy_bins, cwd=workdir)
    print(f"\nhead workload, 1e9 decays: this library {mine.transport_ms:.1f} ms, reference CUDA build "
          f"{ref['kernel_ms']:.1f} ms ({ref['kernel_ms'] / mine.transport_ms:.2f}x); coincidences "
          f"{mine.coincidences} vs {int(ref['trues'].sum(dtype=np.int64) + ref['scatter'].sum(dtype=np.int64))}")

    # decays: Poisson counts of the same mean
    assert within_3_sigma(mine.total_histories // 2, ref["total_histories"] // 2)
    t_m, t_r = int(mine.trues.sum(dtype=np.int64)), int(ref["trues"].sum(dtype=np.int64))
    s_m, s_r = int(mine.scatter.sum(dtype=np.int64)), int(ref["scatter"].sum(dtype=np.int64))
    assert t_r > 10_000_000 and s_r > 10_000_000
    assert within_3_sigma(t_m, t_r), ("trues", t_m, t_r)
    assert within_3_sigma(s_m, s_r), ("scatter", s_m, s_r)
    assert within_3_sigma(t_m + s_m, t_r + s_r), ("total", t_m + s_m, t_r + s_r)

    # 8065 x 256 x 256 -> 1613 x 16 x 16 blocks of ~140 counts
    f = (5, 16, 16)
    cm = coarse_sum(mine.trues, mine.scatter, cfg, f)
    cr = coarse_sum(ref["trues"], ref["scatter"], cfg, f)
    chi, dof = scenes.chi2_per_dof(cm, cr, min_count=20)
    print(f"sinogram chi2/dof {chi:.4f} over {dof} blocks")
    assert dof > 100_000 and 0.9 <= chi <= 1.1, (chi, dof)
    # trues and scatter separately, coarser (scatter is spread thinly)
    for k, g in (("trues", (5, 16, 16)), ("scatter", (5, 32, 32))):
        z = np.zeros_like(mine.trues)
        chi, dof = scenes.chi2_per_dof(coarse_sum(getattr(mine, k), z, cfg, g), coarse_sum(ref[k], z, cfg, g),
                                       min_count=20)
        assert dof > 10_000 and 0.9 <= chi <= 1.1, (k, chi, dof)
    chi, dof = scenes.chi2_per_dof(mine.image_trues + mine.image_scatter, ref["image_trues"] + ref["image_scatter"],
                                   min_count=20)
    assert dof > 100_000 and 0.9 <= chi <= 1.1, ("image", chi, dof)
    chi, dof = scenes.chi2_per_dof(mine.spectrum, ref["spectrum"], min_count=20)
    assert 0.8 <= chi <= 1.2, ("spectrum", chi, dof)


def test_plain_small_workload_at_stated_size_replays_reference_cuda_run(workdir):
    mat, rho, act, vs = inputs.water_cube_phantom(1.0e7)
    inp = scenes.write_case(workdir, "c1_full", mat, rho, act, vs, seed=12345)
    cfg, mine, ref = replay(inp, workdir)
    assert cfg.n_sinograms == 421 and (cfg.n_angles, cfg.n_radial) == (168, 147)
    print(f"\n9^3 water cube, 1e7 decays (reference lanes): this library {mine.transport_ms:.1f} ms, reference "
          f"CUDA build {ref['kernel_ms']:.1f} ms")
    assert mine.total_histories == ref["total_histories"]
    assert mine.coincidences > 900_000
    assert_replay(cfg, mine, ref, min_overlap=0.999)
