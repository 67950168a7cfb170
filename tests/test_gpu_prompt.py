"""Prompt-gamma emitter on the GPU (no counterpart in the reference, which
emits only 511 keV photons, MCGPU-PET_kernel.cu:669).

* Material tables continued to 1250 keV change nothing for 511 keV photons:
  identical tallies to the reference's 5-515 keV tables, and the reference's
  own CUDA run on the extended tables still replays ours.
* An isotope with a 1157 keV prompt gamma at 100 % yield agrees with the
  oracle's restatement of the same emitter (statistically: other seed),
  both lane layouts; the history loop and the event kernel agree; a batch
  mixing pure positron emitters and prompt emitters gives every scene its
  tallies alone.
"""
import math

import numpy as np
import pytest

import mcpet
from mcpet import inputs
from oracle import pyoracle
import refbind
import scenes
from test_gpu_transport import assert_replay, coarse, overlap

pytestmark = pytest.mark.gpu
PROMPT_EV = 1157020.0


def test_extended_tables_leave_511_kev_results_unchanged(workdir):
    mat, rho, act, vs, used = inputs.head_phantom(shape=(24, 48, 48), voxel_cm=0.5, seed=3, total_bq=4e5)
    a = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, **inputs.scanner_for_head())
    b = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, extended=True, **inputs.scanner_for_head())
    assert b.info.n_energy == 24901 and a.info.n_energy == 10200
    for lanes in (mcpet.LANES_REFERENCE, mcpet.LANES_BALANCED):
        ra, rb = a.run(mcpet.RunOptions(lane_mode=lanes)), b.run(mcpet.RunOptions(lane_mode=lanes))
        for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
            np.testing.assert_array_equal(getattr(ra, k), getattr(rb, k), err_msg=f"{lanes}: {k}")
        assert ra.total_histories == rb.total_histories
    a.close()
    b.close()


@pytest.mark.needs_ref("libref_prog.so")
def test_reference_run_on_extended_tables_replays(workdir):
    mat, rho, act, vs = inputs.water_cube_phantom(1.0e6)
    inp = scenes.write_case(workdir, "ext_replay", mat, rho, act, vs, extended=True, seed=4242)
    with mcpet.Scene.load(inp) as sc:
        cfg, info = sc.config, sc.info
        assert info.n_energy == 24901
        mine = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE))
    ref = refbind.RefProg().run(inp, int(cfg.n_bins), int(info.n_voxels), cfg.n_energy_bins, cwd=workdir)
    assert_replay(cfg, mine, ref)


def _prompt_scene(workdir, total_bq=1.0e6, yield_=1.0):
    mat, rho, act, vs = inputs.water_cube_phantom(total_bq)
    return scenes.scene_from_arrays(workdir, mat, rho, act, vs, extended=True, prompt_gamma_energy=PROMPT_EV,
                                    prompt_gamma_yield=yield_)


@pytest.mark.parametrize("lanes", [mcpet.LANES_REFERENCE, mcpet.LANES_BALANCED])
def test_prompt_gamma_statistics_vs_oracle(workdir, lanes):
    sc = _prompt_scene(workdir)
    cfg = sc.config
    res = sc.run(mcpet.RunOptions(lane_mode=lanes, seed_override=1001))
    assert sc.guard_trips() == 0
    ref = pyoracle.OracleScene(sc, seed=2002).run(n_threads=0)
    # three photons per decay, each decay once in both runs up to Poisson noise
    d_m, d_r = res.total_histories / 3, ref["total_histories"] / 3
    assert abs(d_m - d_r) <= 3 * math.sqrt(d_m + d_r) + 1
    for k in ("trues", "scatter"):
        a, b = int(getattr(res, k).sum()), int(ref[k].sum())
        assert abs(a - b) <= 3 * math.sqrt(a + b) + 1, (k, a, b)
    chi, dof = scenes.chi2_per_dof(coarse(res.trues + res.scatter, cfg), coarse(ref["trues"] + ref["scatter"], cfg),
                                   min_count=20)
    assert dof > 1000 and 0.9 <= chi <= 1.1, (chi, dof)
    chi, dof = scenes.chi2_per_dof(res.image_scatter, ref["image_scatter"], min_count=20)
    assert 0.8 <= chi <= 1.2, (chi, dof)
    chi, dof = scenes.chi2_per_dof(res.spectrum, ref["spectrum"], min_count=20)
    assert 0.7 <= chi <= 1.3, (chi, dof)
    # the gamma adds spurious (scatter-class) coincidences and leaves the trues alone
    plain = scenes.water_cube_scene(workdir, 1.0e6).run(mcpet.RunOptions(lane_mode=lanes, seed_override=3003))
    t_p, t_g = int(plain.trues.sum()), int(res.trues.sum())
    assert abs(t_p - t_g) <= 3 * math.sqrt(t_p + t_g) + 1
    assert int(res.scatter.sum()) > int(plain.scatter.sum()) + 5 * math.sqrt(int(plain.scatter.sum()))
    sc.close()


def test_prompt_gamma_partial_yield_vs_oracle(workdir):
    sc = _prompt_scene(workdir, yield_=0.5)
    res = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, seed_override=11))
    ref = pyoracle.OracleScene(sc, seed=12).run(n_threads=0)
    for k in ("trues", "scatter"):
        a, b = int(getattr(res, k).sum()), int(ref[k].sum())
        assert abs(a - b) <= 3 * math.sqrt(a + b) + 1, (k, a, b)
    # 2 photons per decay plus one per emitted gamma: about 2.5 per decay
    assert abs(res.total_histories / ref["total_histories"] - 1) < 0.01
    sc.close()


def test_prompt_gamma_history_and_event_kernels_agree(workdir):
    sc = _prompt_scene(workdir, total_bq=3.0e5)
    a = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, algorithm=mcpet.ALGORITHM_EVENTS))
    b = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, algorithm=mcpet.ALGORITHM_HISTORIES))
    assert a.total_histories == b.total_histories
    for k in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
        assert overlap(getattr(a, k), getattr(b, k)) >= 0.9999, k
    sc.close()


def test_batch_mixing_prompt_and_pure_emitters_equals_runs_alone(workdir):
    torch = pytest.importorskip("torch")
    scs = []
    for k, (mat, rho, act, vs, used) in enumerate(inputs.batch_phantoms(4, 2.0e5, seed=9)):
        kw = dict(inputs.scanner_batch(), seed=500 + k)
        if k % 2:
            kw.update(prompt_gamma_energy=PROMPT_EV)
        scs.append(scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=list(inputs.TISSUES)[:8],
                                            extended=True, **kw))
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=64)
    alone = []
    for s in scs:
        t = mcpet.device_tallies_for(s)
        s.run_device(t, opts)
        torch.cuda.synchronize()
        alone.append({k: v.cpu().numpy() for k, v in t.items()})
    tal = [mcpet.device_tallies_for(s) for s in scs]
    mcpet.Scene.run_batch_device(scs, tal, opts)
    torch.cuda.synchronize()
    for k, (t, want) in enumerate(zip(tal, alone)):
        for key in ("trues", "scatter", "image_trues", "image_scatter", "spectrum", "histories", "coincidences"):
            np.testing.assert_array_equal(t[key].cpu().numpy(), want[key], err_msg=f"scene {k}: {key}")
    assert scs[0].guard_trips() == 0
    for s in scs:
        s.close()


def test_batch_with_a_large_prompt_scene_in_its_own_launch(workdir):
    """A prompt-gamma head of 2.5e7 decays runs as a chained launch of its
    own (the single-scene kernel's prompt variant), the small scenes share
    the batch launch: every scene equals its run alone (automatic lanes)."""
    mat, rho, act, vs, _ = inputs.head_phantom(shape=(40, 64, 64), voxel_cm=0.4, seed=21, total_bq=2.5e7)
    big = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=list(inputs.TISSUES)[:8], extended=True,
                                   seed=31, prompt_gamma_energy=PROMPT_EV, **inputs.scanner_batch())
    scs = [big]
    for k, (m, r, a, v, used) in enumerate(inputs.batch_phantoms(2, 2.0e5, seed=5)):
        scs.append(scenes.scene_from_arrays(workdir, m, r, a, v, tissues=list(inputs.TISSUES)[:8], extended=True,
                                            seed=600 + k, **inputs.scanner_batch()))
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED)
    alone = [s.run(opts) for s in scs]
    batch = mcpet.Scene.run_batch(scs, opts)
    for k, (a, b) in enumerate(zip(alone, batch)):
        for key in ("trues", "scatter", "image_trues", "image_scatter", "spectrum"):
            np.testing.assert_array_equal(getattr(a, key), getattr(b, key), err_msg=f"scene {k}: {key}")
        assert a.total_histories == b.total_histories and a.detected == b.detected
    assert alone[0].total_histories > 2 * 2.4e7     # three photons per decay
    for s in scs:
        s.close()
