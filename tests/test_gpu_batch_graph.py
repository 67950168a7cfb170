"""Batched regeneration in a CUDA graph (mcpet_batch_graph_*) and the
autotuner (mcpet_autotune).

* Graph launch r runs scene k with seed s_k + r * seed_step: its tallies equal
  those of the scene run alone with that seed, bit for bit, replay after
  replay; explicit seeds (set_seeds) likewise.
* The graph keeps its own lane plans: runs of the scenes with other options
  between replays do not change what the graph computes.
* The autotuner returns one of its candidates, restores the scenes (a default
  run after tuning equals one before), and its choice runs correctly.
"""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
import scenes

pytestmark = pytest.mark.gpu
HEAD_TISSUES = ("air", "soft", "grey", "white", "bone", "fat", "blood", "csf")
KEYS = ("trues", "scatter", "image_trues", "image_scatter", "spectrum")


def _scenes(tmp):
    out = []
    for k, (shape, vox, bq, seed) in enumerate((((16, 32, 32), 0.8, 2.0e5, 101), ((24, 40, 40), 0.6, 3.0e5, 202),
                                                 ((20, 36, 36), 0.7, 2.5e5, 303))):
        mat, rho, act, vs, _ = inputs.head_phantom(shape=shape, voxel_cm=vox, seed=7 + k, total_bq=bq)
        out.append(scenes.scene_from_arrays(str(tmp), mat, rho, act, vs, tissues=HEAD_TISSUES, seed=seed,
                                            **inputs.scanner_batch()))
    return out


def _check(sc, t, seed, opts, tag):
    import dataclasses
    a = sc.run(dataclasses.replace(opts, seed_override=seed))
    for k in KEYS:
        np.testing.assert_array_equal(t[k].cpu().numpy(), getattr(a, k), err_msg=f"{tag}: {k}")
    assert int(t["histories"].item()) == a.total_histories, tag
    assert int(t["coincidences"].item()) == a.detected, tag
    assert a.detected > 20, tag


def test_graph_replays_regenerate_histories(tmp_path):
    import torch
    sc = _scenes(tmp_path)
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=4)
    tal = [mcpet.device_tallies_for(s) for s in sc]
    seeds = [101, 202, 303]
    with mcpet.BatchGraph(sc, tal, opts, seed_step=5) as g:
        g.launch()
        torch.cuda.synchronize()
        for k in range(3):
            _check(sc[k], tal[k], seeds[k], opts, f"replay 0 scene {k}")
        # runs of the scenes with other options rebuild their own plans
        sc[0].run(mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE))
        g.launch()
        g.launch()
        torch.cuda.synchronize()
        for k in range(3):
            _check(sc[k], tal[k], seeds[k] + 10, opts, f"replay 2 scene {k}")
        assert g.guard_trips() == 0
        g.set_seeds([7, 8, 9])
        g.launch()
        torch.cuda.synchronize()
        for k in range(3):
            _check(sc[k], tal[k], 7 + k, opts, f"explicit seeds scene {k}")
    for s in sc:
        s.close()


def test_graph_with_a_scene_in_its_own_launch(tmp_path):
    """A head of 3e7 decays runs as its own launch inside the graph, chained
    before the launch of the small scenes; replays still equal runs alone."""
    import torch
    sc = _scenes(tmp_path)[:2]
    mat, rho, act, vs, _ = inputs.head_phantom(shape=(40, 64, 64), voxel_cm=0.4, seed=31, total_bq=3.0e7)
    sc.insert(1, scenes.scene_from_arrays(str(tmp_path), mat, rho, act, vs, tissues=HEAD_TISSUES, seed=404,
                                          **inputs.scanner_batch()))
    seeds = [101, 404, 202]
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED)
    tal = [mcpet.device_tallies_for(s) for s in sc]
    with mcpet.BatchGraph(sc, tal, opts, seed_step=3) as g:
        for r in range(2):
            g.launch()
            torch.cuda.synchronize()
            for k in range(3):
                _check(sc[k], tal[k], seeds[k] + 3 * r, opts, f"replay {r} scene {k}")
        assert g.guard_trips() == 0
    for s in sc:
        s.close()


def test_graph_with_seed_override_and_reference_lanes(tmp_path):
    import torch
    sc = _scenes(tmp_path)[:2]
    opts = mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE, seed_override=4444)
    tal = [mcpet.device_tallies_for(s) for s in sc]
    g = mcpet.BatchGraph(sc, tal, opts)
    for _ in range(2):
        g.launch()
    torch.cuda.synchronize()
    for k in range(2):
        _check(sc[k], tal[k], 4445, opts, f"scene {k}")
    g.close()
    for s in sc:
        s.close()


def test_autotune_picks_a_candidate_and_restores_scenes(tmp_path):
    import dataclasses
    sc = _scenes(tmp_path)
    base = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED)
    before = [s.run(base) for s in sc]
    tal = [mcpet.device_tallies_for(s) for s in sc]
    tuned, info = mcpet.autotune(sc, tal, base, sample_decays=2.0e5)
    print(info)
    assert info["candidates"] >= 3 and info["best_ms"] > 0
    assert info["best_ms"] <= info["auto_ms"] + 1e-9
    # histories_per_lane 0: the batch's automatic choice (every scene its own lanes) won
    assert tuned.block_threads in (128, 192, 256) and tuned.histories_per_lane >= 0
    after = [s.run(base) for s in sc]
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a.trues, b.trues)
        assert a.total_histories == b.total_histories
    # the tuned options give the same tallies batched and one by one
    alone = [s.run(tuned) for s in sc]
    batch = mcpet.Scene.run_batch(sc, tuned)
    for a, b in zip(alone, batch):
        np.testing.assert_array_equal(a.trues, b.trues)
        assert a.detected == b.detected
    # a single scene tunes through mcpet_run_device
    one, info1 = mcpet.autotune(sc[:1], tal[:1], dataclasses.replace(base, seed_override=9))
    assert info1["candidates"] >= 3
    for s in sc:
        s.close()
