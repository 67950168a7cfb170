"""Gradient of the sinogram Poisson log-likelihood (mcpet_grad).

Checks:
* the activity gradient is the exact derivative of the log-likelihood of the
  recorded events reweighted by A'_v / A_v (central difference in float64 over
  the event records, eps = 1e-3);
* replays reproduce the recorded bins (mismatch fraction below 1e-3);
* activity and density-scale directional derivatives over regions of the
  phantom agree with central finite differences of full forward runs using
  common random numbers (same seed and lanes), within the tolerance written
  in each test;
* the torch.autograd binding returns the same gradients.
"""
import numpy as np
import pytest

import mcpet
from mcpet import inputs
import scenes

pytestmark = pytest.mark.gpu
HEAD_TISSUES = ("air", "soft", "grey", "white", "bone", "fat", "blood", "csf")


def _phantom(seed=5, total_bq=2.0e7):
    mat, rho, act, vs, _ = inputs.head_phantom(shape=(32, 48, 48), voxel_cm=0.5, seed=seed, total_bq=total_bq)
    rng = np.random.default_rng(seed)
    rho = (rho * rng.uniform(0.9, 1.0, rho.shape)).astype(np.float32)   # densities below each tissue's max
    return mat, rho, act.astype(np.float32), vs


# coarse sinogram (16 x 16 x 64 bins): hundreds of counts per bin, so that a
# finite difference that adds or removes whole events measures the derivative
COARSE = dict(detector_radius=-41.0, detector_height=12.8, fov_z=12.8, n_rows=8, n_crystals=32, n_angles=16,
              n_radial=16, n_z_slices=15, max_ring_difference=7, span=1)


def _scene(tmp, mat, rho, act, vs, seed=12345, scanner=None):
    return scenes.scene_from_arrays(str(tmp), mat, rho, act, vs, tissues=HEAD_TISSUES, seed=seed,
                                    **(scanner or inputs.scanner_batch()))


def _target(tmp, torch, mat, rho, act, vs, scanner=None):
    """Measured sinogram: another seed, grey-matter activity x1.5, plus 5 %
    uniform randoms (Poisson); the model's background is their mean."""
    act_true = act.copy()
    act_true[mat == inputs.TISSUES["grey"][0]] *= 1.5
    sc = _scene(tmp, mat, rho, act_true, vs, seed=999, scanner=scanner)
    r = sc.run(mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED))
    sc.close()
    tot = (r.trues + r.scatter).astype(np.float64)
    bg = np.full(tot.size, 0.05 * tot.sum() / tot.size, np.float32)
    y = tot + np.random.default_rng(1).poisson(bg)
    return (torch.from_numpy(y.astype(np.float32)).cuda(), torch.from_numpy(bg).cuda())


def _loglik(tr, sc_, y, bg):
    lam = tr.astype(np.float64) + sc_ + bg
    return float(np.sum(np.where(y > 0, y * np.log(lam), 0.0) - lam))


OPTS = mcpet.RunOptions(lane_mode=mcpet.LANES_BALANCED, histories_per_lane=8)
# common random numbers across activity changes need the reference lane layout
# (a fixed set of lanes and RANECU streams per voxel)
CRN = mcpet.RunOptions(lane_mode=mcpet.LANES_REFERENCE)


def test_activity_gradient_is_exact_derivative_of_reweighted_events(tmp_path):
    torch = pytest.importorskip("torch")
    from mcpet import grad as G
    mat, rho, act, vs = _phantom()
    y, bg = _target(tmp_path, torch, mat, rho, act, vs)
    sc = _scene(tmp_path, mat, rho, act, vs)
    buf = torch.zeros(4_000_000 * 24, dtype=torch.uint8, device="cuda")
    r = G.grad(sc, y, bg, OPTS, event_buffer=buf)
    assert r.events > 20000
    ev = G.event_records(buf, r.events)
    tr = r.tallies["trues"].cpu().numpy()
    sc_ = r.tallies["scatter"].cpu().numpy()
    yn, bgn = y.cpu().numpy().astype(np.float64), bg.cpu().numpy().astype(np.float64)
    # the recorded events are exactly the tallied coincidences
    counts = np.bincount(ev["bin"], minlength=tr.size)
    np.testing.assert_array_equal(counts, (tr + sc_).astype(np.int64))
    assert abs(r.loglik - _loglik(tr, sc_, yn, bgn)) <= 1e-5 * abs(_loglik(tr, sc_, yn, bgn))
    ga = r.grad_activity.cpu().numpy()
    lam = tr.astype(np.float64) + sc_ + bgn
    rng = np.random.default_rng(3)
    vox = rng.choice(np.unique(ev["voxel"]), 64, replace=False)
    eps = 1e-3
    for v in vox:
        b = ev["bin"][ev["voxel"] == v]
        ub, k = np.unique(b, return_counts=True)
        def dl(sign):
            l2 = lam[ub] + sign * eps * k
            return np.sum(yn[ub] * np.log(l2) - l2) - np.sum(yn[ub] * np.log(lam[ub]) - lam[ub])
        fd = (dl(1) - dl(-1)) / (2 * eps * act.ravel()[v])
        scale = np.sum(k * np.abs(yn[ub] / lam[ub] - 1.0)) / act.ravel()[v]
        assert abs(ga[v] - fd) <= 1e-3 * abs(fd) + 1e-5 * scale, (v, ga[v], fd, scale)
    sc.close()


def test_replay_reproduces_events_and_accounting(tmp_path):
    torch = pytest.importorskip("torch")
    from mcpet import grad as G
    mat, rho, act, vs = _phantom()
    y, bg = _target(tmp_path, torch, mat, rho, act, vs)
    sc = _scene(tmp_path, mat, rho, act, vs)
    r = G.grad(sc, y, bg, OPTS)
    assert r.replayed + r.mismatches == r.events
    assert r.mismatches <= 1e-3 * r.events, (r.mismatches, r.events)
    # the forward of mcpet_grad is the plain transport (same seed, same tallies)
    plain = sc.run(OPTS)
    np.testing.assert_array_equal(r.tallies["trues"].cpu().numpy(), plain.trues)
    np.testing.assert_array_equal(r.tallies["scatter"].cpu().numpy(), plain.scatter)
    gs = r.grad_density_scale.cpu().numpy()
    assert np.isfinite(gs).all() and np.abs(gs).sum() > 0
    sc.close()


def _region_fd(tmp, torch, mat, rho, act, vs, y, bg, region, which, eps):
    vals = []
    for sgn in (1, -1):
        a2, r2 = act.copy(), rho.copy()
        if which == "activity":
            a2[region] *= 1 + sgn * eps
        else:
            r2[region] *= 1 + sgn * eps
        sc = _scene(tmp, mat, r2, a2, vs, scanner=COARSE)
        rr = sc.run(CRN)
        vals.append(_loglik(rr.trues, rr.scatter.astype(np.float64), y, bg))
        sc.close()
    return (vals[0] - vals[1]) / (2 * eps)


def test_region_derivatives_match_crn_finite_differences(tmp_path):
    torch = pytest.importorskip("torch")
    from mcpet import grad as G
    mat, rho, act, vs = _phantom(total_bq=5.0e7)
    y, bg = _target(tmp_path, torch, mat, rho, act, vs, scanner=COARSE)
    sc = _scene(tmp_path, mat, rho, act, vs, scanner=COARSE)
    r = G.grad(sc, y, bg, CRN)
    print("events", r.events, "bins", int(sc.config.n_bins))
    ga = r.grad_activity.cpu().numpy().reshape(mat.shape)
    gs = r.grad_density_scale.cpu().numpy().reshape(mat.shape)
    yn, bgn = y.cpu().numpy().astype(np.float64), bg.cpu().numpy().astype(np.float64)
    grey = mat == inputs.TISSUES["grey"][0]
    # d L / d eps with A_grey -> (1 + eps) A_grey
    adj_a = float(np.sum(ga[grey] * act[grey]))
    fd_a = _region_fd(tmp_path, torch, mat, rho, act, vs, yn, bgn, grey, "activity", 0.02)
    print("activity", adj_a, fd_a)
    # measured on B200: 3.0 % apart (finite-difference noise dominates at 5e7 decays)
    assert abs(adj_a - fd_a) <= 0.08 * abs(fd_a), (adj_a, fd_a)
    # d L / d eps with rho -> (1 + eps) rho on white matter below its maximum density
    wm = mat == inputs.TISSUES["white"][0]
    region = wm & (rho < 0.97 * rho[wm].max())
    adj_s = float(np.sum(gs[region]))
    fd_s = _region_fd(tmp_path, torch, mat, rho, act, vs, yn, bgn, region, "density", 0.02)
    print("density", adj_s, fd_s)
    # measured on B200: 2.2 % apart
    assert abs(adj_s - fd_s) <= 0.08 * abs(fd_s), (adj_s, fd_s)
    sc.close()


def test_autograd_binding(tmp_path):
    torch = pytest.importorskip("torch")
    from mcpet import grad as G
    mat, rho, act, vs = _phantom()
    y, bg = _target(tmp_path, torch, mat, rho, act, vs)
    sc = _scene(tmp_path, mat, rho, act, vs)
    a = torch.from_numpy(act.ravel().copy()).requires_grad_(True)
    s = torch.ones(act.size, dtype=torch.float32, requires_grad=True)
    L = G.poisson_loglik(a, s, sc, y, bg, OPTS)
    L.backward()
    r = G.grad(sc, y, bg, OPTS)
    assert abs(float(L) - r.loglik) <= 1e-6 * abs(r.loglik)
    ga, gs = r.grad_activity.cpu().numpy(), r.grad_density_scale.cpu().numpy()
    # same forward; gradients differ only by the order of float atomic sums
    np.testing.assert_allclose(a.grad.numpy(), ga, rtol=1e-4, atol=1e-5 * np.abs(ga).max())
    np.testing.assert_allclose(s.grad.numpy(), gs, rtol=1e-4, atol=1e-5 * np.abs(gs).max())
    sc.close()


needs_ref_prog = pytest.mark.needs_ref("libref_prog.so")


@needs_ref_prog
def test_region_derivatives_match_reference_eps_runs(tmp_path):
    """The same region derivatives against central differences of the
    reference's OWN CUDA runs of the perturbed input files (grey-matter
    activity and white-matter density scaled by 1 +- eps; same seed and
    lane layout, so common random numbers within the reference)."""
    torch = pytest.importorskip("torch")
    import refbind
    from mcpet import grad as G
    mat, rho, act, vs = _phantom(total_bq=5.0e7)
    y, bg = _target(tmp_path, torch, mat, rho, act, vs, scanner=COARSE)
    sc = _scene(tmp_path, mat, rho, act, vs, scanner=COARSE)
    r = G.grad(sc, y, bg, CRN)
    ga = r.grad_activity.cpu().numpy().reshape(mat.shape)
    gs = r.grad_density_scale.cpu().numpy().reshape(mat.shape)
    sc.close()
    yn, bgn = y.cpu().numpy().astype(np.float64), bg.cpu().numpy().astype(np.float64)
    grey = mat == inputs.TISSUES["grey"][0]
    wm = mat == inputs.TISSUES["white"][0]
    dens = wm & (rho < 0.97 * rho[wm].max())        # the majorant's maximum density stays put
    eps = 0.02

    def ref_fd(region, which):
        vals = []
        for sgn in (1, -1):
            a2, r2 = act.copy(), rho.copy()
            if which == "activity":
                a2[region] *= 1 + sgn * eps
            else:
                r2[region] *= 1 + sgn * eps
            inp = scenes.write_case(str(tmp_path), f"ref_{which}_{sgn}", mat, r2, a2, vs, tissues=HEAD_TISSUES,
                                    seed=12345, **COARSE)
            cfg = mcpet.read_config(inp)
            out = refbind.RefProg().run(inp, int(cfg.n_bins), mat.size, cfg.n_energy_bins, cwd=str(tmp_path))
            vals.append(_loglik(out["trues"], out["scatter"].astype(np.float64), yn, bgn))
        return (vals[0] - vals[1]) / (2 * eps)

    adj_a = float(np.sum(ga[grey] * act[grey]))
    fd_a = ref_fd(grey, "activity")
    adj_s = float(np.sum(gs[dens]))
    fd_s = ref_fd(dens, "density")
    print("activity", adj_a, fd_a, "density", adj_s, fd_s)
    # same tolerance as the finite differences of this build's own runs (measured there: 3.0 %, 2.2 %)
    assert abs(adj_a - fd_a) <= 0.08 * abs(fd_a), (adj_a, fd_a)
    assert abs(adj_s - fd_s) <= 0.08 * abs(fd_s), (adj_s, fd_s)
