"""Gradient of the sinogram Poisson log-likelihood (mcpet_grad).

Checks:
* the activity gradient is the exact derivative of the log-likelihood of the
  recorded events reweighted by A'_v / A_v (central difference in float64 over
  the event records, eps = 1e-3);
* replays reproduce the recorded bins (mismatch fraction below 1e-3);
* on the head phantom of the gradient configuration (128x128x64, 2e8
  decays), activity and density-scale derivatives over regions agree with
  central finite differences of full forward runs using common random
  numbers (same seed and lanes) -- of this library and of the reference's
  own CUDA build -- to 2 %, and over 64 random 16^3-voxel neighbourhoods to
  the tolerances written in the test;
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


# ---------------------------------------------------------------- C4 head
# The head phantom of the gradient configuration (128x128x64 voxels of 2 mm,
# 2e8 decays) with densities drawn below each tissue's maximum, so that a
# density perturbation keeps the Woodcock majorant (built from the maximum
# density of each material, MCGPU-PET.cu:1682-1684) and with it the common
# random numbers.  Finite differences of the likelihood measure the
# derivative only where a bin holds many counts (adding one event changes a
# bin's term by y ln(1 + 1/lambda), not y/lambda), so the sinogram is the
# coarse 29 K-bin one (~180 counts per bin at 2e8 decays); single voxels hold
# ~24 detected events, far too few for a finite difference at 2 %, hence
# regions and 16^3-voxel neighbourhoods.
C4_DECAYS = 2.0e8
C4_SEEDS = (12345, 777)
C4_EPS = 0.03


@pytest.fixture(scope="module")
def c4(tmp_path_factory):
    torch = pytest.importorskip("torch")
    from mcpet import grad as G
    tmp = tmp_path_factory.mktemp("c4")
    mat, rho, act, vs, _ = inputs.head_phantom(shape=(64, 128, 128), voxel_cm=0.2, seed=2024, total_bq=C4_DECAYS)
    rho = (rho * np.random.default_rng(5).uniform(0.9, 1.0, rho.shape)).astype(np.float32)
    y, bg = _target(tmp, torch, mat, rho, act, vs, scanner=COARSE)
    yn, bgn = y.cpu().numpy().astype(np.float64), bg.cpu().numpy().astype(np.float64)
    adj = {}
    for seed in C4_SEEDS:
        sc = _scene(tmp, mat, rho, act, vs, seed=seed, scanner=COARSE)
        r = G.grad(sc, y, bg, CRN)
        assert r.mismatches <= 1e-3 * r.events
        adj[seed] = (r.grad_activity.cpu().numpy().reshape(mat.shape),
                     r.grad_density_scale.cpu().numpy().reshape(mat.shape))
        sc.close()
    grey = mat == inputs.TISSUES["grey"][0]
    wm = mat == inputs.TISSUES["white"][0]
    dens = wm & (rho < 0.97 * rho[wm].max())   # rho (1 + eps) stays below the maximum density
    return dict(tmp=str(tmp), mat=mat, rho=rho, act=act, vs=vs, y=yn, bg=bgn, adj=adj, grey=grey, dens=dens)


def _crn_fd(c, region, which, seed, eps=C4_EPS):
    """Central difference of L with common random numbers (reference lanes,
    same seed): activity or density scaled by 1 +- eps on the region."""
    vals = []
    for sgn in (1, -1):
        a2, r2 = c["act"].copy(), c["rho"].copy()
        if which == "activity":
            a2[region] *= 1 + sgn * eps
        else:
            r2[region] *= 1 + sgn * eps
        sc = _scene(c["tmp"], c["mat"], r2, a2, c["vs"], seed=seed, scanner=COARSE)
        rr = sc.run(CRN)
        vals.append(_loglik(rr.trues, rr.scatter.astype(np.float64), c["y"], c["bg"]))
        sc.close()
    return (vals[0] - vals[1]) / (2 * eps)


def _adjoint(c, region, which, seed):
    ga, gs = c["adj"][seed]
    return float(np.sum(ga[region] * c["act"][region])) if which == "activity" else float(np.sum(gs[region]))


@pytest.mark.parametrize("which", ["activity", "density"])
def test_region_derivatives_match_crn_finite_differences(c4, which):
    """dL/d eps with A_grey -> (1 + eps) A_grey, and with rho -> (1 + eps) rho
    on white matter below its maximum density: adjoint vs central finite
    differences of full forward runs with common random numbers, on two
    seeds.  Measured on B200 at 2e8 decays: activity -0.8 % and -0.8 %,
    density +1.5 % and +0.8 % (eps 0.03)."""
    region = c4["grey"] if which == "activity" else c4["dens"]
    adj = [_adjoint(c4, region, which, s) for s in C4_SEEDS]
    fd = [_crn_fd(c4, region, which, s) for s in C4_SEEDS]
    rel = (sum(adj) - sum(fd)) / abs(sum(fd))
    print(which, adj, fd, f"{rel:+.4f}")
    assert abs(rel) <= 0.02, (which, adj, fd)


def test_neighbourhood_activity_derivatives_match_crn_finite_differences(c4):
    """64 seeded random 16^3-voxel neighbourhoods (centres drawn by activity):
    the adjoint's activity derivative of each against its own CRN central
    difference (eps 0.05).  Measured on B200: correlation 0.9986, slope
    1.013, summed derivative within 1.4 %, median difference 1.6 %."""
    mat, act = c4["mat"], c4["act"]
    rng = np.random.default_rng(64)
    w = act.ravel().astype(np.float64)
    centres = rng.choice(act.size, 64, replace=False, p=w / w.sum())
    seed = C4_SEEDS[0]
    adj, fd = [], []
    for c in centres:
        z, y, x = np.unravel_index(c, mat.shape)
        region = np.zeros(mat.shape, bool)
        region[max(z - 8, 0):z + 8, max(y - 8, 0):y + 8, max(x - 8, 0):x + 8] = True
        region &= act > 0
        adj.append(_adjoint(c4, region, "activity", seed))
        fd.append(_crn_fd(c4, region, "activity", seed, eps=0.05))
    adj, fd = np.array(adj), np.array(fd)
    corr = np.corrcoef(adj, fd)[0, 1]
    slope = float(np.sum(adj * fd) / np.sum(adj * adj))
    rel = np.abs(adj - fd) / np.abs(fd)
    print("neighbourhoods: corr", corr, "slope", slope, "sum", adj.sum(), fd.sum(), "median", np.median(rel))
    assert corr >= 0.99 and abs(slope - 1.0) <= 0.03
    assert abs(adj.sum() - fd.sum()) <= 0.025 * abs(fd.sum())
    assert np.median(rel) <= 0.03 and np.mean(rel <= 0.05) >= 0.8


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
@pytest.mark.parametrize("which", ["activity", "density"])
def test_region_derivatives_match_reference_eps_runs(c4, which):
    """The same region derivatives against central differences of the
    reference's OWN CUDA runs of the perturbed input files (grey-matter
    activity and white-matter density scaled by 1 +- eps; same seed and lane
    layout as the adjoint's forward, so common random numbers within the
    reference), on the same two seeds."""
    import refbind
    region = c4["grey"] if which == "activity" else c4["dens"]
    mat, vs = c4["mat"], c4["vs"]

    def ref_fd(seed):
        vals = []
        for sgn in (1, -1):
            a2, r2 = c4["act"].copy(), c4["rho"].copy()
            if which == "activity":
                a2[region] *= 1 + sgn * C4_EPS
            else:
                r2[region] *= 1 + sgn * C4_EPS
            inp = scenes.write_case(c4["tmp"], f"ref_{which}_{seed}_{sgn}", mat, r2, a2, vs, tissues=HEAD_TISSUES,
                                    seed=seed, **COARSE)
            cfg = mcpet.read_config(inp)
            out = refbind.RefProg().run(inp, int(cfg.n_bins), mat.size, cfg.n_energy_bins, cwd=c4["tmp"])
            vals.append(_loglik(out["trues"], out["scatter"].astype(np.float64), c4["y"], c4["bg"]))
        return (vals[0] - vals[1]) / (2 * C4_EPS)

    adj = [_adjoint(c4, region, which, s) for s in C4_SEEDS]
    fd = [ref_fd(s) for s in C4_SEEDS]
    rel = (sum(adj) - sum(fd)) / abs(sum(fd))
    print(which, "reference", adj, fd, f"{rel:+.4f}")
    assert abs(rel) <= 0.02, (which, adj, fd)
