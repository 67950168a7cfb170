"""Scene builders shared by the tests (small, seeded workloads)."""
from __future__ import annotations

import os

import numpy as np

import mcpet
from mcpet import inputs


def write_case(workdir: str, name: str, mat, rho, act, vs, tissues=("air", "soft"), gz: bool = False,
               extended: bool = False, **spec_kw):
    """Write a .vox + .in pair in workdir; returns the .in path.  extended:
    material tables continued to 1250 keV."""
    vox = inputs.write_vox(os.path.join(workdir, f"{name}.vox" + (".gz" if gz else "")), mat, rho, act, vs)
    kw = dict(inputs.scanner_small())
    kw.update(spec_kw)
    spec = inputs.spec_for(inputs.tissue_materials(list(tissues), extended), vox, **kw)
    return inputs.write_input(os.path.join(workdir, f"{name}.in"), spec)


def scene_from_arrays(workdir: str, mat, rho, act, vs, tissues=("air", "soft"), extended: bool = False,
                      **spec_kw) -> mcpet.Scene:
    kw = dict(inputs.scanner_small())
    kw.update(spec_kw)
    spec = inputs.spec_for(inputs.tissue_materials(list(tissues), extended), "unused.vox", **kw)
    cfg = inputs.config_from_spec(spec, workdir)
    return mcpet.Scene.from_arrays(cfg, mat, rho, act, vs)


def sample_scene(workdir: str, **spec_kw) -> mcpet.Scene:
    mat, rho, act, vs = inputs.sample_phantom()
    return scene_from_arrays(workdir, mat, rho, act, vs, **spec_kw)


def water_cube_scene(workdir: str, total_bq: float, **spec_kw) -> mcpet.Scene:
    mat, rho, act, vs = inputs.water_cube_phantom(total_bq)
    return scene_from_arrays(workdir, mat, rho, act, vs, **spec_kw)


def small_head_scene(workdir: str, total_bq: float = 2.0e5, shape=(16, 32, 32), voxel_cm=0.8, seed=7,
                     **spec_kw) -> mcpet.Scene:
    mat, rho, act, vs, used = inputs.head_phantom(shape=shape, voxel_cm=voxel_cm, seed=seed, total_bq=total_bq)
    kw = dict(inputs.scanner_for_head())
    kw.update(spec_kw)
    return scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, **kw)


def random_events(n: int, rng: np.random.Generator, box=(9.0, 9.0, 9.0), seeds=None, e_range=(300e3, 520e3)):
    """Random photon pairs leaving a box, for detector-model checks."""
    def dirs(k):
        z = rng.uniform(-1, 1, k)
        ph = rng.uniform(0, 2 * np.pi, k)
        s = np.sqrt(1 - z * z)
        return np.stack([s * np.cos(ph), s * np.sin(ph), z], 1).astype(np.float32)

    if seeds is None:
        seeds = np.stack([rng.integers(1, 2147483562, n), rng.integers(1, 2147483398, n)], 1).astype(np.int32)
    b = np.asarray(box, np.float32)
    d1 = dirs(n)
    # half of the pairs nearly back to back (as annihilation photons), half independent
    d2 = dirs(n)
    k = n // 2
    jitter = -d1[:k].astype(np.float64) + rng.normal(0, 0.02, (k, 3))
    d2[:k] = (jitter / np.linalg.norm(jitter, axis=1, keepdims=True)).astype(np.float32)
    p1 = (rng.uniform(0, 1, (n, 3)) * b).astype(np.float32)
    p2 = (rng.uniform(0, 1, (n, 3)) * b).astype(np.float32)
    p2[:k] = p1[:k]
    return dict(
        e2=rng.uniform(*e_range, n).astype(np.float32), e1=rng.uniform(*e_range, n).astype(np.float32),
        pos2=p2, pos1=p1, dir2=d2, dir1=d1, st2=rng.integers(0, 4, n).astype(np.int8),
        st1=rng.integers(0, 4, n).astype(np.int8), seeds=seeds.astype(np.int32),
    )


def chi2_per_dof(a: np.ndarray, b: np.ndarray, min_count: int = 5):
    """Two-sample chi^2/dof of independent Poisson histograms over bins whose
    combined count is at least min_count."""
    a = a.astype(np.float64).ravel()
    b = b.astype(np.float64).ravel()
    m = (a + b) >= min_count
    if m.sum() < 2:
        return float("nan"), int(m.sum())
    chi2 = ((a[m] - b[m]) ** 2 / (a[m] + b[m])).sum()
    return float(chi2 / m.sum()), int(m.sum())


def psf_records(raw) -> np.ndarray:
    arr = np.frombuffer(bytes(raw), dtype=mcpet.PSF_DTYPE) if not isinstance(raw, np.ndarray) or raw.dtype != \
        mcpet.PSF_DTYPE else raw
    return np.sort(arr, order=["emission_absvox", "emission_time_ps", "travel_time_ps"])
