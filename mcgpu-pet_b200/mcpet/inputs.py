"""Writers for the reference's input formats and seeded synthetic phantoms.

* ``write_input``  -- the sectioned ``.in`` file read by ``read_input``
  (MCGPU-PET.cu:866-1280) and by ``mcpet_config_read``;
* ``write_vox``    -- the penEasy/MCGPU-PET voxel file (``material density
  activity`` per line, x fastest; MCGPU-PET.cu:1381-1533), optionally gzip;
* phantoms for the workloads used by the tests and the benchmark.

Only the air and water PENELOPE tables ship with the reference, so tissues
are water-equivalent materials at tissue density, one material slot per
tissue (the reference accepts the same table file in several slots).
"""
from __future__ import annotations

import gzip
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MATERIAL_DIR = os.path.join(PKG_DIR, "data", "materials")


def material_path(name: str, extended: bool = False) -> str:
    """Path of a material table (``air`` / ``water``) staged by the build:
    the reference's 5-515 keV table, or (extended=True) the same table
    continued to 1250 keV by mcpet.tables (for prompt gammas)."""
    p = os.path.join(MATERIAL_DIR, f"{name}_5-1250keV.mcgpu.gz" if extended else f"{name}_5-515keV.mcgpu.gz")
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} missing: run __graft_entry__.build() to stage the material tables")
    return p


@dataclass
class InputSpec:
    """Every value of the reference input file, with the reference's units."""

    seed: int = 12345
    gpu_id: int = 0
    threads_per_block: int = 32
    density_factor: float = 1.0
    acquisition_s: float = 1.0
    mean_life_s: float = 1.0e12
    psf_file: str = "MCGPU_PET.psf"
    detector_center: Sequence[float] = (0.0, 0.0, 0.0)
    detector_height: float = 20.0
    detector_radius: float = -40.0          # negative: centred on the phantom
    psf_size: int = 1
    tally_type: int = 0                     # 0 both, 1 trues, 2 scatter
    tally_psf_sinogram: int = 2             # 0 both, 1 PSF, 2 sinogram
    material_dose: bool = False
    voxel_dose: bool = False
    dose_file: str = "mc-gpu_dose.dat"
    dose_roi: Sequence[int] = (1, 1, 1, 1, 1, 1)   # 1-based x_min, x_max, y_min, y_max, z_min, z_max
    energy_resolution: float = 0.12
    energy_low: float = 350000.0
    energy_high: float = 600000.0
    fov_z: float = 20.0
    n_rows: int = 15
    n_crystals: int = 336
    n_angles: int = 168
    n_radial: int = 147
    n_z_slices: int = 29
    image_res: int = 128
    n_energy_bins: int = 700
    max_ring_difference: int = 14
    span: int = 1
    voxel_file: str = "phantom.vox"
    material_files: List[str] = field(default_factory=list)
    prompt_gamma_energy: float = 0.0        # eV; > 0 adds the optional prompt-gamma section
    prompt_gamma_yield: float = 1.0         # per decay


def write_input(path: str, s: InputSpec) -> str:
    c = s.detector_center
    lines = [
        "# MCGPU-PET input file written by mcpet.inputs",
        "#[SECTION SIMULATION CONFIG v.2016-07-05]",
        f"{s.seed}                 # RANDOM SEED",
        f"{s.gpu_id}                 # GPU NUMBER",
        f"{s.threads_per_block}                # GPU THREADS PER CUDA BLOCK",
        f"{s.density_factor!r}               # FACTOR TO SCALE THE INPUT MATERIAL DENSITY",
        "",
        "#[SECTION SOURCE PET SCAN v.2017-03-14]",
        f"{s.acquisition_s!r}        # TOTAL PET SCAN ACQUISITION TIME [seconds]",
        f"{s.mean_life_s!r}        # ISOTOPE MEAN LIFE [s]",
        "   1   0.0     # TABLE MATERIAL NUMBER AND VOXEL ACTIVITY (unused: activity comes from the voxel file)",
        "   0   0.0",
        "",
        "#[SECTION PHASE SPACE FILE v.2016-07-05]",
        f" {s.psf_file}                # OUTPUT PHASE SPACE FILE FILE NAME",
        f" {c[0]!r} {c[1]!r} {c[2]!r} {s.detector_height!r} {s.detector_radius!r}   # CYLINDER CENTER, HEIGHT, RADIUS",
        f" {s.psf_size}                 # PHASE SPACE FILE SIZE",
        f" {s.tally_type}                 # REPORT TRUES (1), SCATTER (2), OR BOTH (0)",
        f" {s.tally_psf_sinogram}                 # REPORT PSF (1), SINOGRAM (2) or BOTH (0)",
        "",
        "#[SECTION DOSE DEPOSITION v.2012-12-12]",
        f"{'YES' if s.material_dose else 'NO'}            # TALLY MATERIAL DOSE? [YES/NO]",
        f"{'YES' if s.voxel_dose else 'NO'}            # TALLY 3D VOXEL DOSE? [YES/NO]",
        f"{s.dose_file}       # OUTPUT VOXEL DOSE FILE NAME",
        f"  {s.dose_roi[0]}  {s.dose_roi[1]}                # VOXEL DOSE ROI: X-index min max",
        f"  {s.dose_roi[2]}  {s.dose_roi[3]}                # VOXEL DOSE ROI: Y-index min max",
        f"  {s.dose_roi[4]}  {s.dose_roi[5]}                # VOXEL DOSE ROI: Z-index min max",
        "",
        "#[SECTION ENERGY PARAMETERS v.2019-04-25]",
        f"{s.energy_resolution!r}       # ENERGY RESOLUTION OF THE CRYSTALS",
        f"{s.energy_low!r}      # ENERGY WINDOW LOW (eV)",
        f"{s.energy_high!r}      # ENERGY WINDOW HIGH (eV)",
        "",
        "#[SECTION SINOGRAM PARAMETERS v.2019-04-25]",
        f"{s.fov_z!r}   # AXIAL FIELD OF VIEW (FOVz) in cm",
        f"{s.n_rows}    # NUMBER OF ROWS",
        f"{s.n_crystals}    # TOTAL NUMBER OF CRYSTALS",
        f"{s.n_angles}    # NUMBER OF ANGULAR BINS",
        f"{s.n_radial}    # NUMBER OF RADIAL BINS",
        f"{s.n_z_slices}    # NUMBER OF Z SLICES",
        f"{s.image_res}    # IMAGE RESOLUTION",
        f"{s.n_energy_bins}    # NUMBER OF ENERGY BINS",
        f"{s.max_ring_difference}    # MAXIMUM RING DIFFERENCE",
        f"{s.span}    # SPAN",
        "",
    ]
    if s.prompt_gamma_energy > 0:
        # read by this library only: the reference skips it while it looks for
        # the voxel-file section
        lines += [
            "#[SECTION PROMPT GAMMA EMISSION v.2026-12-01]",
            f"{s.prompt_gamma_energy!r}     # PROMPT GAMMA ENERGY (eV)",
            f"{s.prompt_gamma_yield!r}      # PROMPT GAMMA YIELD PER DECAY",
            "",
        ]
    lines += [
        "#[SECTION VOXELIZED GEOMETRY FILE v.2009-11-30]",
        f"{s.voxel_file}      # VOXEL GEOMETRY FILE",
        "",
        "#[SECTION MATERIAL FILE LIST v.2009-11-30]",
    ]
    for i, m in enumerate(s.material_files):
        lines.append(f"{m}     # {i + 1}")
    lines.append("#")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def write_vox(path: str, material: np.ndarray, density: np.ndarray, activity: np.ndarray,
              voxel_size_cm: Sequence[float]) -> str:
    """Voxel file; arrays shaped (nz, ny, nx), material 1-based."""
    nz, ny, nx = material.shape
    vs = voxel_size_cm
    head = ("[SECTION VOXELS HEADER v.2008-04-13]\n"
            f"{nx} {ny} {nz}   No. OF VOXELS IN X,Y,Z\n"
            f"{vs[0]!r} {vs[1]!r} {vs[2]!r}   VOXEL SIZE (cm) ALONG X,Y,Z\n"
            " 1                  COLUMN NUMBER WHERE MATERIAL ID IS LOCATED\n"
            " 2                  COLUMN NUMBER WHERE THE MASS DENSITY IS LOCATED\n"
            " 0                  BLANK LINES AT END OF X,Y-CYCLES (1=YES,0=NO)\n"
            "[END OF VXH SECTION]  # MCGPU-PET voxel format: Material  Density  Activity\n")
    m = material.reshape(-1)
    d = density.astype(np.float32).reshape(-1)
    a = activity.astype(np.float32).reshape(-1)
    body = "\n".join(f"{int(mi)} {float(di)!r} {float(ai)!r}" for mi, di, ai in zip(m, d, a))
    data = (head + body + "\n").encode()
    if path.endswith(".gz"):
        with gzip.open(path, "wb", compresslevel=1) as f:
            f.write(data)
    else:
        with open(path, "wb") as f:
            f.write(data)
    return path


# --------------------------------------------------------------------------
# Phantoms.  Arrays are (nz, ny, nx), material 1-based.

TISSUES = {   # name: (material slot, table, density g/cm^3)
    "air": (1, "air", 0.0012),
    "soft": (2, "water", 1.03),
    "grey": (3, "water", 1.04),
    "white": (4, "water", 1.04),
    "bone": (5, "water", 1.85),
    "fat": (6, "water", 0.95),
    "blood": (7, "water", 1.06),
    "csf": (8, "water", 1.0),
    "lung": (9, "water", 0.3),
    "organ": (10, "water", 1.05),
}


def tissue_materials(names: Sequence[str], extended: bool = False) -> List[str]:
    """Material file list (slot order) for the given tissues (extended:
    tables reaching 1250 keV)."""
    slots = {}
    for n in names:
        slot, table, _ = TISSUES[n]
        slots[slot] = material_path(table, extended)
    top = max(slots)
    return [slots.get(i, material_path("water", extended)) for i in range(1, top + 1)]


def sample_phantom():
    """9x9x9 1-cm grid: 5^3 water cube (50 Bq/voxel) in 2-voxel air margin,
    1000/2000/3000 Bq inserts at (3,3,4), (5,3,4), (5,5,4) and an air cavity
    at (3,5,4) -- the reference's sample geometry."""
    n = 9
    mat = np.ones((n, n, n), np.int32)
    rho = np.full((n, n, n), 0.0012, np.float32)
    act = np.zeros((n, n, n), np.float32)
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    inside = (i >= 2) & (j >= 2) & (k >= 2) & (i < n - 2) & (j < n - 2) & (k < n - 2)
    mat[inside] = 2
    rho[inside] = 1.0
    act[inside] = 50.0
    for (x, y, z), a in (((3, 3, 4), 1000.0), ((5, 3, 4), 2000.0), ((5, 5, 4), 3000.0)):
        act[z, y, x] = a
    mat[4, 5, 3] = 1
    rho[4, 5, 3] = 0.0012
    act[4, 5, 3] = 0.0
    return mat, rho, act, (1.0, 1.0, 1.0)


def water_cube_phantom(total_bq: float = 1.0e7):
    """9^3 1-cm water voxels, uniform background b and three voxels at 100 b in
    the central plane, sum of activity = total_bq (1e7 emissions in 1 s)."""
    n = 9
    mat = np.full((n, n, n), 2, np.int32)
    rho = np.ones((n, n, n), np.float32)
    b = total_bq / 1026.0
    act = np.full((n, n, n), b, np.float32)
    for x, y in ((3, 3), (5, 3), (5, 5)):
        act[4, y, x] = 100.0 * b
    return mat, rho, act, (1.0, 1.0, 1.0)


def _ellipsoid(shape, center, radii, vs):
    nz, ny, nx = shape
    z = (np.arange(nz) + 0.5) * vs[2]
    y = (np.arange(ny) + 0.5) * vs[1]
    x = (np.arange(nx) + 0.5) * vs[0]
    X = (((x - center[0]) / radii[0]) ** 2)[None, None, :]
    Y = (((y - center[1]) / radii[1]) ** 2)[None, :, None]
    Z = (((z - center[2]) / radii[2]) ** 2)[:, None, None]
    return (X + Y + Z) <= 1.0


def head_phantom(shape=(64, 128, 128), voxel_cm=0.2, seed: int = 2024, total_bq: float = 1.0e9):
    """Seeded nested random ellipsoids in the shape of a head: skin/soft
    tissue, fat layer, skull, grey-matter cortex, white matter, ventricles
    (CSF), a few blood pools.  FDG-like activity ratios grey 4 : white 1 :
    soft 0.5 : bone 0.2 : air 0 (fat 0.5, blood 1, CSF 0), scaled to total_bq."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    vs = (voxel_cm, voxel_cm, voxel_cm)
    size = np.array([nx * vs[0], ny * vs[1], nz * vs[2]])
    c = size / 2 + rng.uniform(-0.3, 0.3, 3)
    r_head = np.array([0.44 * size[0], 0.47 * size[1], 0.55 * size[2]]) * rng.uniform(0.97, 1.0, 3)
    labels = np.zeros(shape, np.int8)    # 0 air
    order = []

    def paint(mask, name):
        labels[mask] = list(TISSUES).index(name)

    paint(_ellipsoid(shape, c, r_head, vs), "soft")
    paint(_ellipsoid(shape, c, r_head - 0.35, vs), "fat")
    paint(_ellipsoid(shape, c, r_head - 0.6, vs), "bone")
    paint(_ellipsoid(shape, c + [0, 0, 0.2], r_head - 1.3, vs), "grey")
    paint(_ellipsoid(shape, c + [0, 0, 0.3], r_head - 2.0 - rng.uniform(0, 0.3, 3), vs), "white")
    for s in (-1, 1):
        vc = c + np.array([s * rng.uniform(0.8, 1.3), rng.uniform(-0.5, 0.5), rng.uniform(0.5, 1.5)])
        paint(_ellipsoid(shape, vc, rng.uniform([0.4, 1.5, 0.6], [0.7, 2.5, 1.2]), vs), "csf")
    for _ in range(6):
        bc = c + rng.uniform(-1, 1, 3) * (r_head - 2.5)
        paint(_ellipsoid(shape, bc, rng.uniform(0.2, 0.5, 3), vs), "blood")
    names = list(TISSUES)
    ratio = {"air": 0.0, "soft": 0.5, "grey": 4.0, "white": 1.0, "bone": 0.2, "fat": 0.5, "blood": 1.0, "csf": 0.0,
             "lung": 0.2, "organ": 1.0}
    mat = np.zeros(shape, np.int32)
    rho = np.zeros(shape, np.float32)
    act = np.zeros(shape, np.float64)
    for li, name in enumerate(names):
        m = labels == li
        if not m.any():
            continue
        slot, _, d = TISSUES[name]
        mat[m] = slot
        rho[m] = d
        act[m] = ratio[name]
    act *= total_bq / act.sum()
    used = [n for i, n in enumerate(names) if (labels == i).any()]
    return mat, rho, act.astype(np.float32), vs, used


def scanner_for_head() -> dict:
    """41 cm radius, 64 rings x 4 mm, 256x256 sinograms, span 1, MRD 63."""
    return dict(detector_radius=-41.0, detector_height=25.6, fov_z=25.6, n_rows=64, n_crystals=512, n_angles=256,
                n_radial=256, n_z_slices=127, max_ring_difference=63, span=1)


HEAD_WORKLOAD_SEED = 2024


def head_workload(total_bq: float = 1.0e9, scanner: str = "head"):
    """The head workload: 128x128x64 voxels of 2 mm (seed 2024), FDG-like
    activity summing to total_bq, seen by the 64-ring scanner (256 x 256 x
    8065 span-1 sinograms) with RANECU seed 12345.  scanner="head32" keeps the
    phantom and ring pitch with 32 rings and 128 x 256 x 1985 sinograms (a
    smaller case for profiler captures).  Returns (material, density,
    activity, voxel_size, tissues, scanner keywords of spec_for)."""
    mat, rho, act, vs, used = head_phantom(shape=(64, 128, 128), voxel_cm=0.2, seed=HEAD_WORKLOAD_SEED,
                                           total_bq=total_bq)
    scan = scanner_for_head()
    if scanner == "head32":
        scan.update(n_rows=32, n_z_slices=63, max_ring_difference=31, n_radial=128, n_angles=256, n_crystals=512,
                    fov_z=12.8, detector_height=12.8)
    elif scanner != "head":
        raise ValueError(scanner)
    scan["seed"] = 12345
    return mat, rho, act, vs, used, scan


def scanner_batch() -> dict:
    """41 cm radius, 32 rings x 4 mm, 128x128 sinograms (256 crystals), span 1,
    MRD 31: the scanner of the batched many-phantom workload."""
    return dict(detector_radius=-41.0, detector_height=12.8, fov_z=12.8, n_rows=32, n_crystals=256, n_angles=128,
                n_radial=128, n_z_slices=63, max_ring_difference=31, span=1)


def batch_phantoms(n: int, emissions_each: float, seed: int = 3):
    """n seeded head-like phantoms of m^3 voxels, m drawn in [32, 192], voxel
    pitch in [2, 4] mm (at most 40 cm across), each with emissions_each
    decays.  Yields (material, density, activity, voxel_size, tissues)."""
    rng = np.random.default_rng(seed)
    for k in range(n):
        m = int(rng.integers(32, 193))
        vox = float(min(rng.uniform(0.2, 0.4), 40.0 / m))
        mat, rho, act, vs, used = head_phantom(shape=(m, m, m), voxel_cm=vox, seed=seed * 1000 + k,
                                               total_bq=emissions_each)
        yield mat, rho, act, vs, used


def body_phantom(shape=(400, 256, 256), voxel_cm=0.2, seed: int = 2025, total_bq: float = 5.0e9):
    """Seeded whole-body phantom of nested ellipsoids (z is the body axis,
    head at high z): torso of soft tissue under a fat layer, two lungs
    (rho 0.3), a spine and a rib shell of bone (1.85), heart blood pool,
    a hot organ (8x background), and a head with skull, grey and white matter
    and CSF.  Activity ratios: organ 8, grey 4, white 1, heart blood 2,
    soft/fat 1, bone 0.3, lung 0.2, CSF and air 0; scaled to total_bq.
    Returns (material, density, activity, voxel_size, tissues) like
    head_phantom."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    vs = (voxel_cm, voxel_cm, voxel_cm)
    L = np.array([nx * vs[0], ny * vs[1], nz * vs[2]])
    jit = lambda a: a * rng.uniform(0.95, 1.05)
    labels = np.zeros(shape, np.int8)
    names = list(TISSUES)

    def paint(center, radii, name):
        labels[_ellipsoid(shape, center, radii, vs)] = names.index(name)

    cx, cy = L[0] / 2, L[1] / 2
    # torso over the lower 72 % of the length, head above a short neck
    zt = 0.36 * L[2]
    rt = np.array([jit(0.42 * L[0]), jit(0.30 * L[1]), 0.36 * L[2]])
    paint((cx, cy, zt), rt, "fat")
    paint((cx, cy, zt), rt - [1.2, 1.2, 0.5], "soft")
    paint((cx, cy, zt + 0.12 * L[2]), (rt[0] - 2.0, rt[1] - 2.0, 0.16 * L[2]), "bone")     # rib shell
    paint((cx, cy, zt + 0.12 * L[2]), (rt[0] - 2.8, rt[1] - 2.8, 0.155 * L[2]), "soft")
    for sgn in (-1, 1):                                                                 # lungs
        paint((cx + sgn * jit(0.19 * L[0]), cy, zt + 0.14 * L[2]), (jit(0.13 * L[0]), jit(0.19 * L[1]), 0.12 * L[2]),
              "lung")
    paint((cx + jit(0.04 * L[0]), cy + 0.03 * L[1], zt + 0.08 * L[2]), (jit(0.07 * L[0]),) * 2 + (0.05 * L[2],),
          "blood")                                                                      # heart
    paint((cx - jit(0.12 * L[0]), cy, zt - 0.04 * L[2]), (jit(0.14 * L[0]), jit(0.15 * L[1]), 0.06 * L[2]),
          "organ")                                                                      # hot organ
    paint((cx, cy - 0.21 * L[1], zt), (0.03 * L[0], 0.035 * L[1], 0.34 * L[2]), "bone")  # spine
    zh = 0.87 * L[2]
    rh = np.array([jit(0.31 * L[0]), jit(0.36 * L[1]), 0.11 * L[2]])
    paint((cx, cy, 0.75 * L[2]), (0.12 * L[0], 0.12 * L[1], 0.05 * L[2]), "soft")      # neck
    paint((cx, cy, zh), rh, "soft")
    paint((cx, cy, zh), rh - 0.4, "bone")
    paint((cx, cy, zh + 0.2), rh - 1.0, "grey")
    paint((cx, cy, zh + 0.3), rh - 1.8, "white")
    for sgn in (-1, 1):
        paint((cx + sgn * 1.0, cy, zh + 0.5), (0.6, 2.0, 0.9), "csf")
    ratio = {"air": 0.0, "soft": 1.0, "grey": 4.0, "white": 1.0, "bone": 0.3, "fat": 1.0, "blood": 2.0, "csf": 0.0,
             "lung": 0.2, "organ": 8.0}
    mat = np.zeros(shape, np.int32)
    rho = np.zeros(shape, np.float32)
    act = np.zeros(shape, np.float64)
    for li, name in enumerate(names):
        m = labels == li
        if not m.any():
            continue
        slot, _, d = TISSUES[name]
        mat[m] = slot
        rho[m] = d
        act[m] = ratio[name]
    act *= total_bq / act.sum()
    used = [n for i, n in enumerate(names) if (labels == i).any()]
    return mat, rho, act.astype(np.float32), vs, used


def scanner_long_axial(max_ring_difference: int = 255, span: int = 11, n_angles: int = 384,
                       n_radial: int = 384) -> dict:
    """1 m axial, 39 cm radius, 256 rings x 4 mm, 768 crystals, span 11,
    MRD 255 (12333 sinogram planes of 384 x 384 at full size)."""
    return dict(detector_radius=-39.0, detector_height=102.4, fov_z=102.4, n_rows=256, n_crystals=768,
                n_angles=n_angles, n_radial=n_radial, n_z_slices=511, max_ring_difference=max_ring_difference,
                span=span)


def bed_centers(phantom_size_cm, n_beds: int, step_cm: float):
    """Detector centres (x, y, z) of n_beds bed positions along the body
    axis, step_cm apart and symmetric about the phantom's centre."""
    cx, cy, cz = (0.5 * phantom_size_cm[0], 0.5 * phantom_size_cm[1], 0.5 * phantom_size_cm[2])
    return [(cx, cy, cz + (k - 0.5 * (n_beds - 1)) * step_cm) for k in range(n_beds)]


def scanner_small() -> dict:
    """40 cm radius, 20 cm axial, 15 rings, 147 radial x 168 angles, span 1."""
    return dict(detector_radius=-40.0, detector_height=20.0, fov_z=20.0, n_rows=15, n_crystals=336, n_angles=168,
                n_radial=147, n_z_slices=29, max_ring_difference=14, span=1)


def spec_for(mat_files: List[str], voxel_file: str, **kw) -> InputSpec:
    s = InputSpec(voxel_file=voxel_file, material_files=mat_files)
    for k, v in kw.items():
        if not hasattr(s, k):
            raise AttributeError(k)
        setattr(s, k, v)
    return s


def config_from_spec(spec: InputSpec, workdir: str):
    """Parse an InputSpec through the C ABI (through a temporary .in file of
    its own in workdir, so that processes sharing workdir do not collide)."""
    import tempfile
    from .scene import read_config
    fd, p = tempfile.mkstemp(prefix="_spec_", suffix=".in", dir=workdir)
    os.close(fd)
    try:
        write_input(p, spec)
        return read_config(p)
    finally:
        os.unlink(p)
