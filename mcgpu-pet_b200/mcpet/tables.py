"""Material tables extended above 515 keV, in the reference's own format.

The reference ships PENELOPE-2006 tables for air and water from 5 keV to
514.95 keV in 50 eV steps (``*_5-515keV.mcgpu.gz``; format read by
load_material, MCGPU-PET.cu:1565-1831) and only emits 511 keV photons.  A
prompt gamma (e.g. 1157 keV) needs the mean free paths up to at least its
energy.  ``extend_table`` writes a table with the same header, the same
Rayleigh (RITA) and Compton-shell sections and the same energy grid, whose
rows up to 514.95 keV are the source rows copied verbatim, continued to
``e_max`` by these models:

* Compton: the tabulated mean free path at the last row scaled by the ratio
  of Klein-Nishina total cross sections per electron, sigma_KN(E_last) /
  sigma_KN(E).  Above 500 keV the binding corrections of the incoherent
  cross section are far below 0.1 %, so the ratio carries the shape.
* Rayleigh and photoelectric: power laws mu ~ E^-n whose exponents are
  least-squares fits of log(mfp) against log(E) over the last 10 % of the
  tabulated rows (about 2 for coherent scattering in the form-factor regime,
  about 2.7 for photoabsorption in water near 500 keV).  Both together are
  below 0.5 % of the attenuation above 500 keV.
* Total: 1 / (sum of the three inverse mean free paths).  Pair production,
  which the transport does not sample, is below 0.05 % of the attenuation
  under 1.26 MeV and is left out.
* Rayleigh "max cumulative probability of F^2": the last tabulated value
  (0.99999997 for water), held constant; the true value rises towards 1
  by less than 3e-8.

The energy grid keeps its step; the reference's limit of 25005 rows
(MAX_ENERGYBINS_RAYLEIGH, MCGPU-PET.h:99) allows up to 1255.2 keV.
"""
from __future__ import annotations

import gzip
import math
import os
from typing import List, Tuple

import numpy as np

ELECTRON_REST_EV = 510998.95
MAX_ROWS = 25005


def klein_nishina_sigma(e_ev: np.ndarray) -> np.ndarray:
    """Klein-Nishina total cross section per electron, in units of
    2 pi r_e^2 (only ratios are used)."""
    k = np.asarray(e_ev, np.float64) / ELECTRON_REST_EV
    l2k = np.log1p(2.0 * k)
    return ((1.0 + k) / k ** 2 * (2.0 * (1.0 + k) / (1.0 + 2.0 * k) - l2k / k) + l2k / (2.0 * k)
            - (1.0 + 3.0 * k) / (1.0 + 2.0 * k) ** 2)


def _open(path: str, mode: str):
    return gzip.open(path, mode) if path.endswith(".gz") else open(path, mode)


def read_table(path: str) -> Tuple[List[str], List[str], np.ndarray, List[str]]:
    """(header lines, data row lines, data as float64 [n, 6], tail lines
    from the Rayleigh section on)."""
    with _open(path, "rt") as f:
        lines = f.read().split("\n")
    i = next(k for k, ln in enumerate(lines) if ln.startswith("#[NUMBER OF DATA VALUES]"))
    n = int(lines[i + 1].lstrip("#").split()[0])
    j = next(k for k, ln in enumerate(lines) if ln.startswith("#[MEAN FREE PATHS"))
    j += 1                                   # the column-title line
    header = lines[: j + 1]
    rows = lines[j + 1: j + 1 + n]
    tail = lines[j + 1 + n:]
    data = np.array([[float(x) for x in r.split()[:6]] for r in rows], np.float64)
    if data.shape != (n, 6):
        raise ValueError(f"{path}: expected {n} rows of 6 values")
    return header, rows, data, tail


def _power_exponent(e: np.ndarray, mfp: np.ndarray) -> float:
    """n of mfp ~ E^n fitted over the given rows (least squares in log-log)."""
    x, y = np.log(e), np.log(mfp)
    return float(np.polyfit(x, y, 1)[0])


def extended_rows(data: np.ndarray, e_max: float) -> np.ndarray:
    """Rows (E, Rayleigh, Compton, photoelectric, total, pmax) continuing the
    table's energy grid from its last row up to e_max (inclusive)."""
    e = data[:, 0]
    de = e[1] - e[0]
    n_old = len(e)
    n_new = int(math.floor((e_max - e[-1]) / de + 1e-9))
    if n_old + n_new > MAX_ROWS:
        raise ValueError(f"{n_old + n_new} rows exceed the format's {MAX_ROWS}")
    if n_new <= 0:
        return np.zeros((0, 6))
    tail = slice(n_old - max(n_old // 10, 2), n_old)
    n_ray = _power_exponent(e[tail], data[tail, 1])
    n_pho = _power_exponent(e[tail], data[tail, 3])
    e_last = e[-1]
    en = e_last + de * np.arange(1, n_new + 1, dtype=np.float64)
    ray = data[-1, 1] * (en / e_last) ** n_ray
    com = data[-1, 2] * klein_nishina_sigma(e_last) / klein_nishina_sigma(en)
    pho = data[-1, 3] * (en / e_last) ** n_pho
    tot = 1.0 / (1.0 / ray + 1.0 / com + 1.0 / pho)
    pmax = np.full(n_new, data[-1, 5])
    return np.stack([en, ray, com, pho, tot, pmax], 1)


def extend_table(src: str, dst: str, e_max: float = 1.25e6) -> int:
    """Write dst: src's table continued to e_max (eV).  Returns the rows."""
    header, rows, data, tail = read_table(src)
    new = extended_rows(data, e_max)
    n = len(rows) + len(new)
    out = []
    for ln in header:
        out.append(ln)
    k = next(i for i, ln in enumerate(out) if ln.startswith("#[NUMBER OF DATA VALUES]"))
    out[k + 1] = f"#  {n}"
    out.extend(rows)
    for r in new:
        out.append("  " + "  ".join(f"{v:.10E}" for v in r))
    out.extend(tail)
    os.makedirs(os.path.dirname(os.path.abspath(dst)), exist_ok=True)
    with _open(dst, "wt") as f:
        f.write("\n".join(out))
    return n


def extended_name(table: str, e_max: float = 1.25e6) -> str:
    return f"{table}_5-{int(round(e_max / 1e3))}keV.mcgpu.gz"
