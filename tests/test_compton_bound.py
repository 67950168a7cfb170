"""The bound of GCOa's rejection normaliser that balanced lanes use
(MfpRecord::s0_bound).

GCOa accepts a trial with probability S(E, theta) * T(tau) / S(E, pi)
(MCGPU-PET_kernel.cu:1390-1451), where S is the incoherent scattering
function of the analytical shell profiles and T <= 1.  Any constant not
below S(E, pi) gives the same accepted distribution; balanced lanes take,
for the energy bin of the photon, S at the upper edge of the next bin times
1 + 1e-5.  That is a bound only because S(E, pi) does not decrease with E:
checked here on the shell tables of every staged material, the 5-515 keV
tables and the ones continued to 1250 keV, in double precision on the bin
edges and in the single-precision arithmetic of the device formula at
random energies inside each bin."""
import numpy as np
import pytest

from mcpet import inputs
import scenes

MC2, INV_MC2, R2, IR2 = 510998.918, 1.956951306108245e-6, 1.4142135623731, 0.70710678118654502


def _s0(E, mat, t, dtype):
    """S(E, pi) for an array of energies, in the given precision."""
    E = np.asarray(E, dtype)
    s = np.zeros_like(E)
    for i in range(int(t["noscco"][mat])):
        u, f, j = (dtype(t[k][mat + i * 15]) for k in ("uico", "fco", "fj0"))
        aux = E * (E - u) * dtype(2)
        on = u < E
        pz = j * (aux - u * dtype(MC2)) / np.sqrt(np.where(on, aux + aux + u * u, dtype(1))) * dtype(INV_MC2)
        a = np.where(pz > 0, dtype(IR2) + pz * dtype(R2), dtype(IR2) - pz * dtype(R2))
        term = dtype(0.5) * np.exp(dtype(0.5) - a * a)
        term = np.where(pz > 0, dtype(1) - term, term)
        s = s + np.where(on, f * term, dtype(0))
    return s


@pytest.mark.parametrize("extended", [False, True], ids=["5-515keV", "5-1250keV"])
def test_normaliser_grows_with_energy_and_the_bin_bound_holds(workdir, extended):
    mat, rho, act, vs, used = inputs.head_phantom(shape=(12, 24, 24), voxel_cm=1.0, seed=5, total_bq=1e4)
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, tissues=used, extended=extended,
                                  **inputs.scanner_for_head())
    t, info = sc.export_tables(), sc.info
    e0, ide, ne = float(info.e0), float(info.inv_de), int(info.n_energy)
    edges = e0 + np.arange(ne + 2, dtype=np.float64) / ide
    rng = np.random.default_rng(11)
    checked = 0
    for m in range(15):
        if t["noscco"][m] <= 0:
            continue
        s = _s0(edges, m, t, np.float64)
        assert np.all(np.diff(s) >= -1e-12 * s[1:]), f"material {m}: S(E, pi) decreases"
        bound = s[2:] * (1.0 + 1e-5)                      # bin k: S at edge k + 2
        k = np.arange(ne)
        for _ in range(4):
            e = (e0 + (k + rng.random(ne)) / ide).astype(np.float32)
            kk = np.floor((e - np.float32(e0)) * np.float32(ide)).astype(np.int64)
            ok = (kk >= 0) & (kk < ne)
            s32 = _s0(e, m, t, np.float32).astype(np.float64)
            assert np.all(s32[ok] <= bound[kk[ok]]), f"material {m}: bound exceeded"
        checked += 1
    assert checked >= 2
    sc.close()
