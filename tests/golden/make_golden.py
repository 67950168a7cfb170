"""Generate the golden fixtures of tests/golden from the REFERENCE's own code.

Run in a tree where oracle/ref/Makefile has built oracle/_ref (the reference
sources compiled as a host library, libref_cpu.so, and its loaders,
libref_prog.so).  Every value stored here is produced by the reference code:

* rng_streams.npz   init_PRNG jump + first ranecu/ranecu_double draws
                    (MCGPU-PET_kernel.cu:925-1083) for seed 12345;
* detector_kat.npz  tally_Sinogram (MCGPU-PET_kernel.cu:1624-1836) on fixed
                    event lists for a span-1 and a span-11 scanner, with and
                    without energy blur;
* sample_run.npz    the reference transport on the sample geometry (9^3
                    voxels, seed 12345), host build: tallies as sparse bins;
* tables.npz        checksums of the interpolation tables built by
                    load_material for air + water;
* detector_kat_long_axial.npz  tally_Sinogram on photon pairs spread over
                    the 1 m long-axial scanner (256 rings, span 11, MRD 255:
                    bins up to 1.82e9, which the reference's int bin index
                    still holds).

    python tests/golden/make_golden.py                # every fixture
    python tests/golden/make_golden.py long_axial     # only the long-axial one
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "mcgpu-pet_b200"), os.path.join(ROOT, "tests"), ROOT]

import refbind  # noqa: E402
import scenes  # noqa: E402
from mcpet import inputs  # noqa: E402

SPAN11 = dict(fov_z=12.656, n_rows=80, n_crystals=336, n_angles=168, n_radial=147, n_z_slices=159,
              max_ring_difference=79, span=11, detector_radius=-9.05, detector_height=12.656)


def sparse(a):
    nz = np.nonzero(a)[0]
    return nz.astype(np.int64), a[nz].astype(np.int32)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def long_axial(work, ref):
    rng = np.random.default_rng(20261203)
    mat, rho, act, vs, used = inputs.body_phantom(shape=(50, 32, 32), voxel_cm=1.6, seed=5, total_bq=1.0e3)
    kat = {}
    for blur in (0.0, 0.12):
        sc = scenes.scene_from_arrays(work, mat, rho, act, vs, tissues=used, energy_resolution=blur,
                                      **inputs.scanner_long_axial())
        p = refbind.params_from_scene(sc)
        ev = scenes.random_events(4000, rng, box=(4.0, 4.0, 100.0), e_range=(360e3, 590e3))
        out = ref.sinogram_events(p, ev)
        key = f"res{int(blur * 100)}"
        for k, v in ev.items():
            kat[f"{key}_{k}"] = v
        kat[f"{key}_out"] = out
        sc.close()
    np.savez_compressed(os.path.join(HERE, "detector_kat_long_axial.npz"), **kat)


def main():
    work = tempfile.mkdtemp()
    if sys.argv[1:] == ["long_axial"]:
        long_axial(work, refbind.RefCPU())
        print("long-axial fixture written to", HERE)
        return
    ref = refbind.RefCPU()
    ids = np.concatenate([np.arange(0, 64), [1000, 65535, 1 << 20, 33554431, 123456789, 838860799]]).astype(np.int64)
    s, f, d = ref.prng(12345, ids.astype(np.int32), 12)
    np.savez_compressed(os.path.join(HERE, "rng_streams.npz"), seed=12345, ids=ids, seeds=s, draws=f, ddraws=d)

    kat = {}
    rng = np.random.default_rng(20240611)
    for name, kw in (("span1", dict(inputs.scanner_small())), ("span11", SPAN11)):
        for blur in (0.0, 0.12):
            sc = scenes.sample_scene(work, energy_resolution=blur, **kw)
            p = refbind.params_from_scene(sc)
            ev = scenes.random_events(1500, rng, e_range=(360e3, 590e3))
            out = ref.sinogram_events(p, ev)
            key = f"{name}_res{int(blur * 100)}"
            for k, v in ev.items():
                kat[f"{key}_{k}"] = v
            kat[f"{key}_out"] = out
            sc.close()
    np.savez_compressed(os.path.join(HERE, "detector_kat.npz"), **kat)

    sc = scenes.sample_scene(work, tally_psf_sinogram=0, psf_size=100000, seed=12345)
    t = sc.export_tables()
    p = refbind.params_from_scene(sc)
    r = ref.run(p, t["voxels"], refbind.RefTables.from_scene_export(t), psf_capacity=100000)
    out = {"total_histories": r["total_histories"], "psf_count": r["psf_count"]}
    for k in ["trues", "scatter", "image_trues", "image_scatter", "spectrum"]:
        out[f"{k}_idx"], out[f"{k}_val"] = sparse(r[k])
    recs = scenes.psf_records(r["psf_raw"])
    out["psf_sha"] = sha(recs)
    np.savez_compressed(os.path.join(HERE, "sample_run.npz"), **out)

    io_cfg, vox, rt = refbind.RefIO().load(scenes.write_case(work, "golden_tab", *inputs.sample_phantom()))
    used = [0, 1]
    np.savez_compressed(os.path.join(HERE, "tables.npz"),
                        woodcock=sha(rt.woodcock[:-1]), mfp_a=sha(rt.mfp_a[:, used]), mfp_b=sha(rt.mfp_b[:, used]),
                        pmax=sha(rt.pmax[: io_cfg.n_e, used]), compton=sha(np.concatenate([rt.fco, rt.uico, rt.fj0])),
                        rayleigh=sha(np.concatenate([rt.xco, rt.pco, rt.aco, rt.bco])), voxels=sha(vox),
                        nsinos=io_cfg.nsinos, n_e=io_cfg.n_e)
    long_axial(work, ref)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
