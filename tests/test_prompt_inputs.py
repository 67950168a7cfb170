"""Prompt-gamma emitter, host side: the extended material tables, the
optional input-file section, and the refusals.

The reference emits only 511 keV photons (MCGPU-PET_kernel.cu:669) and ships
tables that stop at 514.95 keV; mcpet.tables continues them to 1250 keV in
the reference's format (its own loader reads them: tests/test_tables.py)."""
import numpy as np
import pytest

import mcpet
from mcpet import inputs, tables
import refbind
import scenes


def test_extended_table_keeps_the_source_rows_and_continues_smoothly():
    src = inputs.material_path("water")
    ext = inputs.material_path("water", extended=True)
    h0, rows0, d0, tail0 = tables.read_table(src)
    h1, rows1, d1, tail1 = tables.read_table(ext)
    assert len(rows1) == 24901 and rows1[: len(rows0)] == rows0 and tail1 == tail0
    assert d1[-1, 0] == 1.25e6
    np.testing.assert_allclose(np.diff(d1[:, 0]), 50.0, rtol=0, atol=1e-6)
    n = len(rows0)
    # Compton mean free path continues as the Klein-Nishina cross-section ratio
    e = d1[n:, 0]
    np.testing.assert_allclose(d1[n:, 2] / d0[-1, 2], tables.klein_nishina_sigma(d0[-1, 0]) /
                               tables.klein_nishina_sigma(e), rtol=1e-9)
    # every mean free path grows with energy and joins the tabulated rows
    # without a step larger than the tabulated rows' own last step
    for col in (1, 2, 3, 4):
        assert np.all(np.diff(d1[n - 5:, col]) > 0), col
        last_step = d0[-1, col] / d0[-2, col]
        first_step = d1[n, col] / d0[-1, col]
        assert abs(np.log(first_step) - np.log(last_step)) < 2e-2 * abs(np.log(last_step)) + 1e-9, col
    tot = 1.0 / (1.0 / d1[n:, 1] + 1.0 / d1[n:, 2] + 1.0 / d1[n:, 3])
    np.testing.assert_allclose(d1[n:, 4], tot, rtol=1e-9)


def test_input_section_is_read_by_this_library_and_skipped_by_the_reference(workdir):
    mat, rho, act, vs = inputs.water_cube_phantom(1.0e4)
    plain = scenes.write_case(workdir, "pg_plain", mat, rho, act, vs, extended=True)
    prompt = scenes.write_case(workdir, "pg_prompt", mat, rho, act, vs, extended=True,
                               prompt_gamma_energy=1157020.0, prompt_gamma_yield=0.9)
    a, b = mcpet.read_config(plain), mcpet.read_config(prompt)
    assert a.prompt_gamma_energy == 0.0
    assert b.prompt_gamma_energy == np.float32(1157020.0) and b.prompt_gamma_yield == np.float32(0.9)
    assert bytes(a.voxel_file) != b"" and a.n_bins == b.n_bins
    if refbind.available("libref_prog.so"):
        ra, _, _ = refbind.RefIO().load(plain)
        rb, _, _ = refbind.RefIO().load(prompt)
        for f in ("nbins", "nrows", "mrd", "span", "e_low", "e_high", "radius"):
            assert getattr(ra, f) == getattr(rb, f), f
        assert bytes(ra.voxel_file).split(b"/")[-1] != b"" and bytes(rb.materials[0]) == bytes(ra.materials[0])


@pytest.mark.parametrize("case", ["tables_too_short", "psf_tally", "bad_yield"])
def test_prompt_gamma_refusals(workdir, case):
    mat, rho, act, vs = inputs.water_cube_phantom(1.0e4)
    kw = dict(prompt_gamma_energy=1157020.0, extended=True)
    if case == "tables_too_short":
        kw["extended"] = False
    elif case == "psf_tally":
        kw.update(tally_psf_sinogram=0, psf_size=1000)
    else:
        kw["prompt_gamma_yield"] = 1.5
    if case == "bad_yield":
        with pytest.raises(mcpet.McpetError) as e:
            scenes.scene_from_arrays(workdir, mat, rho, act, vs, **kw)
        assert e.value.status == 3 and "yield" in str(e.value)
        return
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs, **kw)
    with pytest.raises(mcpet.McpetError) as e:
        sc.run(mcpet.RunOptions())
    assert e.value.status == 1
    assert ("tables" in str(e.value)) if case == "tables_too_short" else ("sinogram tally only" in str(e.value))
    sc.close()
