"""Failure handling on the host: malformed or truncated inputs come back as
error statuses with a message (the reference prints and exit()s); nothing
here touches a GPU."""
import gzip
import os

import numpy as np
import pytest

import mcpet
from mcpet import _abi, inputs
import scenes

ERR = {"arg": 1, "io": 2, "format": 3, "cuda": 4, "limit": 6}


def _expect(kind, fn, *a, match=None):
    with pytest.raises(mcpet.McpetError) as e:
        fn(*a)
    assert e.value.status == ERR[kind], str(e.value)
    if match:
        assert match in str(e.value), str(e.value)
    return e.value


def _case(workdir, name, **kw):
    mat, rho, act, vs = inputs.sample_phantom()
    return scenes.write_case(workdir, name, mat, rho, act, vs, **kw)


def test_missing_input_file(workdir):
    _expect("io", mcpet.Scene.load, os.path.join(workdir, "nope.in"))
    _expect("io", mcpet.read_config, os.path.join(workdir, "nope.in"))


@pytest.mark.parametrize("section", ["SECTION SOURCE PET SCAN", "SECTION PHASE SPACE FILE", "SECTION DOSE DEPOSITION",
                                     "SECTION ENERGY PARAMETERS", "SECTION SINOGRAM PARAMETERS",
                                     "SECTION VOXELIZED GEOMETRY", "SECTION MATERIAL"])
def test_missing_section(workdir, section):
    inp = _case(workdir, "nosec")
    text = open(inp).read().replace(section, "SECTION REMOVED")
    open(inp, "w").write(text)
    _expect("format", mcpet.read_config, inp, match="lacks")


def test_old_dose_section_and_bad_answers(workdir):
    inp = _case(workdir, "olddose")
    text = open(inp).read()
    open(inp, "w").write(text.replace("DOSE DEPOSITION v.2012-12-12", "DOSE DEPOSITION v.2011-02-18"))
    _expect("format", mcpet.read_config, inp, match="v.2011-02-18")
    open(inp, "w").write(text.replace("NO            # TALLY MATERIAL DOSE", "MAYBE         # TALLY MATERIAL DOSE"))
    _expect("format", mcpet.read_config, inp, match="YES or NO")


def test_zero_span_rejected(workdir):
    inp = _case(workdir, "span0", span=0)
    _expect("format", mcpet.read_config, inp, match="SPAN")


def test_voxel_file_errors(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, "vox", mat, rho, act, vs)
    vox = os.path.join(workdir, "vox.vox")
    good = open(vox).read()
    lines = good.splitlines()
    open(vox, "w").write("\n".join(lines[:-10]) + "\n")                       # truncated
    _expect("format", mcpet.Scene.load, inp, match="ended after")
    bad = list(lines)
    bad[20] = "2 1.0"                                                          # two items
    open(vox, "w").write("\n".join(bad) + "\n")
    _expect("format", mcpet.Scene.load, inp, match="3 items")
    for repl, msg in (("16 1.0 0.0", "too high"), ("0 1.0 0.0", "zero or negative"), ("2 0.0 0.0", "density")):
        bad = list(lines)
        bad[30] = repl
        open(vox, "w").write("\n".join(bad) + "\n")
        _expect("format", mcpet.Scene.load, inp, match=msg)
    open(vox, "w").write(good.replace("[END OF VXH SECTION]", "[END OF SOMETHING]"))
    _expect("format", mcpet.Scene.load, inp, match="END OF VXH")
    os.remove(vox)
    _expect("io", mcpet.Scene.load, inp)


def test_truncated_gzip_voxels(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    inp = scenes.write_case(workdir, "gzv", mat, rho, act, vs, gz=True)
    path = os.path.join(workdir, "gzv.vox.gz")
    data = open(path, "rb").read()
    open(path, "wb").write(data[: len(data) // 2])
    _expect("format", mcpet.Scene.load, inp)


def _material_copy(workdir, name, edit):
    with gzip.open(inputs.material_path("water"), "rt") as f:
        lines = f.read().splitlines()
    lines = edit(lines)
    p = os.path.join(workdir, name)
    with open(p, "w") as f:
        f.write("\n".join(lines) + "\n")
    return p


def test_material_file_errors(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    air = inputs.material_path("air")

    def with_water(path, name):
        spec = inputs.spec_for([air, path], scenes.inputs.write_vox(os.path.join(workdir, f"{name}.vox"), mat, rho,
                                                                      act, vs), **inputs.scanner_small())
        return inputs.write_input(os.path.join(workdir, f"{name}.in"), spec)

    # different number of energy rows than the first material
    def fewer_rows(lines):
        i = lines.index("#[NUMBER OF DATA VALUES]")
        lines[i + 1] = "#  10199"
        return lines
    _expect("format", mcpet.Scene.load, with_water(_material_copy(workdir, "w1", fewer_rows), "m1"),
            match="number of energy values")

    # non-constant energy step
    def bad_step(lines):
        parts = lines[200].split()
        parts[0] = f"{float(parts[0]) + 7.0:.10E}"
        lines[200] = "  " + "  ".join(parts)
        return lines
    _expect("format", mcpet.Scene.load, with_water(_material_copy(workdir, "w2", bad_step), "m2"),
            match="not constant")

    # truncated inside the Compton shells
    _expect("format", mcpet.Scene.load, with_water(_material_copy(workdir, "w3", lambda l: l[:-2]), "m3"),
            match="Compton")
    # missing file
    _expect("io", mcpet.Scene.load, with_water(os.path.join(workdir, "missing.mcgpu.gz"), "m4"))


def test_table_must_reach_511_kev(workdir):
    def short(lines):
        i = lines.index("#[NUMBER OF DATA VALUES]")
        n = 9000
        lines[i + 1] = f"#  {n}"
        j = i + 4          # first data row
        return lines[: j + n] + lines[j + 10200:]
    p_air = _material_copy(workdir, "a_short.mcgpu", lambda l: l)
    with gzip.open(inputs.material_path("air"), "rt") as f:
        air_lines = f.read().splitlines()
    i = air_lines.index("#[NUMBER OF DATA VALUES]")
    air_lines[i + 1] = "#  9000"
    air_lines = air_lines[: i + 4 + 9000] + air_lines[i + 4 + 10200:]
    open(p_air, "w").write("\n".join(air_lines) + "\n")
    p_w = _material_copy(workdir, "w_short.mcgpu", short)
    mat, rho, act, vs = inputs.sample_phantom()
    spec = inputs.spec_for([p_air, p_w], inputs.write_vox(os.path.join(workdir, "short.vox"), mat, rho, act, vs),
                           **inputs.scanner_small())
    inp = inputs.write_input(os.path.join(workdir, "short.in"), spec)
    _expect("format", mcpet.Scene.load, inp, match="do not have data up to")


def test_material_slot_problems(workdir):
    mat, rho, act, vs = inputs.sample_phantom()
    vox = inputs.write_vox(os.path.join(workdir, "slots.vox"), mat, rho, act, vs)
    spec = inputs.spec_for(["", inputs.material_path("water")], vox, **inputs.scanner_small())
    spec.material_files = ["#", inputs.material_path("water")]
    p = inputs.write_input(os.path.join(workdir, "slots.in"), spec)
    text = open(p).read().replace("#     # 1\n", "")
    open(p, "w").write(text)
    _expect("format", mcpet.Scene.load, p)
    spec = inputs.spec_for([inputs.material_path("air")], vox, **inputs.scanner_small())
    p = inputs.write_input(os.path.join(workdir, "slots2.in"), spec)
    _expect("format", mcpet.Scene.load, p, match="no material file")


def test_run_argument_checks(workdir):
    sc = scenes.sample_scene(workdir)
    _expect("arg", sc.run, mcpet.RunOptions(seed_override=-5))
    _expect("arg", sc.run, mcpet.RunOptions(lane_mode=7))
    sc.close()
    sc = scenes.sample_scene(workdir, seed=12345)
    cfg = sc.config
    cfg.span = 0
    _expect("arg", mcpet.Scene.from_arrays, cfg, *inputs.sample_phantom())
    sc.close()


def test_null_arguments_return_status():
    L = _abi.lib()
    assert L.mcpet_scene_load(None, None) == ERR["arg"]
    assert L.mcpet_run(None, None, None) == ERR["arg"]
    assert L.mcpet_scene_get_info(None, None) == ERR["arg"]
    assert L.mcpet_probe_rng(0, 1, None, 0, None, None, None) == ERR["arg"]
    assert b"null" in L.mcpet_last_error() or b"invalid" in L.mcpet_last_error()


def test_run_without_gpu_reports_cuda_error(workdir):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    sc = scenes.sample_scene(workdir)
    _expect("cuda", sc.run)
    sc.close()


def test_grad_argument_checks(workdir):
    """mcpet_grad rejects missing inputs before any device work."""
    import ctypes as C
    L = _abi.lib()
    sc = scenes.sample_scene(workdir)
    t = _abi.Tallies()
    g = _abi.GradArgs()
    assert L.mcpet_grad(None, None, C.byref(t), C.byref(g)) == ERR["arg"]
    assert L.mcpet_grad(sc.handle, None, C.byref(t), C.byref(g)) == ERR["arg"]      # no measured sinogram
    assert b"measured" in L.mcpet_last_error()
    g.measured = 16
    assert L.mcpet_grad(sc.handle, None, C.byref(t), C.byref(g)) == ERR["arg"]      # no forward sinograms
    assert b"trues and scatter" in L.mcpet_last_error()
    t.trues, t.scatter = 16, 16
    g.event_buffer, g.event_capacity = 16, 0
    assert L.mcpet_grad(sc.handle, None, C.byref(t), C.byref(g)) == ERR["arg"]
    assert b"event_capacity" in L.mcpet_last_error()
    sc.close()
    psf_only = scenes.sample_scene(workdir, tally_psf_sinogram=1)
    g.event_buffer, g.event_capacity = None, 0
    assert L.mcpet_grad(psf_only.handle, None, C.byref(t), C.byref(g)) == ERR["arg"]
    assert b"sinogram tally" in L.mcpet_last_error()
    psf_only.close()


def test_psf_stream_argument_checks(workdir):
    import ctypes as C
    L = _abi.lib()
    t = _abi.Tallies()
    sino_only = scenes.sample_scene(workdir, tally_psf_sinogram=2)
    cb = _abi.PSF_SINK(lambda p, n, u: 0)
    assert L.mcpet_run_psf_stream(sino_only.handle, None, 64, C.cast(cb, C.c_void_p), None, C.byref(t)) == ERR["arg"]
    assert b"does not tally a PSF" in L.mcpet_last_error()
    sino_only.close()
    psf = scenes.sample_scene(workdir, tally_psf_sinogram=1)
    assert L.mcpet_run_psf_stream(psf.handle, None, 1, C.cast(cb, C.c_void_p), None, C.byref(t)) == ERR["arg"]
    assert b"chunk_records" in L.mcpet_last_error()
    assert L.mcpet_run_psf_stream(psf.handle, None, 64, None, None, C.byref(t)) == ERR["arg"]
    psf.close()


def test_batch_graph_and_autotune_argument_errors(workdir):
    """Host-side checks of the graph and autotuner entry points (no device work)."""
    import ctypes as C
    L = _abi.lib()
    h = C.c_void_p()
    t = (_abi.Tallies * 1)()
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_batch_graph_create(None, 0, None, t, 1, C.byref(h)))
    assert e.value.status == ERR["arg"]
    mat, rho, act, vs = inputs.sample_phantom()
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs)
    ptrs = (C.c_void_p * 1)(sc.handle)
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_batch_graph_create(ptrs, 1, None, t, -1, C.byref(h)))
    assert e.value.status == ERR["arg"] and "seed step" in str(e.value)
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_batch_graph_create(ptrs, 1, None, None, 1, C.byref(h)))
    assert e.value.status == ERR["arg"]
    for fn, args in ((L.mcpet_batch_graph_launch, (None, None)), (L.mcpet_batch_graph_set_seeds, (None, None, None)),
                     (L.mcpet_batch_graph_guard_trips, (None, None))):
        with pytest.raises(mcpet.McpetError) as e:
            _abi.check(fn(*args))
        assert e.value.status == ERR["arg"]
    L.mcpet_batch_graph_destroy(None)
    r = _abi.TuneResult()
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_autotune(ptrs, 1, None, None, 1e6, C.byref(r)))
    assert e.value.status == ERR["arg"]
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_autotune(ptrs, 0, None, t, 1e6, C.byref(r)))
    assert e.value.status == ERR["arg"]
    sc.close()


def test_async_run_argument_errors(workdir):
    """Host-side checks of the asynchronous entry points (no device work)."""
    import ctypes as C
    L = _abi.lib()
    t = _abi.Tallies()
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_run_async(None, None, C.byref(t)))
    assert e.value.status == ERR["arg"]
    mat, rho, act, vs = inputs.sample_phantom()
    sc = scenes.scene_from_arrays(workdir, mat, rho, act, vs)
    psf = np.zeros(44, np.uint8)
    t.psf = psf.ctypes.data
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_run_async(sc.handle, None, C.byref(t)))
    assert e.value.status == ERR["arg"] and "PSF" in str(e.value)
    with pytest.raises(mcpet.McpetError) as e:
        _abi.check(L.mcpet_run_wait(None))
    assert e.value.status == ERR["arg"]
    _abi.check(L.mcpet_run_wait(sc.handle))      # nothing in flight
    sc.close()
