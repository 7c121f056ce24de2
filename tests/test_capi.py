"""The C ABI without a GPU: the library builds, loads, and exports every
entry point include/splat_b200.h declares; defaults mirror the reference's
GSTrainer options (src/gs/trainer.js:18-49)."""
import ctypes as C
import os
import re

import pytest

from splat_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "splat_b200.h")).read()
    return sorted(set(re.findall(r"GS_API\s+[\w\s\*]*?\b(gs_\w+)\s*\(", src)))


def test_library_builds_and_exports_every_declared_symbol():
    import importlib.util
    spec = importlib.util.spec_from_file_location("gs_build", os.path.join(ROOT, "splat.js_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    path = mod.build()
    assert os.path.exists(path)
    syms = declared_symbols()
    assert len(syms) >= 25, syms
    L = C.CDLL(path)
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    # the binding covers the header exactly
    N.lib()
    assert N.lib().gs_abi_version() == 2


def test_default_options_match_reference():
    o = N.GsOptions()
    assert N.lib().gs_default_options(C.byref(o)) == 0
    assert o.eCut == pytest.approx(4.5) and o.aMin == pytest.approx(0.0039)
    assert o.radClamp == 1.0 and o.anisoReg == pytest.approx(0.005)
    assert o.shDeg == 2 and o.tileGrad == 1 and o.capMult == 4.0 and o.maxIters == 60000
    assert o.minScale == pytest.approx(1e-4) and o.opacityReg == pytest.approx(0.01)
    assert o.shLr == pytest.approx(1.25e-4) and o.growRate == pytest.approx(0.15)
    assert o.tile == 16 and o.tileCull == 1 and o.donorSampling == 0


def test_struct_sizes_match_header():
    assert C.sizeof(N.GsOptions) == 4 * 6 + 8 + 4 * 2 + 8 * 4 + 4 * 2 + 4 * 9 + 4  # tail padding to 8
    assert C.sizeof(N.GsCamera) == 4 * (9 + 3 + 3 + 3) + 8 * 2
    assert C.sizeof(N.GsImage) == 16
    assert C.sizeof(N.GsRefineResult) == 24


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """Every field offset and struct size of the ctypes mirror equals what a
    C compiler lays out from include/splat_b200.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"gs_options": N.GsOptions, "gs_camera": N.GsCamera, "gs_image": N.GsImage,
               "gs_state": N.GsState, "gs_refine_result": N.GsRefineResult, "gs_frame": N.GsFrame}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "splat_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'  printf("{cname}.{f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(ln.split() for ln in subprocess.run([str(exe)], check=True, capture_output=True,
                                                   text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f in py._fields_:
            assert int(got[f"{cname}.{f[0]}"]) == getattr(py, f[0]).offset, f"{cname}.{f[0]}"


def test_create_without_device_fails_cleanly():
    """On a host with no GPU gs_create reports an error instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = N.lib().gs_create(None, C.byref(h))
    assert rc != 0
    assert b"device" in N.lib().gs_last_error(None)


def test_static_sort_rejects_sizes_above_its_limit():
    """The allocation-free sort refuses n > GS_STATIC_SORT_MAX before any device work."""
    rc = N.lib().gs_sort_entries_static(None, None, N.STATIC_SORT_MAX + 1, 16, None)
    assert rc == N.GS_E_LIMIT
    hdr = open(os.path.join(ROOT, "include", "splat_b200.h")).read()
    assert "#define GS_STATIC_SORT_MAX (1u << 20)" in hdr


def test_lookback_check_rejects_bad_spin_limits():
    st, ms = C.c_uint32(), C.c_double()
    assert N.lib().gs_debug_lookback_timeout(0, 0, C.byref(st), C.byref(ms)) == -1
    assert N.lib().gs_debug_lookback_timeout(0, (1 << 22) + 1, C.byref(st), C.byref(ms)) == -1


def test_ingestion_entry_points_check_their_arguments():
    """gs_undistort_frames and gs_debug_targets refuse bad arguments before
    touching a device; below the distortion noise floor nothing is resampled
    and no device is needed."""
    L = N.lib()
    done = C.c_int32(7)
    assert L.gs_undistort_frames(0, None, 1, 0.3, 0.0, 10.0, C.byref(done)) == -1
    assert done.value == 0
    fr = (N.GsFrame * 1)()
    fr[0].tw, fr[0].th, fr[0].fw = 4, 4, 4.0          # pixels but no buffer
    assert L.gs_undistort_frames(0, fr, 1, 0.3, 0.0, 10.0, C.byref(done)) == -1
    done.value = 7
    assert L.gs_undistort_frames(0, fr, 1, 0.005, -0.005, 10.0, C.byref(done)) == 0
    assert done.value == 0
    assert L.gs_debug_targets(None, None, 0) == -1
