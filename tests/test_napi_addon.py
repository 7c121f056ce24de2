"""The Node-API addon and its JavaScript GSTrainer class, without Node.js
(neither this machine nor the GPU box has a JavaScript runtime).

- The addon (splat.js_b200/native/gs_b200_napi.c) compiles warning-free as
  C11 against Node-API's declarations (a declaration-only header written from
  the documented interface) and include/splat_b200.h.
- Every library function it calls is declared in the header and exported by
  libsplat_b200.so, and it exports the module entry point.
- Every addon function the JavaScript class (splat.js_b200/js/
  trainer_b200.js) calls is registered by the addon, and the class has every
  method and field of the reference's GSTrainer surface that callers use
  (src/gs/trainer.js; session.js:284-305)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "splat.js_b200", "native")
ADDON = os.path.join(NATIVE, "gs_b200_napi.c")
SHIM = os.path.join(ROOT, "splat.js_b200", "js", "trainer_b200.js")


def compile_addon(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    obj = str(tmp_path / "gs_b200_napi.o")
    r = subprocess.run([cc, "-std=c11", "-D_POSIX_C_SOURCE=200809L", "-Wall", "-Wextra", "-Werror", "-fPIC",
                        "-I", os.path.join(NATIVE, "napi_stub"), "-I", os.path.join(ROOT, "include"), "-c",
                        ADDON, "-o", obj], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return obj


def nm(args, path):
    r = subprocess.run(["nm", *args, path], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_addon_compiles_and_links_only_exported_entry_points(tmp_path):
    obj = compile_addon(tmp_path)
    out = nm([], obj)
    used = set(re.findall(r"\bU (gs_\w+)", out))
    assert {"gs_create", "gs_setup", "gs_step", "gs_step_batch", "gs_read_stats", "gs_read_gaussians",
            "gs_refine", "gs_render", "gs_eval_pass", "gs_sync"} <= used
    assert re.search(r"\bT napi_register_module_v1\b", out)
    hdr = open(os.path.join(ROOT, "include", "splat_b200.h")).read()
    declared = set(re.findall(r"GS_API\s+[\w\s\*]*?\b(gs_\w+)\s*\(", hdr))
    assert used <= declared, used - declared
    import importlib.util
    spec = importlib.util.spec_from_file_location("gs_build", os.path.join(ROOT, "splat.js_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    lib = mod.build()
    exported = set(re.findall(r"\bT (gs_\w+)", nm(["-D", "--defined-only"], lib)))
    assert used <= exported, used - exported


def test_javascript_class_uses_registered_functions_and_keeps_the_surface():
    src = open(ADDON).read()
    table = src[src.index("NAPI_MODULE_INIT()"):]
    registered = set(re.findall(r'\{"(\w+)",\s*\w+\}', table))
    shim = open(SHIM).read()
    called = set(re.findall(r"\baddon\.(\w+)\(", shim))
    assert called and called <= registered, called - registered
    methods = set(re.findall(r"^  (?:async |static async |get |set )?(\w+)\(", shim, re.M))
    for m in ["create", "setup", "stepOnce", "renderView", "renderTrainCam", "readLoss", "refine", "readGaussians",
              "evalCamPsnr", "evalCamPsnrRefined", "_applyCamGrads", "iter", "n", "cap", "horizon", "pixelsSeen"]:
        assert m in methods, m
    for field in ["holdout", "excluded", "lastCam", "lastRefine", "growLimit", "camMeta", "shK", "shDeg",
                  "stride", "entryOverflowTiles", "rand", "device"]:
        assert re.search(rf"this\.{field}\s*=", shim), field
