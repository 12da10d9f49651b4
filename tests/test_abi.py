"""The C-ABI library: it loads, exports every entry point include/cr.h
declares, and rejects bad input on the host without touching a GPU."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cr.h")).read()
    return sorted(set(re.findall(r"\b(cr_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_symbols()
    for must in ("cr_scene_create", "cr_trace_rays", "cr_render", "cr_render_device", "cr_last_error",
                 "cr_scene_destroy", "cr_render_file", "cr_bsdf_eval", "cr_bsdf_sample", "cr_light_table"):
        assert must in names


def test_library_exports_every_declared_symbol(cr):
    lib = cr.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_strings(cr):
    assert b"sm_100a" in cr.lib().cr_version()
    assert isinstance(cr.lib().cr_last_error(), bytes)


def _empty(cr):
    h = C.c_void_p()
    assert cr.lib().cr_scene_create_empty(C.byref(h)) == cr.CR_OK
    return h


def test_shader_registry_and_errors(cr):
    lib = cr.lib()
    h = _empty(cr)
    try:
        ok = lib.cr_scene_add_shader(h, b"w", json.dumps(["Lambert", {"R": [0.5, 0.5, 0.5]}]).encode())
        assert ok == 0
        ok = lib.cr_scene_add_shader(h, b"g", json.dumps(
            ["GlossyBSDF", {"distribution": ["Beckmann", {"roughness": 0.3}], "color": [1, 1, 1]}]).encode())
        assert ok == 1
        assert lib.cr_scene_add_shader(h, b"e", b'["Emission", {"strength": 5}]') == 2
        # malformed JSON, unknown type, out-of-scope type
        assert lib.cr_scene_add_shader(h, b"x", b'["Lambert", {') == -2
        assert b"json" in lib.cr_last_error()
        assert lib.cr_scene_add_shader(h, b"x", b'["NoSuchShader", {}]') == -2
        assert b"no such type" in lib.cr_last_error()
        # the whole registry (shader.impl.cu:16-23); required properties as
        # the reference's get<T>( props, key ) demands them
        assert lib.cr_scene_add_shader(h, b"x", b'["GlassBSDF", {}]') == -2
        assert b"ior" in lib.cr_last_error()
        assert lib.cr_scene_add_shader(h, b"x", b'["GlassBSDF", {"ior": 1.5}]') == -2
        assert b"distribution" in lib.cr_last_error()
        beck = ["Beckmann", {"roughness": 0.2}]
        for cfg in (["GlossyBSDF", {"distribution": ["Cosine", {}]}], ["Transparent", {"color": [1, 1, 0]}],
                    ["Blackhole", {}], ["RefractionBSDF", {"ior": 1.33, "distribution": beck}],
                    ["GlassBSDF", {"ior": 1.5, "distribution": beck}],
                    ["Mixed", {"fac": ["Fresnel", {"ior": 1.5}], "shaders": [["Lambert", {}], ["Blackhole", {}]]}]):
            assert lib.cr_scene_add_shader(h, b"ok", json.dumps(cfg).encode()) >= 0, lib.cr_last_error()
        assert lib.cr_scene_add_shader(h, b"x", b'["GlossyBSDF", {"distribution": ["GGX", {}]}]') == -2
        assert lib.cr_scene_add_shader(h, b"x", b'["Mixed", {"shaders": [["Lambert", {}], ["Lambert", {}]]}]') == -2
        assert b"fac" in lib.cr_last_error()
        assert lib.cr_scene_add_shader(h, b"x", b'["Mixed", {"fac": ["Constant", {"value": 0.5}], '
                                                b'"shaders": [["Lambert", {}]]}]') == -2
        assert lib.cr_scene_add_shader(h, b"x", b'["Mixed", {"fac": ["Noise", {}], '
                                                b'"shaders": [["Lambert", {}], ["Lambert", {}]]}]') == -2
        assert lib.cr_scene_add_shader(h, b"x", b'["Mixed", {"fac": ["Constant", {}], '
                                                b'"shaders": [["Lambert", {}], ["Lambert", {}]]}]') == -2
        deep = ["Lambert", {}]
        for _ in range(17):
            deep = ["Mixed", {"fac": ["Constant", {"value": 0.5}], "shaders": [deep, ["Lambert", {}]]}]
        assert lib.cr_scene_add_shader(h, b"x", json.dumps(deep).encode()) == -5
        # the pointLight asset (pointLight.hpp:13-18)
        pos = np.array([1, 2, 3], np.float32)
        assert lib.cr_scene_add_point_light(h, C.c_void_p(pos.ctypes.data), None, 2.0) == 0
        assert lib.cr_scene_add_point_light(h, None, None, 2.0) == -1
        # CameraConfig::lens (config.hpp:14-27)
        assert lib.cr_scene_set_lens(h, 1) == 0 and lib.cr_scene_set_lens(h, 0) == 0
        assert lib.cr_scene_set_lens(h, 2) == -1
    finally:
        lib.cr_scene_destroy(h)


def test_mesh_validation(cr):
    lib = cr.lib()
    h = _empty(cr)
    try:
        lib.cr_scene_add_shader(h, b"w", b'["Lambert", {}]')
        v = np.zeros((3, 3), np.float32)
        v[1, 0] = v[2, 1] = 1
        good = np.array([[0, 1, 2]], np.uint32)
        bad = np.array([[0, 1, 3]], np.uint32)
        p = lambda a: C.c_void_p(a.ctypes.data)
        assert lib.cr_scene_add_mesh(h, p(v), 3, None, p(bad), 1, b"w") == -1
        assert b"out of range" in lib.cr_last_error()
        assert lib.cr_scene_add_mesh(h, p(v), 3, None, p(good), 1, b"missing") == -1
        assert b"not found" in lib.cr_last_error()
        nanv = v.copy()
        nanv[0, 0] = np.nan
        assert lib.cr_scene_add_mesh(h, p(nanv), 3, None, p(good), 1, b"w") == -1
        assert lib.cr_scene_add_mesh(h, p(v), 3, None, p(good), 1, b"w") == 0
        c = np.zeros(3, np.float32)
        assert lib.cr_scene_add_sphere(h, p(c), -1.0, b"w") == -1
        assert lib.cr_scene_add_sphere(h, p(c), 1.0, b"w") == 1
        # not committed yet: queries are refused with a state error
        hits = np.zeros(1, cr.HIT_DTYPE)
        rays = np.zeros((1, 7), np.float32)
        assert lib.cr_trace_rays(h, p(rays), 1, p(hits), 0) == -4
        desc = cr.render_desc(8, 8, 1)
        film = np.zeros((8, 8, 3))
        assert lib.cr_render(h, C.byref(desc), p(film), None) == -4
    finally:
        lib.cr_scene_destroy(h)


def test_null_arguments(cr):
    lib = cr.lib()
    assert lib.cr_scene_create(None, None, None) == -1
    assert lib.cr_scene_create_empty(None) == -1
    assert lib.cr_write_png(None, 1, 1, None) == -1


def test_png_writer(cr, tmp_path):
    rgb = np.zeros((4, 5, 3))
    rgb[..., 0] = np.linspace(-1, 2, 5)[None, :]
    path = str(tmp_path / "x.png")
    assert cr.lib().cr_write_png(path.encode(), 5, 4, C.c_void_p(rgb.ctypes.data)) == 0
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    import zlib
    # IHDR then IDAT: decode the stored deflate stream and check clamping (image.hpp:29-40)
    i = data.index(b"IDAT")
    n = int.from_bytes(data[i - 4:i], "big")
    raw = zlib.decompress(data[i + 4:i + 4 + n])
    row = np.frombuffer(raw[1:16], np.uint8).reshape(5, 3)
    assert list(row[:, 0]) == [0, 0, 127, 255, 255]


def test_empty_batch_is_rejected(cr):
    """cr_batch_create refuses an empty job table before touching the GPU."""
    with pytest.raises(cr.CrError):
        cr.Batch([])


def test_scene_schema_errors_before_any_gpu_work(cr):
    """Scene::Scene's schema checks (scene.cu:27-168, config.hpp:14-27): the
    parse fails, with the reference's messages, before the scene is uploaded."""
    lib = cr.lib()

    def create(doc):
        out = C.c_void_p()
        rc = lib.cr_scene_create(json.dumps(doc).encode(), b".", C.byref(out))
        assert not out.value
        return rc, lib.cr_last_error().decode()

    cam = {"lens": "pinhole", "position": [0, 0, 0], "target": [0, 1, 0]}
    base = lambda assets, shaders=None, camera=cam: {"scene": {"camera": [camera], "assets": assets,
                                                               "shaders": shaders or {}}}
    rc, msg = create(base([["pointLight", {"color": [1, 1, 1]}]]))
    assert rc == -2 and "position" in msg
    rc, msg = create(base([["areaLight", {}]]))
    assert rc == -2 and "unknown light type" in msg
    rc, msg = create(base([["teapot", {}]]))
    assert rc == -2 and "unknown asset type" in msg
    rc, msg = create(base([], camera=dict(cam, lens="fisheye")))
    assert rc == -2 and "unknown lens type" in msg
    rc, msg = create(base([["sphere", {"o": [0, 2, 0], "r": 1, "shader": "s"}]],
                          {"s": ["Mixed", {"fac": ["Constant", {"value": 0.5}]}]}))
    assert rc == -2 and "shaders" in msg
    rc, msg = create(base([["sphere", {"o": [0, 2, 0], "r": 1, "shader": "missing"}]]))
    assert rc == -1 and "not found" in msg


def _reference_sources():
    d = os.environ.get("CR_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")
    return d if os.path.isdir(os.path.join(d, "src")) else None


@pytest.mark.skipif(_reference_sources() is None, reason="reference sources absent")
def test_tracer_plugin_builds_into_the_reference():
    """The CudaWavefront Tracer plugin (cuda-raytracer_b200/plugin/) compiles
    against the unmodified reference, registers in Factory<Tracer> and links
    the library (make -C oracle plugin); the GPU test runs it."""
    import subprocess
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "plugin", f"REF={_reference_sources()}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    exe = os.path.join(ROOT, "oracle", "_ref", "cr_ref_plugin")
    assert os.path.exists(exe)
    r = subprocess.run(["ldd", exe], capture_output=True, text=True)
    assert "libcr_b200.so" in r.stdout and "not found" not in r.stdout, r.stdout


def _header_struct_fields(text, name):
    """(field, C type) pairs of `typedef struct name { ... } name;` in order,
    comments removed; `uint32_t a, b;` gives two fields, pointers read as "*"."""
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for decl in (d.strip() for d in body.split(";")):
        if not decl:
            continue
        m = re.match(r"([A-Za-z_][A-Za-z_0-9]*)\s*(\*?)\s*(.*)", decl)
        ctype = "*" if m.group(2) else m.group(1)
        for nm in m.group(3).split(","):
            out.append((nm.strip(), ctype))
    return out


def test_ctypes_mirrors_match_the_header(cr):
    """Every struct the package passes through the C ABI has the header's
    fields, in the header's order, with the same widths: the library writes
    whole structs (cr_stats is cleared with memset), so a shorter mirror would
    be overwritten past its end."""
    ctype = {"int32_t": C.c_int32, "uint32_t": C.c_uint32, "uint64_t": C.c_uint64, "float": C.c_float,
             "double": C.c_double, "*": C.c_void_p}
    with open(os.path.join(ROOT, "include", "cr.h")) as fh:
        text = fh.read()
    pairs = {"cr_hit": cr.Hit, "cr_render_desc": cr.RenderDesc, "cr_tuning": cr.Tuning, "cr_stats": cr.Stats,
             "cr_guide_config": cr.GuideConfig, "cr_build_config": cr.BuildConfig, "cr_batch_job": cr.BatchJob}
    for cname, py in pairs.items():
        want = [(n, ctype[t]) for n, t in _header_struct_fields(text, cname)]
        assert list(py._fields_) == want, cname
