"""The per-bounce debug dump of the reference's Profiler
(src/core/kernel/kernel.hpp:35-81, RadianceKernel::Slice in
src/core/kernel/radiance.hpp:17-55, radiance.cu:41-53).

CPU: cr_profile_write prints slices in the reference's text format.
GPU: a scene file with an enabled "profiler" block renders its area through
cr_render_file and writes a dump that lines up with the one the reference's
own CPUMulticoreTracer + Profiler writes (oracle/_ref/cr_ref profile): the same
"at [ x, y, k ]" sequence, the same camera ray and first shader for every
sample both print, and as many printed (bright) samples within Monte Carlo
error; the raw slices follow the reference loop's bounce counter.
"""
import ctypes as C
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import require_gpu

AREA = (24, 8, 40, 24)
W = H = 64
SPP = 16
DEPTH = 8


class Bounce(C.Structure):
    _fields_ = [("ray_o", C.c_float * 3), ("ray_d", C.c_float * 3), ("f", C.c_float * 3), ("theta", C.c_float),
                ("L", C.c_float * 3), ("shader", C.c_uint32)]


class Slice(C.Structure):
    _fields_ = [("bounce", C.c_uint32), ("L", C.c_float * 3)]


def parse(path):
    """{(x, y, k): [records]} of a dump; a record is a dict of its lines."""
    out, cur, rec = {}, None, None
    for line in open(path):
        line = line.rstrip("\n")
        m = re.match(r"at \[ (\d+), (\d+), (\d+) \]: $", line)
        if m:
            cur = tuple(int(v) for v in m.groups())
            out[cur] = {"bounce": None, "records": []}
            continue
        key, _, val = line.partition(": ")
        if key == "bounce":
            out[cur]["bounce"] = tuple(int(v) for v in val.split(" / "))
        elif key == "ray":
            rec = {"ray": [float(v) for v in re.findall(r"[-+0-9.eE]+|nan|inf", val)]}
            out[cur]["records"].append(rec)
        elif key in ("f", "L"):
            rec[key] = [float(v) for v in re.findall(r"[-+0-9.eE]+|nan|inf", val)]
        elif key == "theta":
            rec[key] = float(val)
        elif key == "shader":
            rec[key] = int(val)
    return out


def test_profile_text_format(cr, tmp_path):
    lib = cr.lib()
    area = (C.c_uint32 * 4)(5, 7, 6, 8)
    sl = (Slice * 2)()
    bo = (Bounce * 4)()
    sl[0].bounce, sl[0].L[:] = 3, (150.0, 200.5, 1000.0)   # printed: every channel >= 100
    sl[1].bounce, sl[1].L[:] = 1, (150.0, 99.0, 1000.0)    # not printed
    b = bo[0]
    b.ray_o[:], b.ray_d[:], b.f[:] = (1.0, -2.5, 0.125), (0.6, 0.8, 0.0), (0.25, 0.5, 0.75)
    b.theta, b.L[:], b.shader = 1.5, (3.0, 4.0, 5.0), 7
    bo[1].ray_o[:], bo[1].L[:], bo[1].shader = (9.0, 9.0, 9.0), (150.0, 200.5, 1000.0), 2
    lib.cr_profile_write.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
    p = tmp_path / "a.prof"
    assert lib.cr_profile_write(str(p).encode(), area, 2, 2, C.byref(sl), C.byref(bo)) == 0
    want = ("at [ 5, 7, 0 ]: \n"
            "bounce: 3 / 2\n"
            "ray: [ 1, -2.5, 0.125 ][ 0.6, 0.8, 0 ]\nf: [ 0.25, 0.5, 0.75 ]\ntheta: 1.5\nL: [ 3, 4, 5 ]\nshader: 7\n"
            "ray: [ 9, 9, 9 ][ 0, 0, 0 ]\nf: [ 0, 0, 0 ]\ntheta: 0\nL: [ 150, 200.5, 1000 ]\nshader: 2\n"
            "at [ 5, 7, 1 ]: \n")
    assert p.read_text() == want


def _profile_scene(scenes, tmp, out_name):
    d = scenes.config0()
    # a brighter panel, so that some samples reach 100 in every channel and print
    d.shaders["light"] = ["Emission", {"color": [1, 1, 1], "strength": 400.0}]
    path = scenes.write_scene(d, str(tmp))
    doc = json.load(open(path))
    doc["profiler"] = {"enable": True, "output": out_name, "area": list(AREA), "props": {"depth": DEPTH}}
    json.dump(doc, open(path, "w"))
    return d, path


@pytest.mark.gpu
def test_profile_matches_the_reference_profiler(cr, scenes, oracle, tmp_path):
    require_gpu()
    if not oracle.ref_available():
        pytest.skip("reference harness not built")
    d, path = _profile_scene(scenes, tmp_path, "ours.prof")
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        cr.render_file(path, str(tmp_path / "ours.png"), spp=SPP, width=W, height=H)
    finally:
        os.chdir(cwd)
    r = subprocess.run([oracle.REF_BIN, "profile", os.path.basename(path), str(W), str(H), str(SPP), *map(str, AREA),
                        str(DEPTH), "ref.prof"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ours, ref = parse(tmp_path / "ours.prof"), parse(tmp_path / "ref.prof")
    # the same samples in the same order
    assert list(ours) == list(ref)
    assert len(ours) == (AREA[2] - AREA[0]) * (AREA[3] - AREA[1]) * SPP
    po = {k for k, v in ours.items() if v["bounce"]}
    pr = {k for k, v in ref.items() if v["bounce"]}
    assert len(pr) > 20, len(pr)
    # bright samples are rare paths (the panel is not seen directly): as many
    # print as the reference prints, within Monte Carlo error, with a similar
    # number of bounces
    assert abs(len(po) - len(pr)) <= 4 * np.sqrt(len(pr)) + 5, (len(po), len(pr))
    mo = np.mean([ours[k]["bounce"][0] for k in po])
    mr = np.mean([ref[k]["bounce"][0] for k in pr])
    assert abs(mo - mr) < 1.0, (mo, mr)
    # in both dumps, the first record of every printed sample holds the camera
    # ray PinholeLens::sample gives for its (x, y, k): the records sit in
    # their samples' slices
    for dump, printed in ((ours, po), (ref, pr)):
        keys = sorted(printed)
        pix = np.array([[k[0], k[1]] for k in keys])
        o, dd = scenes.pinhole_rays(d.camera, W, H, SPP, pix, np.array([k[2] for k in keys]))
        got = np.array([dump[k]["records"][0]["ray"] for k in keys])
        np.testing.assert_allclose(got[:, :3], o, rtol=2e-5, atol=2e-5)  # six printed digits
        np.testing.assert_allclose(got[:, 3:], dd, rtol=2e-5, atol=2e-5)
        assert all(dump[k]["bounce"][1] == DEPTH for k in keys)
    # printed records: a record per counted bounce (up to the depth), and the
    # recorded radiance never decreases along the path
    for v in ours.values():
        if v["bounce"]:
            assert len(v["records"]) == min(v["bounce"][0], DEPTH)
            Ls = [rec["L"] for rec in v["records"]]
            assert all(np.all(np.asarray(Ls[i + 1]) >= np.asarray(Ls[i]) - 1e-3 * np.abs(Ls[i])) for i in range(len(Ls) - 1))


@pytest.mark.gpu
def test_profile_slices_follow_the_reference_loop(cr, scenes):
    """Raw slices of the whole 64x64x16 image: the bounce counter is what
    radiance.cu's loop leaves (at most maxBounce + 1, records for every
    counted vertex up to the depth), the slice radiance is the sample's, and
    the profiled film equals an unprofiled render's statistics."""
    require_gpu()
    sc = cr.Scene.from_desc(scenes.config0())
    lib = cr.lib()
    lib.cr_render_profile.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    n = W * H * SPP
    sl = (Slice * n)()
    bo = (Bounce * (n * DEPTH))()
    film = np.zeros((H, W, 3))
    desc = cr.render_desc(W, H, SPP, max_bounce=7, estimator=cr.KOISHI, seed=3)
    assert lib.cr_render_profile(sc.h, C.byref(desc), DEPTH, C.byref(sl), C.byref(bo),
                                 film.ctypes.data_as(C.c_void_p)) == 0, lib.cr_last_error()
    cnt = np.frombuffer(sl, dtype=np.dtype([("bounce", "<u4"), ("L", "<f4", 3)]))
    b = cnt["bounce"]
    assert b.max() <= 8 and b.min() >= 0
    assert (b == 8).any() and (b < 8).any()
    L = cnt["L"].reshape(H, W, SPP, 3)
    ok = np.isfinite(L).all(-1)
    mean = np.where(ok[..., None], L, 0).sum(2) / np.maximum(ok.sum(2), 1)[..., None]
    np.testing.assert_allclose(mean, film, rtol=1e-4, atol=1e-5)
    rec = np.frombuffer(bo, dtype=np.dtype([("o", "<f4", 3), ("d", "<f4", 3), ("f", "<f4", 3), ("theta", "<f4"),
                                            ("L", "<f4", 3), ("shader", "<u4")])).reshape(n, DEPTH)
    # a record exists (non-zero ray direction) for every counted vertex, and
    # for one more where Russian roulette ended the loop (radiance.cu records
    # the vertex, then breaks before counting it)
    has = np.abs(rec["d"]).sum(-1) > 0
    nrec = has.sum(1)
    assert ((nrec == np.minimum(b, DEPTH)) | (nrec == np.minimum(b + 1, DEPTH))).all()
    assert (nrec == np.minimum(b + 1, DEPTH)).any()
    # each slice's radiance is its last counted record's (Russian roulette ends
    # the loop after the vertex is recorded but before it is counted)
    last = np.minimum(b, DEPTH) - 1
    sel = (b >= 1) & (b <= DEPTH) & np.isfinite(cnt["L"]).all(-1)
    # a camera ray that misses records nothing; otherwise L only grows
    assert (rec["L"][sel, last[sel]] <= cnt["L"][sel] * (1 + 1e-5) + 1e-5).all()
    sc.close()
