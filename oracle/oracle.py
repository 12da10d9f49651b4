"""Python access to the checkers under oracle/ (TEST INFRASTRUCTURE ONLY).

* :class:`OracleScene` wraps build/liboracle.so, the FP64 restatement of the
  reference's Radiance path (oracle.h documents both estimator modes).
* :func:`ref_run` runs _ref/cr_ref, the reference's own CPU code compiled from
  its sources with the harness in ref_harness/ (oracle/Makefile).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.  The product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "cr_ref")

KOISHI, MIS = 0, 1
AOV_NORMAL, AOV_VISIBILITY, AOV_HALFVECTOR = 4, 5, 6  # the reference's debug kernels
LAMBERT, GLOSSY, EMISSION, TRANSPARENT, BLACKHOLE, REFRACTION, GLASS, MIXED = range(8)
DIST = {"Beckmann": 0, "Cosine": 1}
FAC_CONSTANT, FAC_FRESNEL = 0, 1
LIGHT_SEED = 0x330E

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle oracle)")
        L = C.CDLL(LIB_PATH)
        P, U32, U64, I, D, F = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double, C.c_float
        sig = {
            "orc_scene_new": (P, []), "orc_scene_free": (None, [P]),
            "orc_add_shader": (I, [P, I, P]),
            "orc_add_point_light": (I, [P, P, P, D]),
            "orc_shade": (I, [P, I, I, P, P, P, I, P, P]),
            "orc_mis_eval": (None, [P, I, P, P, I, P, P]),
            "orc_mis_sample": (I, [P, I, P, I, P, P, P, P]),
            "orc_add_mesh": (I, [P, P, U32, P, P, U32, I]),
            "orc_add_sphere": (I, [P, P, F, I]),
            "orc_set_camera": (None, [P, P, P, P, F]), "orc_set_lens": (None, [P, I]),
            "orc_finalize": (I, [P, U64]), "orc_num_lights": (I, [P]),
            "orc_light_table": (D, [P, I, P]),
            "orc_trace": (None, [P, P, U64, P, P, P, P, P]),
            "orc_ray_triangle": (None, [P, P, I, I, P, P, P]),
            "orc_occluded": (None, [P, P, U64, P]),
            "orc_render": (I, [P, U32, U32, U32, U32, I, U64, U32, U32, U32, U32, U32, P, P, P]),
            "orc_bsdf_eval": (None, [I, I, P, P, P, P, P]),
            "orc_bsdf_sample": (None, [I, I, P, P, P, P, P, P]),
            "orc_seg_box": (I, [P, P, P]), "orc_sphere_hit": (I, [P, F, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _dist(props, owner):
    d = props.get("distribution")
    if d is None:
        raise ValueError(f"{owner} needs a distribution")
    kind = d[0]
    if kind not in DIST:
        raise ValueError(f"no such type: {kind}")
    rough = (d[1].get("roughness", 0.5) if len(d) > 1 else 0.5) if kind == "Beckmann" else 0.5
    return rough, DIST[kind]


def shader_params(cfg):
    """(type, params) for a reference-schema single-node shader config
    [Type, props] (shader.impl.cu:16-23: Lambert lambert.hpp:12-19;
    GlossyBSDF glossy.hpp:11-17 with beckmann.hpp:11-17 or cosine.hpp;
    Emission emission.hpp:12-20; Transparent transparent.hpp:11-15;
    Blackhole; RefractionBSDF refraction.hpp:11-19; GlassBSDF glass.hpp:11-21).
    Mixed nests shaders: use add_shader."""
    kind, props = cfg[0], (cfg[1] if len(cfg) > 1 else {})
    color = list(props.get("color", [1, 1, 1]))
    if kind == "Lambert":
        return LAMBERT, list(props.get("R", [1, 1, 1])) + color
    if kind == "GlossyBSDF":
        rough, dist = _dist(props, kind)
        return GLOSSY, color + [rough, dist]
    if kind == "Emission":
        return EMISSION, color + [props.get("strength", 2.0)]
    if kind == "Transparent":
        return TRANSPARENT, color
    if kind == "Blackhole":
        return BLACKHOLE, []
    if kind in ("RefractionBSDF", "GlassBSDF"):
        rough, dist = _dist(props, kind)
        return (GLASS if kind == "GlassBSDF" else REFRACTION), color + [float(props["ior"]), rough, dist]
    raise ValueError(f"unsupported shader {kind}")


def add_shader(h, cfg):
    """Adds cfg to the oracle scene h (nested Mixed children first,
    mixed.hpp:11-20 with constant.hpp / fresnel.hpp for fac); returns its id."""
    L = lib()
    if cfg[0] == "Mixed":
        props = cfg[1]
        fac = props["fac"]
        fk, fp = fac[0], (fac[1] if len(fac) > 1 else {})
        if fk == "Constant":
            fv = (FAC_CONSTANT, float(fp["value"]))
        elif fk == "Fresnel":
            fv = (FAC_FRESNEL, float(fp["ior"]))
        else:
            raise ValueError(f"no such type: {fk}")
        a, b = (add_shader(h, c) for c in props["shaders"][:2])
        params = np.asarray([fv[0], fv[1], a, b], np.float64)
        r = L.orc_add_shader(h, MIXED, _p(params))
    else:
        t, p = shader_params(cfg)
        params = np.asarray(p + [0.0], np.float64)  # bound: ctypes keeps only the address
        r = L.orc_add_shader(h, t, _p(params))
    assert r >= 0
    return r


class OracleScene:
    """FP64 oracle scene built from a scenes.SceneDesc (meshes first in group
    order, then spheres: the reference's primitive order for an import asset
    listed before the spheres)."""

    def __init__(self, desc, light_seed=LIGHT_SEED):
        L = lib()
        self.h = L.orc_scene_new()
        self.desc = desc
        ids = {}

        def sid(name):
            if name not in ids:
                ids[name] = add_shader(self.h, desc.shaders[name])
            return ids[name]

        self.prim_kind = []
        for g in desc.groups:
            v = np.ascontiguousarray(g.v, np.float32)
            n = np.ascontiguousarray(g.n, np.float32)
            f = np.ascontiguousarray(g.f, np.uint32)
            r = L.orc_add_mesh(self.h, _p(v), len(v), _p(n), _p(f), len(f), sid(g.name))
            assert r >= 0
            self.prim_kind.append(0)
        for s in desc.spheres:
            c = np.asarray(s["o"], np.float32)
            L.orc_add_sphere(self.h, _p(c), float(s["r"]), sid(s["shader"]))
            self.prim_kind.append(1)
        for pl in getattr(desc, "point_lights", []):
            p = np.asarray(pl["position"], np.float32)
            col = np.asarray(pl.get("color", [1, 1, 1]), np.float64)
            L.orc_add_point_light(self.h, _p(p), _p(col), float(pl.get("strength", 2.0)))
        cam = desc.camera
        pos = np.asarray(cam["position"], np.float32)
        tgt = np.asarray(cam["target"], np.float32)
        up = np.asarray(cam.get("upaxis", [0, 0, 1]), np.float32)
        L.orc_set_camera(self.h, _p(pos), _p(tgt), _p(up), float(cam.get("fovx", 90)))
        L.orc_set_lens(self.h, 1 if cam.get("lens", "pinhole") == "orthographic" else 0)
        L.orc_finalize(self.h, light_seed)

    def __del__(self):
        try:
            lib().orc_scene_free(self.h)
        except Exception:
            pass

    @property
    def n_lights(self):
        return lib().orc_num_lights(self.h)

    def light_table(self, l):
        pts = np.zeros((1024, 6), np.float32)
        pdf = lib().orc_light_table(self.h, l, _p(pts))
        return pts, pdf

    def trace(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        prim = np.zeros(n, np.int32)
        tri = np.zeros(n, np.int32)
        t, u, v = (np.zeros(n) for _ in range(3))
        lib().orc_trace(self.h, _p(rays), n, _p(prim), _p(tri), _p(t), _p(u), _p(v))
        return prim, tri, t, u, v

    def ray_triangle(self, ray, prim, tri):
        ray = np.ascontiguousarray(ray, np.float32)
        t, u, v = (np.zeros(1) for _ in range(3))
        lib().orc_ray_triangle(self.h, _p(ray), int(prim), int(tri), _p(t), _p(u), _p(v))
        return float(t[0]), float(u[0]), float(v[0])

    def occluded(self, segs):
        segs = np.ascontiguousarray(segs, np.float32)
        out = np.zeros(len(segs), np.uint8)
        lib().orc_occluded(self.h, _p(segs), len(segs), _p(out))
        return out

    def render(self, W, H, spp, max_bounce, estimator=KOISHI, seed=1, threads=0, window=None):
        x0, y0, x1, y1 = window or (0, 0, W, H)
        n = (x1 - x0) * (y1 - y0)
        s = np.zeros((n, 3))
        q = np.zeros((n, 3))
        c = np.zeros(n, np.uint32)
        r = lib().orc_render(self.h, W, H, spp, max_bounce, estimator, seed, threads, x0, y0, x1, y1,
                             _p(s), _p(q), _p(c))
        if r != 0:
            raise RuntimeError(f"orc_render returned {r}")
        shp = (y1 - y0, x1 - x0)
        return Film(s.reshape(*shp, 3), q.reshape(*shp, 3), c.reshape(shp))


class OracleShader:
    """One shader config (nested Mixed included) in an otherwise empty oracle
    scene, for Shader::execute with scripted draws."""

    def __init__(self, cfg):
        self.h = lib().orc_scene_new()
        self.id = add_shader(self.h, cfg)

    def __del__(self):
        try:
            lib().orc_scene_free(self.h)
        except Exception:
            pass

    def mis_eval(self, wo, wi, entering=True):
        """MIS-estimator f and pdf per (wo, wi) pair."""
        wo, wi = (np.ascontiguousarray(x, np.float64) for x in (wo, wi))
        f, pdf = np.zeros((len(wo), 3)), np.zeros(len(wo))
        L, ff, pp = lib(), np.zeros(3), np.zeros(1)
        for i in range(len(wo)):
            L.orc_mis_eval(self.h, self.id, _p(wo[i]), _p(wi[i]), int(entering), _p(ff), _p(pp))
            f[i], pdf[i] = ff, pp[0]
        return f, pdf

    def mis_sample(self, wo, u, entering=True):
        """MIS-estimator samples per wo with u = (u1, u2, selection): wi,
        weight, pdf, delta."""
        wo, u = (np.ascontiguousarray(x, np.float64) for x in (wo, u))
        n = len(wo)
        wi, w, pdf, delta = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n, bool)
        L, a, b, pp = lib(), np.zeros(3), np.zeros(3), np.zeros(1)
        for i in range(n):
            delta[i] = L.orc_mis_sample(self.h, self.id, _p(wo[i]), int(entering), _p(u[i]), _p(a), _p(b), _p(pp)) == 1
            wi[i], w[i], pdf[i] = a, b, pp[0]
        return wi, w, pdf, delta

    def execute(self, target, wo, u, wi=None):
        """Per sample: f, wi, emission, draws used (target 0 eval, 1 sample)."""
        wo = np.ascontiguousarray(wo, np.float64)
        n = len(wo)
        u = np.ascontiguousarray(np.asarray(u, np.float64).reshape(n, -1))
        wi = np.zeros((n, 3)) if wi is None else np.array(wi, np.float64, order="C", copy=True)
        f, em, used = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n, np.int32)
        L = lib()
        ff, ee = np.zeros(3), np.zeros(3)
        for i in range(n):
            w = np.ascontiguousarray(wi[i])
            used[i] = L.orc_shade(self.h, self.id, target, _p(wo[i]), _p(w), _p(u[i]), u.shape[1], _p(ff), _p(ee))
            f[i], em[i], wi[i] = ff, ee, w
        return f, wi, em, used


def bsdf_eval(estimator, cfg, wo, wi):
    t, p = shader_params(cfg)
    f = np.zeros(3)
    pdf = np.zeros(1)
    params, a, b = (np.asarray(x, np.float64) for x in (p, wo, wi))
    lib().orc_bsdf_eval(estimator, t, _p(params), _p(a), _p(b), _p(f), _p(pdf))
    return f, float(pdf[0])


def bsdf_sample(estimator, cfg, wo, u):
    t, p = shader_params(cfg)
    wi, w, pdf = np.zeros(3), np.zeros(3), np.zeros(1)
    params, a, b = (np.asarray(x, np.float64) for x in (p, wo, u))
    lib().orc_bsdf_sample(estimator, t, _p(params), _p(a), _p(b), _p(wi), _p(w), _p(pdf))
    return wi, w, float(pdf[0])


def seg_box(seg7, bmin, bmax):
    a, b, c = (np.asarray(x, np.float32) for x in (seg7, bmin, bmax))
    return bool(lib().orc_seg_box(_p(a), _p(b), _p(c)))


def sphere_hit(center, r, ray6):
    t = np.zeros(1)
    c, ray = np.asarray(center, np.float32), np.asarray(ray6, np.float32)
    h = lib().orc_sphere_hit(_p(c), float(r), _p(ray), _p(t))
    return bool(h), float(t[0])


class Film:
    """Per-pixel sums over finite samples, as CPUMulticoreTracer::execute
    averages them (src/core/tracer/cpuMulticore.cu:53-64)."""

    def __init__(self, s, q, c):
        self.sum, self.sumsq, self.count = s, q, c

    @property
    def mean(self):
        return self.sum / np.maximum(self.count, 1)[..., None]

    @property
    def var_of_mean(self):
        c = np.maximum(self.count, 1)[..., None].astype(np.float64)
        m = self.sum / c
        var = np.maximum(self.sumsq / c - m * m, 0.0) * c / np.maximum(c - 1, 1)
        return var / c


def read_crf(path):
    with open(path, "rb") as fh:
        d = fh.read()
    assert d[:4] == b"CRF1"
    W, H, spp = struct.unpack_from("<III", d, 4)
    off = 16
    s = np.frombuffer(d, "<f8", W * H * 3, off).reshape(H, W, 3)
    off += W * H * 24
    q = np.frombuffer(d, "<f8", W * H * 3, off).reshape(H, W, 3)
    off += W * H * 24
    c = np.frombuffer(d, "<u4", W * H, off).reshape(H, W)
    return Film(s.copy(), q.copy(), c.copy())


def ref_available():
    return os.path.exists(REF_BIN)


def ref_run(*args, cwd=None, timeout=600):
    """Run the compiled reference harness; returns its CompletedProcess."""
    if not ref_available():
        raise RuntimeError(f"reference harness missing: {REF_BIN} (run make -C oracle ref)")
    return subprocess.run([REF_BIN, *map(str, args)], cwd=cwd, capture_output=True, text=True,
                          timeout=timeout, check=True)
