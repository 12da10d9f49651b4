"""Seeded synthetic scenes in the reference's JSON scene schema.

Every scene is written as a reference-schema JSON document
(``{"scene": {"camera", "assets", "shaders"}, "tracer": [...]}``, the schema read
by src/core/renderer/renderer.hpp:17-23 and src/core/meta/scene.cu:18-219 of
xlnx/cuda-raytracer) plus one mesh file named by an ``["import", {"path"}]``
asset.  Meshes are split per material, one group per material name, the way the
reference's importer splits an imported scene into one Mesh per material
(src/core/primitive/mesh.cu:332-402).

Mesh file format ``CRM1`` (little-endian)::

    char[4] "CRM1"; u32 n_groups
    per group: u32 name_len; char name[name_len]; u32 nv; u32 nt;
               f32 v[nv*3]; f32 n[nv*3]; u32 idx[nt*3]

Geometry conventions shared by all scenes:
  * z is up; the Cornell-style box is 5.55 units wide (x) and tall (z).
  * the whole scene is rotated 30 degrees about z so that no flat face has a
    normal parallel to +-y: the reference builds its shading frame from
    cross(n, (0,1,0)) (src/core/meta/scene.hpp:48-50), which is NaN for such
    faces and silently drops their samples.
  * lights are quads of two equal-area triangles.
"""
from __future__ import annotations

import json
import math
import os
import struct
from dataclasses import dataclass, field

import numpy as np

S = 5.55          # box width/height
FRONT = -2.6      # y of the wall behind the camera (the box is closed)
ROT_DEG = 30.0    # rotation about z around the box centre


@dataclass
class Group:
    name: str
    v: np.ndarray          # (nv, 3) float32
    n: np.ndarray          # (nv, 3) float32
    f: np.ndarray          # (nt, 3) uint32


@dataclass
class SceneDesc:
    groups: list = field(default_factory=list)
    spheres: list = field(default_factory=list)     # dicts {o, r, shader}
    shaders: dict = field(default_factory=dict)     # name -> [Type, props]
    point_lights: list = field(default_factory=list)  # dicts {position, color, strength}
    camera: dict = field(default_factory=dict)
    width: int = 256
    height: int = 256
    spp: int = 64
    max_bounce: int = 7
    name: str = "scene"

    @property
    def n_triangles(self) -> int:
        return int(sum(len(g.f) for g in self.groups))


# ----------------------------------------------------------------------------
# small geometry helpers

def _rot_matrix(deg: float) -> np.ndarray:
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


_PIVOT = np.array([S / 2, S / 2, 0.0])


def _rot_points(p, deg=ROT_DEG):
    p = np.asarray(p, dtype=np.float64)
    return (p - _PIVOT) @ _rot_matrix(deg).T + _PIVOT


def _rot_dirs(d, deg=ROT_DEG):
    return np.asarray(d, dtype=np.float64) @ _rot_matrix(deg).T


def quad(p0, p1, p2, p3, normal):
    """Two triangles (p0,p1,p2), (p0,p2,p3) with separate vertices and a flat normal."""
    v = np.array([p0, p1, p2, p3], dtype=np.float64)
    n = np.tile(np.asarray(normal, dtype=np.float64), (4, 1))
    f = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32)
    return v, n, f


def _merge(parts):
    vs, ns, fs, off = [], [], [], 0
    for v, n, f in parts:
        vs.append(v)
        ns.append(n)
        fs.append(f + off)
        off += len(v)
    return np.concatenate(vs), np.concatenate(ns), np.concatenate(fs).astype(np.uint32)


def _finish(name, v, n, f, rotate=True):
    if rotate:
        v = _rot_points(v)
        n = _rot_dirs(n)
    n = n / np.linalg.norm(n, axis=1, keepdims=True)
    return Group(name, v.astype(np.float32), n.astype(np.float32), np.ascontiguousarray(f, dtype=np.uint32))


def box_groups(light_x=(2.125, 3.425), light_y=(1.9, 2.95), light_z=S - 0.25, with_light=True,
               light_name="light"):
    """Closed box of 10 quads (floor, ceiling, back and front walls split in two;
    left and right walls whole) plus a light panel hanging 0.25 below the
    ceiling.  Normals face inward.  The panel hangs clear of the ceiling because
    the reference's 1024-point light tables include points outside the light's
    faces (src/core/primitive/mesh.hpp:71-73); a panel flush with the ceiling
    would put such points a hair away from lit ceiling points and make the
    reference's estimator heavy-tailed."""
    lx0, lx1 = light_x
    ly0, ly1 = light_y
    y0, y1, zc, ym, xm = FRONT, S, S, 1.5, S / 2
    white = [
        quad((0, y0, 0), (S, y0, 0), (S, ym, 0), (0, ym, 0), (0, 0, 1)),            # floor front
        quad((0, ym, 0), (S, ym, 0), (S, y1, 0), (0, y1, 0), (0, 0, 1)),            # floor back
        quad((0, y0, zc), (0, ym, zc), (S, ym, zc), (S, y0, zc), (0, 0, -1)),       # ceiling front
        quad((0, ym, zc), (0, y1, zc), (S, y1, zc), (S, ym, zc), (0, 0, -1)),       # ceiling back
        quad((0, y1, 0), (xm, y1, 0), (xm, y1, zc), (0, y1, zc), (0, -1, 0)),       # back wall left
        quad((xm, y1, 0), (S, y1, 0), (S, y1, zc), (xm, y1, zc), (0, -1, 0)),       # back wall right
        quad((0, y0, 0), (0, y0, zc), (xm, y0, zc), (xm, y0, 0), (0, 1, 0)),        # front wall left
        quad((xm, y0, 0), (xm, y0, zc), (S, y0, zc), (S, y0, 0), (0, 1, 0)),        # front wall right
    ]
    red = [quad((0, y0, 0), (0, y1, 0), (0, y1, zc), (0, y0, zc), (1, 0, 0))]
    green = [quad((S, y0, 0), (S, y0, zc), (S, y1, zc), (S, y1, 0), (-1, 0, 0))]
    groups = [
        _finish("white", *_merge(white)),
        _finish("red", *_merge(red)),
        _finish("green", *_merge(green)),
    ]
    if with_light:
        lq = quad((lx0, ly0, light_z), (lx0, ly1, light_z), (lx1, ly1, light_z), (lx1, ly0, light_z), (0, 0, -1))
        groups.append(_finish(light_name, *lq))
    return groups


def box_shaders(strength=50.0):
    return {
        "white": ["Lambert", {"R": [0.73, 0.73, 0.73], "color": [1, 1, 1]}],
        "red": ["Lambert", {"R": [0.65, 0.05, 0.05], "color": [1, 1, 1]}],
        "green": ["Lambert", {"R": [0.12, 0.45, 0.15], "color": [1, 1, 1]}],
        "light": ["Emission", {"color": [1, 1, 1], "strength": float(strength)}],
    }


def box_camera(fovx=40.0):
    pos = _rot_points([S / 2, FRONT + 0.1, S / 2])
    tgt = _rot_dirs([0.0, 1.0, 0.0])
    return {"lens": "pinhole", "fovx": float(fovx), "position": [float(x) for x in pos],
            "target": [float(x) for x in tgt], "upaxis": [0.0, 0.0, 1.0]}


# ----------------------------------------------------------------------------
# icosphere + value noise

def icosphere(level: int):
    """Unit icosphere; the 4 children of face f after one split are 4f..4f+3,
    so face f at level L belongs to base face f // 4**L."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        e = np.stack([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)], 1).reshape(-1, 2)
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uk, inv = np.unique(key, return_inverse=True)
        ua, ub = uk // (len(v) + 1), uk % (len(v) + 1)
        mid = v[ua] + v[ub]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mid_idx = (len(v) + np.arange(len(uk)))[inv].reshape(-1, 3)
        v = np.concatenate([v, mid])
        ab, bc, ca = mid_idx[:, 0], mid_idx[:, 1], mid_idx[:, 2]
        f = np.stack([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1),
                      np.stack([ca, bc, c], 1), np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3)
    return v, f


def value_noise(p: np.ndarray, seed: int, octaves: int = 4, freq: float = 2.0) -> np.ndarray:
    """Fractal lattice value noise in [-1, 1] (smoothstep-interpolated)."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, 4096)
    perm = rng.permutation(4096)
    out = np.zeros(len(p))
    amp, norm, f = 1.0, 0.0, freq
    for o in range(octaves):
        q = p * f + 17.31 * o
        i0 = np.floor(q).astype(np.int64)
        w = q - i0
        w = w * w * (3 - 2 * w)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    ix, iy, iz = i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz
                    h = perm[(ix * 73856093 ^ iy * 19349663 ^ iz * 83492791) & 4095]
                    wt = (w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1]) * \
                         (w[:, 2] if dz else 1 - w[:, 2])
                    acc += wt * table[h]
        out += amp * acc
        norm += amp
        amp *= 0.5
        f *= 2.0
    return out / norm


def smooth_normals(v, f):
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return n


def displaced_icosphere(level, seed, center, radius, amp=0.15):
    v, f = icosphere(level)
    d = value_noise(v, seed)
    v = v * (radius * (1.0 + amp * d))[:, None] + np.asarray(center)[None, :]
    n = smooth_normals(v, f)
    return v, n, f


def split_groups(v, n, f, face_group, names, rotate=True):
    """One Group per material id, each with its own compacted vertex set."""
    out = []
    for gi, name in enumerate(names):
        sel = np.nonzero(face_group == gi)[0]
        if len(sel) == 0:
            continue
        ff = f[sel]
        used, inv = np.unique(ff.reshape(-1), return_inverse=True)
        out.append(_finish(name, v[used], n[used], inv.reshape(-1, 3), rotate=rotate))
    return out


def _random_material(rng, name_prefix, i, alpha_range=(0.05, 0.8)):
    if rng.uniform() < 0.5:
        alb = rng.uniform(0.2, 0.9, 3)
        return f"{name_prefix}{i:02d}", ["Lambert", {"R": [float(x) for x in alb], "color": [1, 1, 1]}]
    a = rng.uniform(*alpha_range)
    col = rng.uniform(0.4, 0.9, 3)
    return f"{name_prefix}{i:02d}", ["GlossyBSDF", {"distribution": ["Beckmann", {"roughness": float(a)}],
                                                    "color": [float(x) for x in col]}]


# ----------------------------------------------------------------------------
# the configurations

def config0(width=256, height=256, spp=64) -> SceneDesc:
    """Box + ceiling light + Beckmann sphere + Lambert sphere (the small case that
    the reference's CPU tracer renders in seconds)."""
    sh = box_shaders(50.0)
    sh["glossy"] = ["GlossyBSDF", {"distribution": ["Beckmann", {"roughness": 0.3}],
                                   "color": [0.545, 0.463, 0.427]}]
    sh["ball"] = ["Lambert", {"R": [0.73, 0.73, 0.73], "color": [1, 1, 1]}]
    spheres = [
        {"o": [float(x) for x in _rot_points([1.85, 1.7, 1.0])], "r": 1.0, "shader": "glossy"},
        {"o": [float(x) for x in _rot_points([3.7, 3.5, 1.0])], "r": 1.0, "shader": "ball"},
    ]
    return SceneDesc(groups=box_groups(), spheres=spheres, shaders=sh, camera=box_camera(),
                     width=width, height=height, spp=spp, max_bounce=7, name="config0")


def config0_ortho(width=256, height=256, spp=64) -> SceneDesc:
    """Config 0 seen through the reference's OrthographicLens (lens.hpp:40-53):
    parallel rays from a 4-unit-wide plane at the camera position."""
    d = config0(width, height, spp)
    d.camera = dict(d.camera, lens="orthographic")
    d.name = "config0_ortho"
    return d


def config_materials(width=256, height=256, spp=64, cosine=True, point_light=True) -> SceneDesc:
    """The box with the reference's remaining shaders and a point light:
    GlassBSDF, RefractionBSDF, Transparent, Blackhole, Mixed over a Fresnel
    and over a Constant fac (one with a Cosine GlossyBSDF; `cosine=False`:
    a Beckmann one, which the MIS estimator takes), lit by the ceiling panel
    and by a pointLight (the first light in the list; `point_light=False`
    leaves it out)."""
    sh = box_shaders(50.0)
    beck = lambda a: ["Beckmann", {"roughness": a}]
    sh["glass"] = ["GlassBSDF", {"ior": 1.5, "distribution": beck(0.2), "color": [0.95, 0.97, 1.0]}]
    sh["coat"] = ["Mixed", {"fac": ["Fresnel", {"ior": 1.5}],
                            "shaders": [["Lambert", {"R": [0.6, 0.3, 0.2], "color": [1, 1, 1]}],
                                        ["GlossyBSDF", {"distribution": beck(0.15), "color": [1, 1, 1]}]]}]
    sh["water"] = ["RefractionBSDF", {"ior": 1.33, "distribution": beck(0.25), "color": [0.9, 0.95, 1.0]}]
    sh["veil"] = ["Transparent", {"color": [0.85, 0.9, 0.7]}]
    sh["hole"] = ["Blackhole", {}]
    sh["blend"] = ["Mixed", {"fac": ["Constant", {"value": 0.35}],
                             "shaders": [["Lambert", {"R": [0.2, 0.5, 0.7], "color": [1, 1, 1]}],
                                         ["GlossyBSDF", {"distribution": ["Cosine", {}] if cosine else beck(0.4),
                                                         "color": [0.8, 0.8, 0.6]}]]}]
    place = [("glass", [1.6, 1.6, 1.0], 1.0), ("coat", [3.9, 3.6, 1.0], 1.0), ("water", [3.8, 1.0, 0.6], 0.6),
             ("veil", [1.4, 3.9, 0.8], 0.8), ("hole", [2.8, 4.7, 2.8], 0.4), ("blend", [2.6, 2.6, 0.45], 0.45)]
    spheres = [{"o": [float(x) for x in _rot_points(c)], "r": r, "shader": n} for n, c, r in place]
    lights = [{"position": [float(x) for x in _rot_points([2.0, 2.0, 4.2])], "color": [1.0, 0.9, 0.8],
               "strength": 1.5}] if point_light else []
    return SceneDesc(groups=box_groups(), spheres=spheres, shaders=sh, camera=box_camera(), point_lights=lights,
                     width=width, height=height, spp=spp, max_bounce=7, name="materials")


def config1(level=8, seed=1, width=1024, height=768, spp=256) -> SceneDesc:
    """Displaced icosphere (20*4**level triangles) inside the box.  Materials are
    drawn per icosahedron patch (20 patches), 50 % Lambert albedo U[0.2,0.9]^3 and
    50 % Beckmann roughness U[0.05,0.8], so that every material group is a
    spatially compact mesh for the reference's per-mesh BVH."""
    rng = np.random.default_rng(seed)
    sh = box_shaders(50.0)
    names = []
    for i in range(20):
        nm, cfg = _random_material(rng, "m", i)
        names.append(nm)
        sh[nm] = cfg
    v, n, f = displaced_icosphere(level, seed, center=(S / 2, 1.7, 1.75), radius=1.45)
    patch = np.arange(len(f)) // (4 ** level)
    groups = box_groups() + split_groups(v, n, f, patch, names)
    return SceneDesc(groups=groups, shaders=sh, camera=box_camera(), width=width, height=height,
                     spp=spp, max_bounce=7, name=f"config1_l{level}")


def _boxes(rng, count, lo, hi):
    """`count` axis-aligned boxes (12 triangles each, flat outward normals) with
    random centres in [lo, hi] and edge lengths U[0.05, 0.4]."""
    if count <= 0:
        return np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3), np.uint32)
    c = rng.uniform(lo, hi, (count, 3))
    h = rng.uniform(0.025, 0.2, (count, 3))
    # 6 faces x 4 corners: (axis, sign) faces with corner offsets in the other two axes
    vs, ns = [], []
    for axis in range(3):
        a1, a2 = (axis + 1) % 3, (axis + 2) % 3
        for sign in (-1.0, 1.0):
            nrm = np.zeros(3)
            nrm[axis] = sign
            for s1, s2 in ((-1, -1), (1, -1), (1, 1), (-1, 1)) if sign > 0 else ((-1, -1), (-1, 1), (1, 1), (1, -1)):
                off = np.zeros((count, 3))
                off[:, axis] = sign * h[:, axis]
                off[:, a1] = s1 * h[:, a1]
                off[:, a2] = s2 * h[:, a2]
                vs.append(c + off)
                ns.append(np.tile(nrm, (count, 1)))
    v = np.stack(vs, 1).reshape(-1, 3)      # box-major: 24 vertices per box
    n = np.stack(ns, 1).reshape(-1, 3)
    quad = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    per_box = np.concatenate([quad + 4 * q for q in range(6)])             # 12 x 3
    f = (per_box[None, :, :] + 24 * np.arange(count, dtype=np.uint32)[:, None, None]).reshape(-1, 3)
    return v, n, f.astype(np.uint32)


def config2_params(index, seed=2):
    """Size of scene `index` of the batched workload: triangle count log-uniform in
    [1e3, 2e6], square resolution log-uniform in 128..1024 (multiple of 16), spp
    from {16, 32, 64, 128, 256}, 1-4 lights of emission U[10, 80]."""
    rng = np.random.default_rng(seed * 100003 + index)
    tris = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e6)))))
    side = int(round(math.exp(rng.uniform(math.log(128), math.log(1024))) / 16.0)) * 16
    spp = int(rng.choice([16, 32, 64, 128, 256]))
    lights = int(rng.integers(1, 5))
    return {"triangles": tris, "width": side, "height": side, "spp": spp, "lights": lights, "rng": rng}


def config2(index, seed=2, max_triangles=None) -> SceneDesc:
    """Scene `index` of the batched workload: a displaced icosphere of the largest
    subdivision level below the drawn triangle count, topped up with random
    boxes, inside the box with 1-4 ceiling lights; 8 materials (50 % Lambert,
    50 % Beckmann).  `max_triangles` caps the count (small test batches)."""
    p = config2_params(index, seed)
    rng = p["rng"]
    target = p["triangles"] if max_triangles is None else min(p["triangles"], max_triangles)
    level = max(0, int(math.floor(math.log(max(target, 20) / 20.0, 4))))
    sh = box_shaders(50.0)
    del sh["light"]
    names = []
    for i in range(8):
        nm, cfg = _random_material(rng, "b", i)
        names.append(nm)
        sh[nm] = cfg
    v, n, f = displaced_icosphere(level, seed * 1000 + index, center=(S / 2, 1.7, 1.6), radius=1.2)
    groups = box_groups(with_light=False)
    patch = (np.arange(len(f)) // (4 ** level)) % len(names)
    groups += split_groups(v, n, f, patch, names)
    nbox = max(0, (target - len(f)) // 12)
    bv, bn, bf = _boxes(rng, nbox, (0.3, -2.2, 0.05), (S - 0.3, S - 0.3, S - 1.0))
    if nbox:
        bmat = rng.integers(0, len(names), nbox)
        fm = np.repeat(bmat, 12)
        groups += split_groups(bv, bn, bf, fm, names)
    for li in range(p["lights"]):
        lx, ly = rng.uniform(0.8, S - 1.6), rng.uniform(-1.5, S - 1.6)
        wx, wy = rng.uniform(0.4, 1.2), rng.uniform(0.4, 1.2)
        z = S - 0.25
        lq = quad((lx, ly, z), (lx, ly + wy, z), (lx + wx, ly + wy, z), (lx + wx, ly, z), (0, 0, -1))
        groups.append(_finish(f"light{li}", *lq))
        sh[f"light{li}"] = ["Emission", {"color": [1, 1, 1], "strength": float(rng.uniform(10, 80))}]
    merged = {}
    for g in groups:
        if g.name in merged:
            a = merged[g.name]
            merged[g.name] = Group(g.name, np.concatenate([a.v, g.v]), np.concatenate([a.n, g.n]),
                                   np.concatenate([a.f, g.f + len(a.v)]).astype(np.uint32))
        else:
            merged[g.name] = g
    return SceneDesc(groups=list(merged.values()), shaders=sh, camera=box_camera(), width=p["width"],
                     height=p["height"], spp=p["spp"], max_bounce=7, name=f"config2_{index}")


def _rotation(rng):
    """Uniformly random rotation matrix (QR of a Gaussian matrix, sign-fixed)."""
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def config4(level=8, seed=4, instances=16, bases=4, width=3840, height=2160, spp=1024) -> SceneDesc:
    """Large combined scene: `instances` copies of `bases` displaced icospheres
    (20*4**level triangles each, 1.31M at level 8) under random rigid
    transforms, flattened into one triangle set on a 4 x 4 grid over the box
    floor; 6 ceiling lights of emission U[10, 80]; 16 materials (50 % Lambert,
    50 % Beckmann roughness U[0.05, 0.8]); depth 12 (max_bounce 11)."""
    rng = np.random.default_rng(seed)
    sh = box_shaders(50.0)
    del sh["light"]
    names = []
    for i in range(16):
        nm, cfg = _random_material(rng, "c", i)
        names.append(nm)
        sh[nm] = cfg
    base = [displaced_icosphere(level, seed * 100 + b, center=(0.0, 0.0, 0.0), radius=0.55) for b in range(bases)]
    groups = box_groups(with_light=False)
    xs = np.linspace(0.75, S - 0.75, 4)
    ys = np.linspace(-1.6, S - 0.9, 4)
    for k in range(instances):
        v, n, f = base[k % bases]
        R = _rotation(rng)
        c = np.array([xs[k % 4], ys[(k // 4) % 4], rng.uniform(0.6, 1.6)])
        vi = v @ R.T + c[None, :]
        ni = n @ R.T
        patch = (np.arange(len(f)) // (4 ** level) + k) % len(names)
        groups += split_groups(vi, ni, f, patch, names)
    for li in range(6):
        lx, ly = rng.uniform(0.5, S - 1.5), rng.uniform(-2.0, S - 1.5)
        wx, wy = rng.uniform(0.4, 1.0), rng.uniform(0.4, 1.0)
        z = S - 0.25
        lq = quad((lx, ly, z), (lx, ly + wy, z), (lx + wx, ly + wy, z), (lx + wx, ly, z), (0, 0, -1))
        groups.append(_finish(f"light{li}", *lq))
        sh[f"light{li}"] = ["Emission", {"color": [1, 1, 1], "strength": float(rng.uniform(10, 80))}]
    merged = {}
    for g in groups:
        merged.setdefault(g.name, []).append(g)
    out = []
    for name, gs in merged.items():
        if len(gs) == 1:
            out.append(gs[0])
            continue
        offs = np.cumsum([0] + [len(g.v) for g in gs[:-1]])
        out.append(Group(name, np.concatenate([g.v for g in gs]), np.concatenate([g.n for g in gs]),
                         np.concatenate([g.f + o for g, o in zip(gs, offs)]).astype(np.uint32)))
    return SceneDesc(groups=out, shaders=sh, camera=box_camera(), width=width, height=height, spp=spp,
                     max_bounce=11, name=f"config4_l{level}")


def config3(level=7, seed=3, width=1024, height=1024, spp=64, diffuse=False) -> SceneDesc:
    """Occluded light: the box is split by a wall at y=2.6 with a 0.4x0.4 aperture;
    a single 0.3x0.3 light of strength 400 hangs on the far side; three displaced
    icospheres (one at `level`, two at `level - 1`: ~492k triangles at level 7)
    with Beckmann roughness U[0.05,0.5] are the receivers on the camera side
    (`diffuse`: Lambert receivers of albedo 0.7 instead)."""
    rng = np.random.default_rng(seed)
    sh = box_shaders(400.0)
    names = []
    for i in range(20):
        nm, cfg = _random_material(rng, "g", i, alpha_range=(0.05, 0.5))
        if cfg[0] == "Lambert":
            a = rng.uniform(0.05, 0.5)
            cfg = ["GlossyBSDF", {"distribution": ["Beckmann", {"roughness": float(a)}],
                                  "color": [0.8, 0.8, 0.8]}]
        if diffuse:  # the same geometry with Lambert receivers (no glossy caustics)
            cfg = ["Lambert", {"R": [0.7, 0.7, 0.7], "color": [1, 1, 1]}]
        names.append(nm)
        sh[nm] = cfg
    wall_y = 2.6
    ax0, ax1, az0, az1 = S / 2 - 0.2, S / 2 + 0.2, 2.6, 3.0
    groups = box_groups(with_light=False)
    parts = []
    for side, nrm in ((wall_y - 1e-3, (0, -1, 0)), (wall_y + 1e-3, (0, 1, 0))):
        y = side
        rects = [(0, ax0, 0, S), (ax1, S, 0, S), (ax0, ax1, 0, az0), (ax0, ax1, az1, S)]
        for x0, x1, z0, z1 in rects:
            if nrm[1] < 0:
                parts.append(quad((x0, y, z0), (x0, y, z1), (x1, y, z1), (x1, y, z0), nrm))
            else:
                parts.append(quad((x0, y, z0), (x1, y, z0), (x1, y, z1), (x0, y, z1), nrm))
    groups.append(_finish("divider", *_merge(parts)))
    sh["divider"] = ["Lambert", {"R": [0.73, 0.73, 0.73], "color": [1, 1, 1]}]
    lx, ly, lz = S / 2, 4.6, S - 0.25
    lq = quad((lx - .15, ly - .15, lz), (lx - .15, ly + .15, lz), (lx + .15, ly + .15, lz),
              (lx + .15, ly - .15, lz), (0, 0, -1))
    groups.append(_finish("light", *lq))
    # receivers: one displaced icosphere at `level` and two at `level - 1`
    for ci, (cen, rad, lv) in enumerate((((S / 2, 0.4, 1.3), 1.2, level), ((1.0, -1.3, 0.8), 0.7, level - 1),
                                         ((4.5, -1.0, 0.9), 0.8, level - 1))):
        v, n, f = displaced_icosphere(lv, seed + ci, center=cen, radius=rad)
        patch = np.arange(len(f)) // (4 ** lv)
        groups += split_groups(v, n, f, patch, names)
    # the receivers share one material palette: one group per material
    merged = {}
    for g in groups:
        if g.name in merged:
            a = merged[g.name]
            merged[g.name] = Group(g.name, np.concatenate([a.v, g.v]), np.concatenate([a.n, g.n]),
                                   np.concatenate([a.f, g.f + len(a.v)]).astype(np.uint32))
        else:
            merged[g.name] = g
    groups = list(merged.values())
    return SceneDesc(groups=groups, shaders=sh, camera=box_camera(), width=width, height=height,
                     spp=spp, max_bounce=7, name=f"config3_l{level}")


# ----------------------------------------------------------------------------
# I/O

def write_crm(path, groups):
    with open(path, "wb") as fh:
        fh.write(b"CRM1")
        fh.write(struct.pack("<I", len(groups)))
        for g in groups:
            nb = g.name.encode()
            fh.write(struct.pack("<I", len(nb)))
            fh.write(nb)
            fh.write(struct.pack("<II", len(g.v), len(g.f)))
            fh.write(np.ascontiguousarray(g.v, dtype="<f4").tobytes())
            fh.write(np.ascontiguousarray(g.n, dtype="<f4").tobytes())
            fh.write(np.ascontiguousarray(g.f, dtype="<u4").tobytes())


def read_crm(path):
    groups = []
    with open(path, "rb") as fh:
        data = fh.read()
    assert data[:4] == b"CRM1"
    (ng,), off = struct.unpack_from("<I", data, 4), 8
    for _ in range(ng):
        (ln,) = struct.unpack_from("<I", data, off)
        off += 4
        name = data[off:off + ln].decode()
        off += ln
        nv, nt = struct.unpack_from("<II", data, off)
        off += 8
        v = np.frombuffer(data, "<f4", nv * 3, off).reshape(nv, 3)
        off += nv * 12
        n = np.frombuffer(data, "<f4", nv * 3, off).reshape(nv, 3)
        off += nv * 12
        f = np.frombuffer(data, "<u4", nt * 3, off).reshape(nt, 3)
        off += nt * 12
        groups.append(Group(name, v, n, f))
    return groups


def write_obj(path, groups):
    """Wavefront OBJ with one `usemtl` block per group (for importer tests)."""
    with open(path, "w") as fh:
        base = 1
        for g in groups:
            fh.write(f"o {g.name}\nusemtl {g.name}\n")
            for p in g.v:
                fh.write(f"v {p[0]:.9g} {p[1]:.9g} {p[2]:.9g}\n")
            for q in g.n:
                fh.write(f"vn {q[0]:.9g} {q[1]:.9g} {q[2]:.9g}\n")
            for t in g.f:
                a, b, c = (int(x) + base for x in t)
                fh.write(f"f {a}//{a} {b}//{b} {c}//{c}\n")
            base += len(g.v)


def write_ply(path, groups, encoding="binary_little_endian", normals=True, quads=False, extras=False):
    """Stanford PLY of all groups merged into one mesh (PLY carries no
    materials; an importer names it "DefaultMaterial").  encoding: "ascii",
    "binary_little_endian" or "binary_big_endian".  quads: a triangle
    (a, b, c) followed by (a, c, d) is written as the 4-gon (a, b, c, d), which
    a reader fans back into the same two triangles.  extras: add per-vertex
    colours and an "edge" element, which a reader must skip."""
    v = np.concatenate([g.v for g in groups]).astype(np.float32)
    n = np.concatenate([g.n for g in groups]).astype(np.float32)
    offs = np.cumsum([0] + [len(g.v) for g in groups[:-1]])
    f = np.concatenate([g.f.astype(np.int64) + o for g, o in zip(groups, offs)])
    polys = []
    i = 0
    while i < len(f):
        a, b, c = f[i]
        if quads and i + 1 < len(f) and f[i + 1][0] == a and f[i + 1][1] == c:
            polys.append((a, b, c, f[i + 1][2]))
            i += 2
        else:
            polys.append((a, b, c))
            i += 1
    hdr = ["ply", f"format {encoding} 1.0", "comment written by the cuda-raytracer_b200 scene generator",
           f"element vertex {len(v)}", "property float x", "property float y", "property float z"]
    if normals:
        hdr += ["property float nx", "property float ny", "property float nz"]
    if extras:
        hdr += ["property uchar red", "property uchar green", "property uchar blue"]
    hdr += [f"element face {len(polys)}", "property list uchar int vertex_indices"]
    if extras:
        hdr += ["element edge 1", "property int vertex1", "property int vertex2"]
    hdr += ["end_header"]
    with open(path, "wb") as fh:
        fh.write(("\n".join(hdr) + "\n").encode())
        if encoding == "ascii":
            for k in range(len(v)):
                row = [f"{x:.9g}" for x in v[k]] + ([f"{x:.9g}" for x in n[k]] if normals else [])
                row += ["200", "100", "50"] if extras else []
                fh.write((" ".join(row) + "\n").encode())
            for p in polys:
                fh.write((f"{len(p)} " + " ".join(str(int(x)) for x in p) + "\n").encode())
            if extras:
                fh.write(b"0 1\n")
            return
        e = "<" if encoding == "binary_little_endian" else ">"
        cols = [v] + ([n] if normals else [])
        vdt = [("x", e + "f4"), ("y", e + "f4"), ("z", e + "f4")]
        if normals:
            vdt += [("nx", e + "f4"), ("ny", e + "f4"), ("nz", e + "f4")]
        if extras:
            vdt += [("r", "u1"), ("g", "u1"), ("b", "u1")]
        rec = np.zeros(len(v), dtype=vdt)
        rec["x"], rec["y"], rec["z"] = v[:, 0], v[:, 1], v[:, 2]
        if normals:
            rec["nx"], rec["ny"], rec["nz"] = n[:, 0], n[:, 1], n[:, 2]
        if extras:
            rec["r"], rec["g"], rec["b"] = 200, 100, 50
        fh.write(rec.tobytes())
        for p in polys:
            fh.write(np.uint8(len(p)).tobytes() + np.asarray(p, dtype=e + "i4").tobytes())
        if extras:
            fh.write(np.asarray([0, 1], dtype=e + "i4").tobytes())


def scene_json(desc: SceneDesc, mesh_path: str, tracer="CudaWavefront", estimator=None):
    kern = {"maxBounce": int(desc.max_bounce)}
    if estimator:
        kern["estimator"] = estimator
    assets = []
    if desc.groups:
        assets.append(["import", {"path": mesh_path}])
    for s in desc.spheres:
        assets.append(["sphere", {"o": s["o"], "r": s["r"], "shader": s["shader"]}])
    for pl in desc.point_lights:
        assets.append(["pointLight", dict(pl)])
    return {
        "scene": {"camera": [desc.camera], "assets": assets, "shaders": desc.shaders},
        "tracer": [tracer, {"kernel": ["Radiance", kern]}],
    }


def write_scene(desc: SceneDesc, out_dir: str, fmt="crm", **kw) -> str:
    os.makedirs(out_dir, exist_ok=True)
    mesh_name = f"{desc.name}.{fmt}"
    if desc.groups:
        (write_crm if fmt == "crm" else write_obj)(os.path.join(out_dir, mesh_name), desc.groups)
    path = os.path.join(out_dir, f"{desc.name}.json")
    with open(path, "w") as fh:
        json.dump(scene_json(desc, mesh_name, **kw), fh, indent=1)
    return path


# ----------------------------------------------------------------------------
# camera rays, restating PinholeLens::sample and OrthographicLens::sample
# (src/core/misc/lens.hpp:15-27, 40-66)

def pinhole_rays(camera, w, h, spp, pixels, ks):
    """float32 primary rays (o, d) for pixel indices (x, y) and sample indices k."""
    f32 = np.float32
    fov = f32(camera.get("fovx", 90.0))
    tgt = np.asarray(camera.get("target", [-1, 0, 0]), f32)
    up = np.asarray(camera.get("upaxis", [0, 0, 1]), f32)
    pos = np.asarray(camera.get("position", [1, 0, 0]), f32)
    pw = int(math.ceil(math.sqrt(spp)))
    nrm = lambda a: (a / np.sqrt(np.sum(a * a, axis=-1, keepdims=True))).astype(f32)
    n = (nrm(tgt) * f32(w) / f32(2 * math.tan(math.radians(float(fov) * 0.5)))).astype(f32)
    u = nrm(np.cross(n, up))
    v = nrm(np.cross(n, u))
    du, dv = (u / f32(pw)).astype(f32), (v / f32(pw)).astype(f32)
    x = pixels[:, 0].astype(f32)[:, None]
    y = pixels[:, 1].astype(f32)[:, None]
    k = np.asarray(ks)
    ju, jv = (k % pw).astype(f32)[:, None], (k // pw).astype(f32)[:, None]
    if camera.get("lens", "pinhole") == "orthographic":
        # OrthographicLens::sample (lens.hpp:40-53)
        p = u[None] * (x - f32(w * 0.5)) + v[None] * (y - f32(h * 0.5)) + (du[None] * ju + dv[None] * jv)
        o = (pos[None] + p * f32(4.0) / f32(w)).astype(f32)
        d = np.broadcast_to(nrm(n), o.shape).astype(f32)
        return o, d
    t = n[None] + u[None] * (x - f32(w * 0.5)) + v[None] * (y - f32(h * 0.5))
    d = nrm(t + du[None] * ju + dv[None] * jv)
    o = np.broadcast_to(pos, d.shape).astype(f32)
    return o, d
