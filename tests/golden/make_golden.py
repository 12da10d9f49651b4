"""Regenerates the golden fixtures in this folder from the reference itself.

Runs oracle/_ref/cr_ref (the reference's own CPU Radiance path compiled from
its sources by `make -C oracle ref`, with the harness in
oracle/ref_harness/) on seeded scenes from the package's scene generator, and
stores its answers:

  c0_lights.npz    the 1024-point light table and pdf of config 0's light
                   (Mesh::generateSamples, src/core/primitive/mesh.hpp:61-84)
  c0_trace.npz     closest hits of primary + random rays (Scene::intersect)
  ico_trace.npz    same on a displaced level-4 icosphere in the box
  c0_occlude.npz   segment occlusion (Scene::intersect(Seg))
  c0_film.npz      per-pixel sums / sums of squares / counts of a Radiance
                   render (RadianceKernel::execute through the harness)
  c0_aov_*.npz     the same for the reference's debug kernels Normal,
                   Visibility and HalfVector (src/core/kernel/*.hpp)
  materials_film.npz, materials_aov_*.npz
                   Radiance, Visibility and HalfVector renders of the box with
                   GlassBSDF, RefractionBSDF, Transparent, Blackhole, Mixed
                   (Fresnel and Constant fac) and a pointLight as light 0
  c0_ortho_film.npz
                   config 0 through the OrthographicLens (lens.hpp:40-53)
  spheres_trace.npz
                   closest hits on a field of 300 spheres (Sphere::intersect,
                   sphere.hpp:31-54, over every sphere per ray)
  ico_film.npz     a Radiance render of the displaced icosphere scene (20
                   Lambert / Beckmann patch materials)
  shaders.npz      Shader::execute of each reference shader (nested Mixed
                   included) on scripted draws: for shared records
                   {wo, wi, u[12]} the f, emission and draw count of
                   compute_f_by_wi_wo and the wi, f, emission and draw count
                   of sample_wi_f_by_wo (the harness's `shade` command)

Usage:  python tests/golden/make_golden.py [--aov-only | --materials-only | --ortho-only | --spheres-only]
(--spheres-only also writes ico_film.npz)
(the harness's render threads take rows dynamically, so a film regenerated
from the same seed is a different Monte Carlo draw of the same image)
"""
import json
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from conftest import load_package  # noqa: E402

load_package()
from cuda_raytracer_b200 import scenes  # noqa: E402
import oracle  # noqa: E402

FILM_W, FILM_H, FILM_SPP = 48, 48, 1024


def scene_hash(desc, full=False):
    """Geometry hash; full=True also covers the shaders and the point lights."""
    h = hashlib.sha256()
    if full:
        h.update(json.dumps([desc.shaders, desc.point_lights], sort_keys=True).encode())
    for g in desc.groups:
        h.update(g.name.encode())
        h.update(np.ascontiguousarray(g.v).tobytes())
        h.update(np.ascontiguousarray(g.n).tobytes())
        h.update(np.ascontiguousarray(g.f).tobytes())
    for s in desc.spheres:
        h.update(repr(s).encode())
    return h.hexdigest()


def ico_scene():
    """Box + light + displaced level-4 icosphere (5120 triangles, 20 patch materials)."""
    return scenes.config1(level=4, seed=11, width=64, height=48, spp=4)


def make_rays(desc, n_random, seed):
    """Primary rays (PinholeLens::sample) plus rays from random interior points."""
    rng = np.random.default_rng(seed)
    w, h, spp = 32, 24, 4
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h)), -1).reshape(-1, 2)
    px = np.repeat(px, 2, axis=0)
    ks = np.tile([0, 3], len(px) // 2)
    o, d = scenes.pinhole_rays(desc.camera, w, h, spp, px, ks)
    lo = np.array([0.2, scenes.FRONT + 0.2, 0.2])
    hi = np.array([scenes.S - 0.2, scenes.S - 0.2, scenes.S - 0.2])
    ro = scenes._rot_points(lo + (hi - lo) * rng.random((n_random, 3))).astype(np.float32)
    rd = rng.normal(size=(n_random, 3))
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    rays = np.zeros((len(o) + n_random, 7), np.float32)
    rays[:len(o), :3], rays[:len(o), 3:6] = o, d
    rays[len(o):, :3], rays[len(o):, 3:6] = ro, rd
    rays[:, 6] = np.inf
    return rays


def make_segments(desc, n, seed):
    rng = np.random.default_rng(seed)
    lo = np.array([0.2, scenes.FRONT + 0.2, 0.2])
    hi = np.array([scenes.S - 0.2, scenes.S - 0.2, scenes.S - 0.2])
    a = scenes._rot_points(lo + (hi - lo) * rng.random((n, 3)))
    b = scenes._rot_points(lo + (hi - lo) * rng.random((n, 3)))
    d = b - a
    ln = np.linalg.norm(d, axis=1)
    segs = np.zeros((n, 7), np.float32)
    segs[:, :3] = a
    segs[:, 3:6] = d / ln[:, None]
    segs[:, 6] = ln
    return segs


def run(*args, cwd):
    return subprocess.run([oracle.REF_BIN, *map(str, args)], cwd=cwd, check=True, capture_output=True, text=True)


AOV_KERNELS = ("Normal", "Visibility", "HalfVector")
AOV_W, AOV_H, AOV_SPP = 48, 48, 256

SHADE_N, SHADE_K = 512, 12


def shader_configs():
    """The reference's shader registry (shader.impl.cu:16-23) with both
    distributions, both fac scalas and a nested Mixed."""
    beck = ["Beckmann", {"roughness": 0.3}]
    return [
        ["Lambert", {"R": [0.5, 0.6, 0.7], "color": [1, 0.9, 0.8]}],
        ["GlossyBSDF", {"distribution": beck, "color": [0.9, 0.8, 0.7]}],
        ["GlossyBSDF", {"distribution": ["Cosine", {}], "color": [0.9, 0.8, 0.7]}],
        ["Emission", {"color": [1, 0.5, 0.25], "strength": 3}],
        ["Transparent", {"color": [0.9, 0.9, 0.5]}],
        ["Blackhole", {}],
        ["RefractionBSDF", {"ior": 1.5, "distribution": beck, "color": [1, 1, 0.9]}],
        ["RefractionBSDF", {"ior": 1.33, "distribution": ["Cosine", {}]}],
        ["GlassBSDF", {"ior": 1.45, "distribution": ["Beckmann", {"roughness": 0.1}], "color": [0.95, 1, 1]}],
        ["Mixed", {"fac": ["Fresnel", {"ior": 1.5}],
                   "shaders": [["Lambert", {"R": [0.3, 0.3, 0.3]}], ["GlossyBSDF", {"distribution": beck}]]}],
        ["Mixed", {"fac": ["Constant", {"value": 0.3}],
                   "shaders": [["Mixed", {"fac": ["Constant", {"value": 0.6}],
                                          "shaders": [["Emission", {"strength": 4}],
                                                      ["GlassBSDF", {"ior": 1.3, "distribution": beck}]]}],
                               ["Transparent", {}]]}],
    ]


def shade_records(seed=41):
    """wo, wi uniform on the sphere (both sides of the surface), with grazing
    and near-normal directions mixed in; u uniform in [0, 1)."""
    rng = np.random.default_rng(seed)

    def dirs(n):
        d = rng.normal(size=(n, 3))
        return d / np.linalg.norm(d, axis=1, keepdims=True)
    wo, wi = dirs(SHADE_N), dirs(SHADE_N)
    k = SHADE_N // 8
    wo[:k, 2] *= 1e-3        # grazing
    wo[k:2 * k, :2] *= 1e-3  # near the normal (both sides)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    return wo.astype(np.float32), wi.astype(np.float32), rng.random((SHADE_N, SHADE_K)).astype(np.float32)


def make_shaders(tmp):
    wo, wi, u = shade_records()
    np.concatenate([wo, wi, u], 1).astype(np.float32).tofile(os.path.join(tmp, "rec.f32"))
    outs = []
    for cfg in shader_configs():
        with open(os.path.join(tmp, "shader.json"), "w") as fh:
            json.dump(cfg, fh)
        run("shade", "shader.json", "rec.f32", SHADE_K, "shade.f32", cwd=tmp)
        outs.append(np.fromfile(os.path.join(tmp, "shade.f32"), np.float32).reshape(SHADE_N, 17))
    np.savez_compressed(os.path.join(HERE, "shaders.npz"), wo=wo, wi=wi, u=u, out=np.stack(outs),
                        configs=json.dumps(shader_configs()))


def make_ortho(tmp):
    d = scenes.config0_ortho()
    scenes.write_scene(d, tmp)
    run("render", f"{d.name}.json", FILM_W, FILM_H, FILM_SPP, os.cpu_count(), "film.crf", d.max_bounce, 59, cwd=tmp)
    film = oracle.read_crf(os.path.join(tmp, "film.crf"))
    np.savez_compressed(os.path.join(HERE, "c0_ortho_film.npz"), sum=film.sum, sumsq=film.sumsq, count=film.count,
                        width=FILM_W, height=FILM_H, spp=FILM_SPP, max_bounce=d.max_bounce,
                        scene_hash=scene_hash(d, full=True), lens=d.camera["lens"])


def sphere_field(n=300, seed=340):
    """n spheres of random radii in the config-0 box with the box's walls
    removed: every hit is a sphere."""
    rng = np.random.default_rng(seed)
    d = scenes.config0()
    d.groups = []
    lo = np.array([0.3, scenes.FRONT + 0.3, 0.3])
    hi = np.array([scenes.S - 0.3, scenes.S - 0.3, scenes.S - 0.3])
    c = scenes._rot_points(lo + (hi - lo) * rng.random((n, 3)))
    r = rng.uniform(0.02, 0.3, n)
    d.spheres = [{"o": [float(x) for x in c[i]], "r": float(r[i]), "shader": "ball" if i % 2 else "glossy"}
                 for i in range(n)]
    d.name = "sphere_field"
    return d


def make_ico_film(tmp):
    d = ico_scene()
    scenes.write_scene(d, tmp)
    run("render", f"{d.name}.json", FILM_W, FILM_H, FILM_SPP, os.cpu_count(), "film.crf", d.max_bounce, 67, cwd=tmp)
    film = oracle.read_crf(os.path.join(tmp, "film.crf"))
    np.savez_compressed(os.path.join(HERE, "ico_film.npz"), sum=film.sum, sumsq=film.sumsq, count=film.count,
                        width=FILM_W, height=FILM_H, spp=FILM_SPP, max_bounce=d.max_bounce,
                        scene_hash=scene_hash(d, full=True))


def make_spheres(tmp):
    d = sphere_field()
    scenes.write_scene(d, tmp)
    rays = make_rays(d, 2048, 12)
    rays.tofile(os.path.join(tmp, "rays.f32"))
    run("trace", f"{d.name}.json", "rays.f32", "hits.bin", cwd=tmp)
    hits = np.fromfile(os.path.join(tmp, "hits.bin"), "<i4").reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, "spheres_trace.npz"), rays=rays, kind=hits[:, 0], index=hits[:, 1],
                        tri=hits[:, 2], t=hits[:, 3].view(np.float32), scene_hash=scene_hash(d))


def make_materials(tmp):
    m = scenes.config_materials()
    scenes.write_scene(m, tmp)
    js = f"{m.name}.json"
    for kname in ("Visibility", "HalfVector"):
        run("render", js, AOV_W, AOV_H, AOV_SPP, os.cpu_count(), "aov.crf", m.max_bounce, 31, kname, cwd=tmp)
        film = oracle.read_crf(os.path.join(tmp, "aov.crf"))
        np.savez_compressed(os.path.join(HERE, f"materials_aov_{kname.lower()}.npz"), sum=film.sum, sumsq=film.sumsq,
                            count=film.count, width=AOV_W, height=AOV_H, spp=AOV_SPP, kernel=kname,
                            scene_hash=scene_hash(m, full=True))
    run("render", js, FILM_W, FILM_H, FILM_SPP, os.cpu_count(), "film.crf", m.max_bounce, 37, cwd=tmp)
    film = oracle.read_crf(os.path.join(tmp, "film.crf"))
    np.savez_compressed(os.path.join(HERE, "materials_film.npz"), sum=film.sum, sumsq=film.sumsq, count=film.count,
                        width=FILM_W, height=FILM_H, spp=FILM_SPP, max_bounce=m.max_bounce,
                        scene_hash=scene_hash(m, full=True))


def main(aov_only=False, materials_only=False, ortho_only=False, spheres_only=False):
    if not oracle.ref_available():
        sys.exit("build the reference harness first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        if materials_only:
            make_shaders(tmp)
            make_materials(tmp)
            return
        if ortho_only:
            make_ortho(tmp)
            return
        if spheres_only:
            make_spheres(tmp)
            make_ico_film(tmp)
            return
        c0 = scenes.config0()
        scenes.write_scene(c0, tmp)
        js = f"{c0.name}.json"

        if not aov_only:
            run("lights", js, "lights.bin", oracle.LIGHT_SEED, cwd=tmp)
            raw = open(os.path.join(tmp, "lights.bin"), "rb").read()
            n = np.frombuffer(raw, "<u4", 1, 0)[0]
            assert n == 1
            group, = np.frombuffer(raw, "<i4", 1, 4)
            pdf, = np.frombuffer(raw, "<f4", 1, 8)
            nf, = np.frombuffer(raw, "<u4", 1, 12)
            table = np.frombuffer(raw, "<f4", 1024 * 6, 16).reshape(1024, 6)
            np.savez_compressed(os.path.join(HERE, "c0_lights.npz"), table=table, pdf=pdf, group=group, n_faces=nf,
                                seed=oracle.LIGHT_SEED, scene_hash=scene_hash(c0))

            for name, desc, nrand, seed in (("c0_trace.npz", c0, 2048, 5), ("ico_trace.npz", ico_scene(), 4096, 6)):
                scenes.write_scene(desc, tmp)
                rays = make_rays(desc, nrand, seed)
                rays.tofile(os.path.join(tmp, "rays.f32"))
                run("trace", f"{desc.name}.json", "rays.f32", "hits.bin", cwd=tmp)
                hits = np.fromfile(os.path.join(tmp, "hits.bin"), "<i4").reshape(-1, 4)
                np.savez_compressed(os.path.join(HERE, name), rays=rays, kind=hits[:, 0], index=hits[:, 1],
                                    tri=hits[:, 2], t=hits[:, 3].view(np.float32), scene_hash=scene_hash(desc))

            segs = make_segments(c0, 4096, 7)
            segs.tofile(os.path.join(tmp, "segs.f32"))
            run("occlude", js, "segs.f32", "occ.bin", cwd=tmp)
            occ = np.fromfile(os.path.join(tmp, "occ.bin"), np.uint8)
            np.savez_compressed(os.path.join(HERE, "c0_occlude.npz"), segs=segs, occluded=occ,
                                scene_hash=scene_hash(c0))

        # the reference's debug kernels on the same scene (Normal, Visibility, HalfVector)
        for kname in AOV_KERNELS:
            run("render", js, AOV_W, AOV_H, AOV_SPP, os.cpu_count(), "aov.crf", c0.max_bounce, 19, kname, cwd=tmp)
            film = oracle.read_crf(os.path.join(tmp, "aov.crf"))
            np.savez_compressed(os.path.join(HERE, f"c0_aov_{kname.lower()}.npz"), sum=film.sum, sumsq=film.sumsq,
                                count=film.count, width=AOV_W, height=AOV_H, spp=AOV_SPP, kernel=kname,
                                scene_hash=scene_hash(c0))
        if aov_only:
            return
        run("render", js, FILM_W, FILM_H, FILM_SPP, os.cpu_count(), "film.crf", c0.max_bounce, 17, cwd=tmp)
        film = oracle.read_crf(os.path.join(tmp, "film.crf"))
        np.savez_compressed(os.path.join(HERE, "c0_film.npz"), sum=film.sum, sumsq=film.sumsq, count=film.count,
                            width=FILM_W, height=FILM_H, spp=FILM_SPP, max_bounce=c0.max_bounce,
                            scene_hash=scene_hash(c0))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main(aov_only="--aov-only" in sys.argv, materials_only="--materials-only" in sys.argv,
         ortho_only="--ortho-only" in sys.argv, spheres_only="--spheres-only" in sys.argv)
