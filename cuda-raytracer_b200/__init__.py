"""B200-native Radiance path tracer: drop-in for the Radiance path of
xlnx/cuda-raytracer ("Koishi").

This module is the Python face of ``include/cr.h`` (ctypes over
``lib/libcr_b200.so``).  It mirrors the reference's plugin surface for the
path: the kernel registry (``Factory<Kernel>``, src/core/kernel/kernel.impl.cu:10-15)
holds ``"Radiance"`` and the reference's debug kernels ``"Normal"``,
``"Visibility"`` and ``"HalfVector"``, the tracer registry (``Factory<Tracer>``,
src/core/tracer/tracer.impl.cu:8-11) holds ``"CudaWavefront"`` and accepts the
reference's ``"CPUMulticore"`` name for scene files written for it, and the
shader registry (``Factory<Shader>``, src/ext/shader/shader.impl.cu:16-23)
holds all eight reference shaders, which ``shader_execute`` runs one
``Shader::execute`` at a time.  Scenes take spheres, meshes, point lights and
the pinhole or orthographic lens.  Every query runs on the GPU; there is no
CPU fallback, and importing this module on a machine where the library is
missing raises immediately on first use.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcr_b200.so")
CLI_PATH = os.path.join(HERE, "lib", "cr")

CR_OK = 0
KOISHI, MIS = 0, 1
KERNELS = ("Radiance", "Normal", "Visibility", "HalfVector")
TRACERS = ("CudaWavefront", "CPUMulticore")
DEFAULT_LIGHT_SEED = 0x330E
U32_MAX = 0xFFFFFFFF


class CrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cr error {code}: {msg}")
        self.code = code


class Hit(C.Structure):
    _fields_ = [("prim", C.c_int32), ("tri", C.c_int32), ("t", C.c_float), ("u", C.c_float), ("v", C.c_float)]


HIT_DTYPE = np.dtype([("prim", "<i4"), ("tri", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])


class RenderDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_bounce", C.c_uint32),
                ("estimator", C.c_int32), ("x0", C.c_uint32), ("y0", C.c_uint32), ("x1", C.c_uint32),
                ("y1", C.c_uint32), ("seed", C.c_uint64), ("wave_paths", C.c_uint32), ("guiding", C.c_int32),
                ("count_work", C.c_int32), ("refill_min", C.c_uint32), ("traverse_blocks_per_sm", C.c_uint32),
                ("shade_threads", C.c_uint32), ("rr_start", C.c_uint32), ("bin_rays", C.c_int32),
                ("shadow_vote", C.c_uint32), ("shadow_refill_min", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("wave_paths", C.c_uint32), ("refill_min", C.c_uint32), ("traverse_blocks_per_sm", C.c_uint32),
                ("candidates_tried", C.c_uint32), ("msamples_per_s", C.c_double),
                ("default_msamples_per_s", C.c_double), ("shade_threads", C.c_uint32), ("bin_rays", C.c_int32),
                ("shadow_vote", C.c_uint32), ("shadow_refill_min", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_extend", C.c_double), ("ms_shadow", C.c_double),
                ("ms_shade", C.c_double), ("ms_other", C.c_double), ("ms_guide", C.c_double), ("samples", C.c_uint64),
                ("rays_extend", C.c_uint64), ("rays_shadow", C.c_uint64), ("nodes", C.c_uint64),
                ("tris", C.c_uint64), ("shadow_nodes", C.c_uint64), ("shadow_tris", C.c_uint64), ("launches", C.c_uint32), ("waves", C.c_uint32),
                ("extend_launches", C.c_uint32), ("shadow_launches", C.c_uint32), ("ms_guide_train", C.c_double),
                ("graph_nodes", C.c_uint32), ("guide_launches", C.c_uint32), ("guide_rows", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GuideConfig(C.Structure):
    """cr_guide_config: the guide's training schedule."""
    _fields_ = [("lr", C.c_float), ("select_prob", C.c_float), ("train_paths", C.c_uint32),
                ("steps_per_wave", C.c_uint32), ("warmup_steps", C.c_uint32), ("product_target", C.c_uint32),
                ("max_steps", C.c_uint32), ("guided_bounces", C.c_uint32), ("learn_select", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BuildConfig(C.Structure):
    """cr_build_config: BVH build options."""
    _fields_ = [("builder", C.c_int32), ("ploc_radius", C.c_uint32), ("max_leaf", C.c_uint32),
                ("cost_node", C.c_float), ("cost_tri", C.c_float), ("collapse", C.c_int32),
                ("wide_cost_node", C.c_float), ("wide_cost_tri", C.c_float)]


class BatchJob(C.Structure):
    """cr_batch_job: one scene's render inside a batch."""
    _fields_ = [("scene", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("seed", C.c_uint64), ("d_sum", C.c_void_p), ("d_sumsq", C.c_void_p), ("d_count", C.c_void_p)]


_lib = None


def lib():
    """The loaded C library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libcr_b200.so not built at {LIB_PATH}; run `make -C cuda-raytracer_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        P, I, U32, U64, F = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_float
        sigs = {
            "cr_last_error": (C.c_char_p, []), "cr_version": (C.c_char_p, []),
            "cr_scene_create": (I, [C.c_char_p, C.c_char_p, P]),
            "cr_scene_create_empty": (I, [P]),
            "cr_scene_add_shader": (I, [P, C.c_char_p, C.c_char_p]),
            "cr_scene_add_mesh": (I, [P, P, U32, P, P, U32, C.c_char_p]),
            "cr_scene_add_sphere": (I, [P, P, F, C.c_char_p]),
            "cr_scene_add_point_light": (I, [P, P, P, F]),
            "cr_scene_set_lens": (I, [P, I]),
            "cr_bvh_build": (I, [P]),
            "cr_scene_set_camera": (I, [P, P, P, P, F]),
            "cr_scene_commit": (I, [P, U64, P]), "cr_scene_set_build": (I, [P, P]),
            "cr_scene_set_kernel": (I, [P, C.c_char_p]), "cr_mesh_file_info": (I, [C.c_char_p, P, P, P, P]),
            "cr_measure_peaks": (I, [P, P, P]), "cr_measure_gather": (I, [P, U32, U64, P]),
            "cr_scene_info": (I, [P, P, P, P, P]),
            "cr_scene_destroy": (None, [P]),
            "cr_light_table": (I, [P, U32, P, P]), "cr_scene_set_light_table": (I, [P, U32, P, F]),
            "cr_trace_rays": (I, [P, P, U64, P, I]),
            "cr_trace_rays_device": (I, [P, P, U64, P, I, P]),
            "cr_render": (I, [P, P, P, P]),
            "cr_render_device": (I, [P, P, P, P, P, P, P]),
            "cr_render_device_noalloc": (I, [P, P, P, P, P, P]),
            "cr_render_file": (I, [C.c_char_p, C.c_char_p, C.c_char_p, U32, U32, U32, C.c_char_p, C.c_char_p]),
            "cr_write_png": (I, [C.c_char_p, U32, U32, P]),
            "cr_autotune": (I, [P, P, P, P]),
            "cr_guide_reset": (I, [P, U64]), "cr_guide_info": (I, [P, P, P, P, P]),
            "cr_guide_params": (I, [P, P, P, P, I]), "cr_guide_forward": (I, [P, P, U64, P]),
            "cr_guide_gradients": (I, [P, P, U64, P, P, P]),
            "cr_guide_configure": (I, [P, P, P]), "cr_guide_loss": (I, [P, P]),
            "cr_guide_forward_tc": (I, [P, P, U64, P]), "cr_guide_gradients_tc": (I, [P, P, U64, P, P, P]),
            "cr_batch_create": (I, [P, U32, U32, C.c_int32, P, P]), "cr_batch_autotune": (I, [P, P]),
            "cr_batch_set_tuning": (I, [P, P]), "cr_trim_memory": (I, []),
            "cr_trace_work": (I, [P, P, U64, I, P]), "cr_guide_train": (I, [P, P, P, P]),
            "cr_batch_render": (I, [P, U64, P]), "cr_batch_destroy": (None, [P]),
            "cr_bsdf_eval": (I, [I, C.c_char_p, P, P, U64, P, P]),
            "cr_bsdf_sample": (I, [I, C.c_char_p, P, P, U64, P, P, P]),
            "cr_shader_execute": (I, [C.c_char_p, I, P, P, P, U32, U64, P, P, P]),
            "cr_philox4x32_10": (I, [P, U64, P]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _check(rc):
    if rc < 0:
        raise CrError(rc, lib().cr_last_error().decode(errors="replace"))
    return rc


def _p(a):
    # data_as keeps a reference to the array inside the pointer object
    return a.ctypes.data_as(C.c_void_p)


def render_desc(width, height, spp, max_bounce=None, estimator=None, seed=1, window=None, wave_paths=0,
                guiding=False, count_work=False, refill_min=0, traverse_blocks_per_sm=0, shade_threads=0,
                rr_start=0, bin_rays=0, shadow_vote=0, shadow_refill_min=0):
    d = RenderDesc()
    d.width, d.height, d.spp = width, height, spp
    d.max_bounce = U32_MAX if max_bounce is None else max_bounce
    d.estimator = -1 if estimator is None else estimator
    if window:
        d.x0, d.y0, d.x1, d.y1 = window
    d.seed = seed
    d.wave_paths = wave_paths
    d.guiding = int(bool(guiding))
    d.count_work = int(bool(count_work))
    d.refill_min = refill_min
    d.traverse_blocks_per_sm = traverse_blocks_per_sm
    d.shade_threads = shade_threads
    d.rr_start = rr_start
    d.bin_rays = bin_rays
    d.shadow_vote = shadow_vote
    d.shadow_refill_min = shadow_refill_min
    return d


class Scene:
    """A committed scene on the GPU (Scene, src/core/meta/scene.hpp:15-71)."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle)

    # -- construction ---------------------------------------------------------
    @classmethod
    def from_json(cls, text, base_dir="."):
        """Scene::Scene from the reference's JSON schema (import/sphere assets)."""
        out = C.c_void_p()
        _check(lib().cr_scene_create(text.encode(), base_dir.encode(), C.byref(out)))
        return cls(out.value)

    @classmethod
    def from_file(cls, path):
        with open(path) as fh:
            return cls.from_json(fh.read(), os.path.dirname(os.path.abspath(path)))

    @classmethod
    def from_desc(cls, desc, light_seed=DEFAULT_LIGHT_SEED, build=None):
        """Build from a scenes.SceneDesc through the add_* calls: meshes in
        group order, then spheres (the order the reference's scene loader
        gives an import asset listed before sphere assets)."""
        out = C.c_void_p()
        _check(lib().cr_scene_create_empty(C.byref(out)))
        s = cls(out.value)
        for name, cfg in desc.shaders.items():
            _check(lib().cr_scene_add_shader(s.h, name.encode(), json.dumps(cfg).encode()))
        for g in desc.groups:
            v = np.ascontiguousarray(g.v, np.float32)
            n = np.ascontiguousarray(g.n, np.float32)
            f = np.ascontiguousarray(g.f, np.uint32)
            _check(lib().cr_scene_add_mesh(s.h, _p(v), len(v), _p(n), _p(f), len(f), g.name.encode()))
        for sp in desc.spheres:
            c = np.asarray(sp["o"], np.float32)
            _check(lib().cr_scene_add_sphere(s.h, _p(c), float(sp["r"]), sp["shader"].encode()))
        for pl in getattr(desc, "point_lights", []):
            pos = np.asarray(pl["position"], np.float32)
            col = np.asarray(pl.get("color", [1, 1, 1]), np.float32)
            _check(lib().cr_scene_add_point_light(s.h, _p(pos), _p(col), float(pl.get("strength", 2.0))))
        cam = desc.camera
        # keep the arrays bound to names: ctypes only holds their addresses
        pos = np.asarray(cam["position"], np.float32)
        tgt = np.asarray(cam["target"], np.float32)
        up = np.asarray(cam.get("upaxis", [0, 0, 1]), np.float32)
        _check(lib().cr_scene_set_camera(s.h, _p(pos), _p(tgt), _p(up), float(cam.get("fovx", 90.0))))
        lens = cam.get("lens", "pinhole")
        if lens not in ("pinhole", "orthographic"):
            raise CrError(-2, f"unknown lens type: {lens}")
        _check(lib().cr_scene_set_lens(s.h, 1 if lens == "orthographic" else 0))
        if build:
            bc = BuildConfig(builder=build.get("builder", 0), ploc_radius=build.get("ploc_radius", 10),
                             max_leaf=build.get("max_leaf", 3), cost_node=build.get("cost_node", 1.2),
                             cost_tri=build.get("cost_tri", 1.0), collapse=build.get("collapse", 0),
                             wide_cost_node=build.get("wide_cost_node", 1.0),
                             wide_cost_tri=build.get("wide_cost_tri", 0.6))
            _check(lib().cr_scene_set_build(s.h, C.byref(bc)))
        _check(lib().cr_scene_commit(s.h, light_seed, None))
        return s

    def close(self):
        if self.h and self.h.value:
            lib().cr_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- queries ----------------------------------------------------------------
    def info(self):
        nt, np_, nl, nn = C.c_uint64(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().cr_scene_info(self.h, C.byref(nt), C.byref(np_), C.byref(nl), C.byref(nn)))
        return {"triangles": nt.value, "primitives": np_.value, "lights": nl.value, "bvh_nodes": nn.value}

    def light_table(self, light):
        out = np.zeros((1024, 6), np.float32)
        pdf = C.c_float()
        _check(lib().cr_light_table(self.h, light, _p(out), C.byref(pdf)))
        return out, pdf.value

    def trace(self, rays, any_hit=False):
        """rays: (n, 7) float32 {o, d, tmax}.  Returns a structured array of hits."""
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros(len(rays), HIT_DTYPE)
        _check(lib().cr_trace_rays(self.h, _p(rays), len(rays), _p(hits), int(bool(any_hit))))
        return hits

    def trace_work(self, rays, any_hit=False):
        """cr_trace_work: (wide nodes fetched, primitives tested) summed over
        the rays (n, 7) {o, d, tmax}."""
        rays = np.ascontiguousarray(rays, np.float32)
        w = np.zeros(2, np.uint64)
        _check(lib().cr_trace_work(self.h, _p(rays), len(rays), int(bool(any_hit)), _p(w)))
        return int(w[0]), int(w[1])

    def trace_device(self, rays_ptr, n, hits_ptr, any_hit=False, stream=0):
        _check(lib().cr_trace_rays_device(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr),
                                          int(bool(any_hit)), C.c_void_p(stream)))

    def set_kernel(self, name):
        """cr_scene_set_kernel: Radiance, or the debug kernels Normal, Visibility, HalfVector."""
        _check(lib().cr_scene_set_kernel(self.h, name.encode()))
        return self

    def render(self, width, height, spp, **kw):
        """Mean radiance per pixel (window-sized H x W x 3 float64) and stats."""
        d = render_desc(width, height, spp, **kw)
        x0, y0, x1, y1 = kw.get("window") or (0, 0, width, height)
        film = np.zeros((y1 - y0, x1 - x0, 3))
        st = Stats()
        _check(lib().cr_render(self.h, C.byref(d), _p(film), C.byref(st)))
        return film, st

    def set_light_table(self, primitive, table, pdf):
        """cr_scene_set_light_table: the 1024-point table (1024 x 6: p, n) and
        area pdf of the emissive mesh `primitive`, e.g. a reference Mesh's own."""
        t = np.ascontiguousarray(table, np.float32).reshape(1024, 6)
        _check(lib().cr_scene_set_light_table(self.h, int(primitive), _p(t), float(pdf)))

    def autotune(self, desc, stream=0):
        """cr_autotune: pick and keep the launch configuration for this scene."""
        t = Tuning()
        _check(lib().cr_autotune(self.h, C.byref(desc), C.c_void_p(stream), C.byref(t)))
        return t

    def render_device(self, desc, sum_ptr, sumsq_ptr, count_ptr, stream=0, stats=True):
        st = Stats() if stats else None
        _check(lib().cr_render_device(self.h, C.byref(desc), C.c_void_p(sum_ptr), C.c_void_p(sumsq_ptr),
                                      C.c_void_p(count_ptr), C.c_void_p(stream),
                                      C.byref(st) if st is not None else None))
        return st


class Guide:
    """The scene's learned path guide (cr_guide_*)."""

    def __init__(self, scene):
        self.scene = scene

    def reset(self, seed=1):
        _check(lib().cr_guide_reset(self.scene.h, seed))
        return self

    def train(self, desc, stream=0):
        """cr_guide_train: train the guide to its budget on scratch passes of
        desc's image (each one wave recorded whole); returns the passes."""
        n = C.c_uint32()
        _check(lib().cr_guide_train(self.scene.h, C.byref(desc), C.c_void_p(stream), C.byref(n)))
        return n.value

    def info(self):
        bmin, binv, sizes = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(3, np.uint32)
        step = C.c_uint32()
        _check(lib().cr_guide_info(self.scene.h, _p(bmin), _p(binv), C.byref(step), _p(sizes)))
        return {"bmin": bmin, "binv": binv, "step": step.value, "sizes": sizes}

    def params(self):
        s = self.info()["sizes"]
        grid, W, b = (np.zeros(int(n), np.float32) for n in s)
        _check(lib().cr_guide_params(self.scene.h, _p(grid), _p(W), _p(b), 0))
        return grid, W, b

    def set_params(self, grid=None, W=None, b=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (grid, W, b)]
        ptrs = [None if a is None else _p(a) for a in arrs]
        _check(lib().cr_guide_params(self.scene.h, *ptrs, 1))

    def forward(self, inputs, tensor_cores=False):
        """Network outputs (n x 64) for n x {x, wo, n}: FP32 CUDA-core path, or
        the BF16 tensor-core path the renderer samples with."""
        inputs = np.ascontiguousarray(inputs, np.float32)
        out = np.zeros((len(inputs), 64), np.float32)
        fn = lib().cr_guide_forward_tc if tensor_cores else lib().cr_guide_forward
        _check(fn(self.scene.h, _p(inputs), len(inputs), _p(out)))
        return out

    def configure(self, **kw):
        """cr_guide_configure: set the given schedule fields, return the schedule."""
        cur = GuideConfig()
        _check(lib().cr_guide_configure(self.scene.h, None, C.byref(cur)))
        if kw:
            for k, v in kw.items():
                if k not in dict(GuideConfig._fields_):
                    raise KeyError(k)
                setattr(cur, k, v)
            _check(lib().cr_guide_configure(self.scene.h, C.byref(cur), C.byref(cur)))
        return cur.as_dict()

    def loss(self):
        """Weighted NLL of the last training batch."""
        v = C.c_float()
        _check(lib().cr_guide_loss(self.scene.h, C.byref(v)))
        return v.value

    def gradients(self, records, tensor_cores=False):
        """Gradients (grid, W, b) of the weighted mixture NLL over records
        n x {x, wo, n, w, weight} (and the BSDF density of w when the guide
        learns its selection): FP32 pass, or the BF16 tensor-core pass the
        renderer trains with."""
        records = np.ascontiguousarray(records, np.float32)
        width = 14 if self.configure()["learn_select"] else 13
        if records.ndim != 2 or records.shape[1] != width:
            raise ValueError(f"records must be n x {width}")
        s = self.info()["sizes"]
        ggrid, gW, gb = (np.zeros(int(n), np.float32) for n in s)
        fn = lib().cr_guide_gradients_tc if tensor_cores else lib().cr_guide_gradients
        _check(fn(self.scene.h, _p(records), len(records), _p(gW), _p(gb), _p(ggrid)))
        return ggrid, gW, gb


def mesh_file_info(path):
    """cr_mesh_file_info: (groups, vertices, triangles, checksum) of an OBJ / PLY / CRM file."""
    ng, nv, nt, cs = C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_double()
    _check(lib().cr_mesh_file_info(path.encode(), C.byref(ng), C.byref(nv), C.byref(nt), C.byref(cs)))
    return ng.value, nv.value, nt.value, cs.value


def measure_peaks(stream=0):
    """cr_measure_peaks: (L2-resident read GB/s, FP32 FMA TFLOP/s) of this GPU."""
    l2, fp = C.c_double(), C.c_double()
    _check(lib().cr_measure_peaks(C.c_void_p(stream), C.byref(l2), C.byref(fp)))
    return l2.value, fp.value


def trim_memory():
    """cr_trim_memory: hand the wave-state memory the library keeps mapped
    between renders back to the device."""
    _check(lib().cr_trim_memory())


def measure_gather(record_bytes=80, array_bytes=64 << 20, stream=0):
    """cr_measure_gather: GB/s of random whole-record gathers (80-byte nodes or
    48-byte triangles) from an array of array_bytes (L2-resident below 126 MB)."""
    g = C.c_double()
    _check(lib().cr_measure_gather(C.c_void_p(stream), record_bytes, array_bytes, C.byref(g)))
    return g.value


class Batch:
    """A batched render of many scenes (cr_batch_*): jobs are (scene, width,
    height, spp, seed, sum_ptr, sumsq_ptr, count_ptr) with device films; the
    first render captures a CUDA graph that later renders replay."""

    def __init__(self, jobs, max_bounce=7, estimator=KOISHI, stream=0):
        self.scenes = [j[0] for j in jobs]  # keep the scenes alive with the batch
        arr = (BatchJob * len(jobs))()
        for a, (sc, w, h, spp, seed, ps, pq, pc) in zip(arr, jobs):
            a.scene, a.width, a.height, a.spp, a.seed = sc.h.value, w, h, spp, seed
            a.d_sum, a.d_sumsq, a.d_count = ps, pq, pc
        out = C.c_void_p()
        _check(lib().cr_batch_create(arr, len(jobs), max_bounce, estimator, C.c_void_p(stream), C.byref(out)))
        self.h = out

    def autotune(self):
        t = Tuning()
        _check(lib().cr_batch_autotune(self.h, C.byref(t)))
        return t

    def set_tuning(self, wave_paths=0, refill_min=0, traverse_blocks_per_sm=0, shade_threads=0):
        """cr_batch_set_tuning: launch configuration (0 keeps a field)."""
        t = Tuning()
        t.wave_paths, t.refill_min, t.traverse_blocks_per_sm = wave_paths, refill_min, traverse_blocks_per_sm
        t.shade_threads = shade_threads
        _check(lib().cr_batch_set_tuning(self.h, C.byref(t)))

    def render(self, seed_offset=0, stats=True):
        st = Stats() if stats else None
        _check(lib().cr_batch_render(self.h, seed_offset, C.byref(st) if st is not None else None))
        return st

    def close(self):
        if self.h and self.h.value:
            lib().cr_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_file(json_path, png_path, spp=1, width=1024, height=768, kernel="Radiance", tracer="CudaWavefront",
                pfm_path=None):
    """Renderer::render (src/core/renderer/renderer.cu:13-52)."""
    _check(lib().cr_render_file(json_path.encode(), png_path.encode(), pfm_path.encode() if pfm_path else None,
                                spp, width, height, kernel.encode(), tracer.encode()))


def bsdf_eval(estimator, shader_cfg, wo, wi):
    wo = np.ascontiguousarray(wo, np.float32)
    wi = np.ascontiguousarray(wi, np.float32)
    n = len(wo)
    f = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    _check(lib().cr_bsdf_eval(estimator, json.dumps(shader_cfg).encode(), _p(wo), _p(wi), n, _p(f), _p(pdf)))
    return f, pdf


def philox4x32_10(ctr_key):
    """The render's device Philox4x32-10 generator on (n, 6) words (c0..c3,
    k0, k1); returns (n, 4) uint32 outputs."""
    ck = np.ascontiguousarray(np.asarray(ctr_key, dtype=np.uint32).reshape(-1, 6))
    out = np.zeros((len(ck), 4), np.uint32)
    _check(lib().cr_philox4x32_10(_p(ck), len(ck), _p(out)))
    return out


SHADE_EVAL, SHADE_SAMPLE = 0, 1


def shader_execute(shader_cfg, target, wo, u, wi=None):
    """Shader::execute of a [Type, {props}] shader config (nested Mixed
    included) with the reference estimator's semantics, for n local-frame
    samples: target SHADE_EVAL (compute_f_by_wi_wo, wi given) or SHADE_SAMPLE
    (sample_wi_f_by_wo).  u is (n, k) uniforms drawn in order.  Returns
    (f, wi, emission, used)."""
    wo = np.ascontiguousarray(wo, np.float32)
    n = len(wo)
    u = np.ascontiguousarray(np.asarray(u, np.float32).reshape(n, -1))
    wi = np.zeros((n, 3), np.float32) if wi is None else np.array(wi, np.float32, order="C", copy=True)
    f = np.zeros((n, 3), np.float32)
    em = np.zeros((n, 3), np.float32)
    used = np.zeros(n, np.uint32)
    _check(lib().cr_shader_execute(json.dumps(shader_cfg).encode(), target, _p(wo), _p(wi), _p(u), u.shape[1], n,
                                   _p(f), _p(em), _p(used)))
    return f, wi, em, used


def bsdf_sample(estimator, shader_cfg, wo, u):
    wo = np.ascontiguousarray(wo, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    n = len(wo)
    wi = np.zeros((n, 3), np.float32)
    w = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    _check(lib().cr_bsdf_sample(estimator, json.dumps(shader_cfg).encode(), _p(wo), _p(u), n, _p(wi), _p(w),
                                _p(pdf)))
    return wi, w, pdf
