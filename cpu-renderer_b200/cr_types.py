"""Record layouts of include/cr_gpu.h as numpy dtypes and ctypes structures.

The layouts match the C structs byte for byte (and therefore CPU-Renderer's cr::Triangle,
cr::Ray, cr::Hit and Bvh::Node, scene.h). This module loads no library: the ctypes binding of
libcr_b200.so (crgpu.py) and the checkers that bind other libraries with the same structs
import their layouts from here.
"""
import ctypes as C

import numpy as np

vertex_dtype = np.dtype([("position", "<f4", 3), ("normal", "<f4", 3), ("tangent", "<f4", 4), ("uv", "<f4", (2, 2))])
triangle_dtype = np.dtype([("v", vertex_dtype, 3), ("material", "<u4"), ("geometric_normal", "<f4", 3), ("area", "<f4")])
ray_dtype = np.dtype([("origin", "<f4", 3), ("direction", "<f4", 3), ("tmin", "<f4"), ("tmax", "<f4"), ("origin_low", "<f4", 3)])
hit_dtype = np.dtype([("t", "<f8"), ("u", "<f8"), ("v", "<f8"), ("triangle", "<u4"), ("reserved", "<u4")])
node_dtype = np.dtype([("lo", "<f4", 3), ("hi", "<f4", 3), ("first", "<u4"), ("count", "<u4")])
slot_dtype = np.dtype([("texture", "<i4"), ("texcoord", "<i4"), ("offset", "<f4", 2), ("scale", "<f4", 2), ("rotation", "<f4")])
material_dtype = np.dtype([
    ("base_color", "<f4", 4), ("metallic", "<f4"), ("roughness", "<f4"), ("emission", "<f4", 3),
    ("transmission", "<f4"), ("ior", "<f4"), ("thickness", "<f4"), ("attenuation_distance", "<f4"),
    ("attenuation_color", "<f4", 3), ("double_sided", "<i4"), ("alpha_mode", "<i4"), ("alpha_cutoff", "<f4"),
    ("normal_scale", "<f4"), ("base_color_texture", slot_dtype), ("metallic_roughness_texture", slot_dtype),
    ("normal_texture", slot_dtype), ("emissive_texture", slot_dtype), ("transmission_texture", slot_dtype)])
light_dtype = np.dtype([("type", "<i4"), ("position", "<f4", 3), ("direction", "<f4", 3), ("color", "<f4", 3),
                        ("intensity", "<f4"), ("range", "<f4"), ("inner_cone", "<f4"), ("outer_cone", "<f4")])
texture_dtype = np.dtype([("image", "<i4"), ("wrap_s", "<i4"), ("wrap_t", "<i4"), ("linear", "<i4")])

# cr_traced_ray: a ray a render traced and the traversal's answer (cr_gpu_render_trace_dump)
traced_ray_dtype = np.dtype({"names": ["ray", "ignore", "kind", "depth", "found", "launch", "hit"],
                             "formats": [ray_dtype, "<u4", "<u4", "<u4", "<u4", "<u4", hit_dtype],
                             "offsets": [0, 44, 48, 52, 56, 60, 64], "itemsize": 96})

assert triangle_dtype.itemsize == 188 and ray_dtype.itemsize == 44 and hit_dtype.itemsize == 32
assert node_dtype.itemsize == 32 and material_dtype.itemsize == 220 and light_dtype.itemsize == 56

WRAP_REPEAT, WRAP_CLAMP, WRAP_MIRROR = 0, 1, 2
ALPHA_OPAQUE, ALPHA_MASK = 0, 1
LIGHT_POINT, LIGHT_DIRECTIONAL, LIGHT_SPOT = 0, 1, 2
INF = float("inf")
NO_TRIANGLE = 0xFFFFFFFF


def new_materials(n):
    """Materials with cr::Material's defaults (scene.h:187-199)."""
    m = np.zeros(n, material_dtype)
    m["base_color"] = 1.0
    m["metallic"] = 1.0
    m["roughness"] = 1.0
    m["ior"] = 1.5
    m["attenuation_distance"] = INF
    m["attenuation_color"] = 1.0
    m["alpha_cutoff"] = 0.5
    m["normal_scale"] = 1.0
    for k in ("base_color_texture", "metallic_roughness_texture", "normal_texture", "emissive_texture", "transmission_texture"):
        m[k]["texture"] = -1
        m[k]["scale"] = 1.0
    return m


def new_triangles(n):
    """Triangles with cr::Vertex defaults (tangent w = 1)."""
    t = np.zeros(n, triangle_dtype)
    t["v"]["tangent"][..., 3] = 1.0
    return t


def new_lights(n):
    l = np.zeros(n, light_dtype)
    l["direction"] = (0, 0, -1)
    l["color"] = 1.0
    l["intensity"] = 1.0
    l["range"] = INF
    l["outer_cone"] = np.float32(np.pi / 4)
    return l


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3), ("up", C.c_float * 3),
                ("yfov", C.c_float), ("aspect", C.c_float), ("near_clip", C.c_float), ("far_clip", C.c_float)]

    @classmethod
    def make(cls, position=(0, 0, 0), forward=(0, 0, -1), right=(1, 0, 0), up=(0, 1, 0), yfov=np.pi / 4,
             aspect=0.0, near_clip=0.01, far_clip=INF):
        """cr::Camera defaults (scene.h:202-207)."""
        c = cls()
        c.position[:] = [float(x) for x in position]
        c.forward[:] = [float(x) for x in forward]
        c.right[:] = [float(x) for x in right]
        c.up[:] = [float(x) for x in up]
        c.yfov, c.aspect, c.near_clip, c.far_clip = float(np.float32(yfov)), aspect, near_clip, far_clip
        return c


class Options(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("samples", C.c_int32), ("bounces", C.c_int32),
                ("threads", C.c_int32), ("seed", C.c_uint64), ("next_event_estimation", C.c_int32),
                ("russian_roulette", C.c_int32)]

    @classmethod
    def make(cls, width=960, height=540, samples=32, bounces=8, threads=0, seed=42, nee=True, rr=True):
        """cr::RenderOptions defaults (render.h:31-39)."""
        return cls(width, height, samples, bounces, threads, seed, int(nee), int(rr))


class Stats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("device_ms", C.c_double), ("trace_ms", C.c_double),
                ("shade_ms", C.c_double), ("regen_ms", C.c_double), ("workers", C.c_int32), ("chunks", C.c_int32),
                ("camera_samples", C.c_uint64), ("boundary_retries", C.c_uint64), ("extend_rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("kernel_launches", C.c_uint64), ("extend_pairs", C.c_uint64),
                ("extend_triangles", C.c_uint64), ("shadow_pairs", C.c_uint64), ("shadow_triangles", C.c_uint64),
                ("iterations", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("exact_traversal", C.c_int32), ("env_alias", C.c_int32), ("paths_per_wave", C.c_int32),
                ("chunk_log2", C.c_int32), ("generic_shading", C.c_int32), ("time_phases", C.c_int32),
                ("count_traversal", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangle_count", C.c_uint64), ("materials", C.c_void_p),
                ("material_count", C.c_uint32), ("lights", C.c_void_p), ("light_count", C.c_uint32),
                ("images", C.c_void_p), ("image_count", C.c_uint32), ("textures", C.c_void_p),
                ("texture_count", C.c_uint32), ("bvh_nodes", C.c_void_p), ("bvh_node_count", C.c_uint64),
                ("bvh_indices", C.c_void_p), ("bvh_index_count", C.c_uint64)]


class Image(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("pixels", C.c_void_p)]


class EnvDesc(C.Structure):
    _fields_ = [("constant", C.c_float * 3), ("pixels", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32),
                ("rotation_radians", C.c_float), ("intensity", C.c_float), ("cdf", C.c_void_p)]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_uint64, C.c_uint64, C.c_double, C.c_void_p)


ENCODE_SRGB8, ENCODE_RGBE, ENCODE_HDR_FILE = 0, 1, 2
FRAME_FN = C.CFUNCTYPE(None, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p)


class GuideOptions(C.Structure):
    _fields_ = [("train_samples", C.c_uint32), ("guide_probability", C.c_float), ("batch", C.c_uint32),
                ("epochs", C.c_uint32)]


class Job(C.Structure):
    """cr_job: one render of a batch or server."""
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("options", Options), ("film_rgb", C.c_void_p),
                ("every_samples", C.c_uint32), ("format", C.c_int32), ("exposure", C.c_float), ("on_frame", FRAME_FN),
                ("user", C.c_void_p), ("status", C.c_int), ("stats", Stats), ("submitted_at", C.c_double),
                ("started_at", C.c_double), ("first_frame_at", C.c_double), ("finished_at", C.c_double),
                ("error", C.c_char * 256)]


class EngineTuning(C.Structure):
    _fields_ = [("pool_paths", C.c_uint32), ("range_samples", C.c_uint32), ("refill_interval", C.c_uint32),
                ("iterations_per_step", C.c_uint32), ("use_graphs", C.c_int32), ("issue_policy", C.c_int32),
                ("memory_budget", C.c_uint64), ("refill_free_percent", C.c_uint32), ("solo_samples_log2", C.c_uint32),
                ("block_size", C.c_uint32), ("reserved", C.c_uint32)]

    @classmethod
    def make(cls, pool_paths=0, range_samples=0, refill_interval=0, iterations_per_step=0, use_graphs=1, memory_budget=0,
             issue_policy=0, refill_free_percent=0, solo_samples_log2=0, block_size=0):
        return cls(pool_paths, range_samples, refill_interval, iterations_per_step, use_graphs, issue_policy, memory_budget,
                   refill_free_percent, solo_samples_log2, block_size, 0)

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AutotuneTrial(C.Structure):
    _fields_ = [("pool_paths", C.c_uint32), ("iterations_per_step", C.c_uint32), ("refill_free_percent", C.c_uint32),
                ("block_size", C.c_uint32), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EngineStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("camera_samples", C.c_uint64), ("iterations", C.c_uint64),
                ("launches", C.c_uint64), ("extend_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("jobs_done", C.c_uint32), ("jobs_failed", C.c_uint32), ("peak_jobs", C.c_uint32),
                ("graph_steps", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}
