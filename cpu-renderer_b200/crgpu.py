"""ctypes binding of include/cr_gpu.h (libcr_b200.so).

The record layouts (cr_types.py) are numpy dtypes that match the C structs byte for byte
(and therefore CPU-Renderer's cr::Triangle, cr::Ray, cr::Hit and Bvh::Node). The binding raises
RuntimeError with the library's message on any non-zero status; there is no fallback path:
if libcr_b200.so is missing, importing this module fails.
"""
import ctypes as C
import os

import numpy as np

from cr_types import (  # noqa: F401  (the layouts are part of this module's interface)
    ALPHA_MASK, ALPHA_OPAQUE, AutotuneTrial, ENCODE_HDR_FILE, ENCODE_RGBE, ENCODE_SRGB8, FRAME_FN, INF, LIGHT_DIRECTIONAL, LIGHT_POINT,
    LIGHT_SPOT, NO_TRIANGLE, PROGRESS_FN, WRAP_CLAMP, WRAP_MIRROR, WRAP_REPEAT, Camera, EngineStats, EngineTuning,
    EnvDesc, GuideOptions, Image, Job, Options, SceneDesc, Stats, Tuning, hit_dtype, light_dtype, material_dtype,
    new_lights, new_materials, new_triangles, node_dtype, ray_dtype, slot_dtype, texture_dtype, traced_ray_dtype,
    triangle_dtype, vertex_dtype)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CR_B200_LIB", os.path.join(HERE, "libcr_b200.so"))


def _ptr(a):
    return None if a is None or len(a) == 0 else a.ctypes.data


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libcr_b200.so is not built (run cpu-renderer_b200/build.py): " + LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    sig = {
        "cr_gpu_abi_version": (C.c_int, []),
        "cr_gpu_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
        "cr_gpu_device_count": (C.c_int, [C.POINTER(C.c_int)]),
        "cr_options_validate": (C.c_int, [C.POINTER(Options)]),
        "cr_scene_finalize": (C.c_int, [P, C.POINTER(C.c_uint64), P, C.c_uint32, P, C.c_uint32, P, C.c_uint32, C.c_char_p, C.c_size_t]),
        "cr_bvh_build": (C.c_int, [P, C.c_uint64, P, C.POINTER(C.c_uint64), P]),
        "cr_environment_rotation": (C.c_float, [C.c_float]),
        "cr_environment_tables": (C.c_int, [C.POINTER(EnvDesc), P, P]),
        "cr_gpu_scene_create": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(EnvDesc), C.c_int, C.POINTER(P)]),
        "cr_gpu_scene_destroy": (C.c_int, [P]),
        "cr_gpu_scene_bytes": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "cr_gpu_intersect": (C.c_int, [P, P, C.c_uint64, C.c_int, C.c_uint32, P, P, C.POINTER(Tuning)]),
        "cr_gpu_camera_rays": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), C.c_uint32, P]),
        "cr_gpu_render": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), PROGRESS_FN, P, P, C.POINTER(Stats), C.POINTER(Tuning)]),
        "cr_gpu_render_resident": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), C.POINTER(Stats), C.POINTER(Tuning), P]),
        "cr_gpu_film_download": (C.c_int, [P, P, C.c_uint64]),
        "cr_gpu_environment_sample": (C.c_int, [P, C.c_int, C.c_uint64, C.c_uint64, P, P]),
        "cr_gpu_render_trace_dump": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), C.POINTER(Tuning), P, C.c_uint64,
                                               C.POINTER(C.c_uint64)]),
        "cr_gpu_render_noalloc": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), P, C.POINTER(Stats)]),
        "cr_gpu_allocation_count": (C.c_int, [C.POINTER(C.c_uint64)]),
        "cr_gpu_debug_fail_allocation": (C.c_int, [C.c_int64]),
        "cr_display_thresholds": (C.c_int, [C.c_float, P]),
        "cr_gpu_film_encode": (C.c_int, [P, C.c_int, C.c_float, P, C.c_uint64, C.POINTER(C.c_uint64)]),
        "cr_gpu_encode": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, P, C.c_uint64, C.POINTER(C.c_uint64)]),
        "cr_gpu_render_progressive": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), C.c_uint32, C.c_int, C.c_float,
                                                FRAME_FN, P, P, C.POINTER(Stats), C.POINTER(Tuning)]),
        "cr_guide_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(P)]),
        "cr_guide_destroy": (C.c_int, [P]),
        "cr_guide_parameter_count": (C.c_uint32, []),
        "cr_guide_get_parameters": (C.c_int, [P, P]),
        "cr_guide_set_parameters": (C.c_int, [P, P]),
        "cr_guide_evaluate": (C.c_int, [P, P, C.c_uint64, P]),
        "cr_guide_gradients": (C.c_int, [P, P, C.c_uint64, P, C.POINTER(C.c_double)]),
        "cr_guide_train": (C.c_int, [P, P, C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(C.c_float)]),
        "cr_gpu_render_guided": (C.c_int, [P, C.POINTER(Camera), C.POINTER(Options), P, C.POINTER(GuideOptions), P,
                                           C.POINTER(Stats), C.POINTER(Tuning)]),
        "cr_gpu_phase_benchmark": (C.c_int, [P, C.POINTER(Camera), C.c_int32, C.c_int32, C.c_uint32, C.c_uint64, P]),
        "cr_gpu_render_batch": (C.c_int, [P, C.c_uint32, C.POINTER(EngineTuning), C.POINTER(EngineStats)]),
        "cr_gpu_autotune_batch": (C.c_int, [P, C.c_uint32, C.POINTER(EngineTuning)]),
        "cr_gpu_autotune_batch_trials": (C.c_int, [P, C.c_uint32, C.POINTER(EngineTuning), P, C.c_uint32,
                                                   C.POINTER(C.c_uint32)]),
        "cr_server_create": (C.c_int, [C.c_int, C.POINTER(EngineTuning), C.POINTER(P)]),
        "cr_server_submit": (C.c_int, [P, P, C.POINTER(C.c_uint64)]),
        "cr_server_wait": (C.c_int, [P, C.c_uint64, C.c_double]),
        "cr_server_stats": (C.c_int, [P, C.POINTER(EngineStats)]),
        "cr_server_clock": (C.c_double, [P]),
        "cr_server_destroy": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


lib = _load()


class CrError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


def last_error():
    buf = C.create_string_buffer(4096)
    lib.cr_gpu_last_error(buf, len(buf))
    return buf.value.decode()


def check(status):
    if status != 0:
        raise CrError(status, last_error())


def allocation_count():
    """Memory blocks the library has requested since it was loaded (device and page-locked host)."""
    n = C.c_uint64(0)
    check(lib.cr_gpu_allocation_count(C.byref(n)))
    return n.value


def fail_allocation(nth):
    """Test hook: the nth device allocation from now (0: the next) fails as out of memory;
    a negative nth disarms it."""
    check(lib.cr_gpu_debug_fail_allocation(int(nth)))


def device_count():
    n = C.c_int(0)
    lib.cr_gpu_device_count(C.byref(n))
    return n.value


def validate_options(options):
    check(lib.cr_options_validate(C.byref(options)))


def environment_rotation(degrees):
    return lib.cr_environment_rotation(float(degrees))


def finalize(triangles, materials, images=(), textures=None):
    """Scene::finalize restated (returns the compacted array and the warnings)."""
    t = np.ascontiguousarray(triangles, dtype=triangle_dtype).copy()
    count = C.c_uint64(len(t))
    img, tex = _images(images), _textures(textures)
    buf = C.create_string_buffer(8192)
    check(lib.cr_scene_finalize(_ptr(t), C.byref(count), _ptr(materials), len(materials),
                                C.cast(img, C.c_void_p) if img else None, len(images),
                                _ptr(tex), 0 if tex is None else len(tex), buf, len(buf)))
    w = buf.value.decode()
    return t[:count.value].copy(), (w.split("\n") if w else [])


def build_bvh(triangles):
    t = np.ascontiguousarray(triangles, dtype=triangle_dtype)
    n = len(t)
    nodes = np.zeros(max(1, 2 * n - 1), node_dtype)
    idx = np.zeros(max(1, n), np.uint32)
    count = C.c_uint64(0)
    check(lib.cr_bvh_build(_ptr(t), n, nodes.ctypes.data, C.byref(count), idx.ctypes.data))
    return nodes[:count.value].copy(), idx[:n].copy()


def _images(images):
    if not images:
        return None
    arr = (Image * len(images))()
    for i, im in enumerate(images):
        im = np.ascontiguousarray(im, dtype=np.float32)
        arr[i] = Image(im.shape[1], im.shape[0], im.ctypes.data)
    arr._keep = images
    return arr


def _textures(textures):
    if textures is None or len(textures) == 0:
        return None
    return np.ascontiguousarray(textures, dtype=texture_dtype)


def env_desc(constant=(0, 0, 0), image=None, rotation_degrees=0.0, intensity=1.0):
    """cr::Environment: a constant radiance, or an RGBA float32 (H, W, 4) equirect image."""
    e = EnvDesc()
    e.constant[:] = [float(x) for x in constant]
    e.intensity = float(intensity)
    e.rotation_radians = environment_rotation(rotation_degrees)
    if image is not None:
        image = np.ascontiguousarray(image, dtype=np.float32)
        assert image.ndim == 3 and image.shape[2] == 4
        e.pixels = image.ctypes.data
        e.height, e.width = image.shape[0], image.shape[1]
        e._keep = image
    return e


class GpuScene:
    """A device-resident scene (cr_gpu_scene)."""

    def __init__(self, triangles, materials, lights=None, images=(), textures=None, env=None, bvh=None, device=0):
        self._arrays = []
        t = np.ascontiguousarray(triangles, dtype=triangle_dtype)
        m = np.ascontiguousarray(materials, dtype=material_dtype)
        l = np.ascontiguousarray(lights if lights is not None else np.zeros(0, light_dtype), dtype=light_dtype)
        img = _images(images)
        tex = _textures(textures)
        d = SceneDesc()
        d.triangles, d.triangle_count = _ptr(t), len(t)
        d.materials, d.material_count = _ptr(m), len(m)
        d.lights, d.light_count = _ptr(l), len(l)
        d.images, d.image_count = (C.cast(img, C.c_void_p).value if img else None), len(images)
        d.textures, d.texture_count = _ptr(tex), (0 if tex is None else len(tex))
        if bvh is not None:
            nodes, idx = bvh
            nodes = np.ascontiguousarray(nodes, dtype=node_dtype)
            idx = np.ascontiguousarray(idx, dtype=np.uint32)
            d.bvh_nodes, d.bvh_node_count = _ptr(nodes), len(nodes)
            d.bvh_indices, d.bvh_index_count = _ptr(idx), len(idx)
            self._arrays += [nodes, idx]
        self._arrays += [t, m, l, img, tex]
        e = env if env is not None else env_desc()
        h = C.c_void_p()
        check(lib.cr_gpu_scene_create(C.byref(d), C.byref(e), device, C.byref(h)))
        self._arrays = None  # the library keeps device copies, never the caller's pointers
        self.handle = h
        self.triangle_count = len(t)

    def close(self):
        if self.handle:
            lib.cr_gpu_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bytes(self):
        b = C.c_uint64(0)
        check(lib.cr_gpu_scene_bytes(self.handle, C.byref(b)))
        return b.value

    def intersect(self, rays, any_hit=False, ignore=NO_TRIANGLE, hits=None, tuning=None):
        """Bvh::intersect over a batch; returns (found bool array, hits)."""
        rays = np.ascontiguousarray(rays, dtype=ray_dtype)
        n = len(rays)
        if hits is None:
            hits = np.zeros(n, hit_dtype)
            hits["t"] = INF
        hits = np.ascontiguousarray(hits, dtype=hit_dtype).copy()
        found = np.zeros(n, np.uint8)
        check(lib.cr_gpu_intersect(self.handle, _ptr(rays), n, int(any_hit), ignore, _ptr(hits), _ptr(found),
                                   C.byref(tuning) if tuning else None))
        return found.astype(bool), hits

    def camera_rays(self, camera, options, sample):
        out = np.zeros(options.width * options.height, ray_dtype)
        check(lib.cr_gpu_camera_rays(self.handle, C.byref(camera), C.byref(options), sample, out.ctypes.data))
        return out

    def render(self, camera, options, progress=None, tuning=None):
        """cr::render: returns (film float32 (H, W, 3), stats dict)."""
        film = np.zeros((options.height, options.width, 3), np.float32)
        stats = Stats()
        cb = PROGRESS_FN(lambda a, b, s, u: progress(a, b, s)) if progress else PROGRESS_FN(0)
        check(lib.cr_gpu_render(self.handle, C.byref(camera), C.byref(options), cb, None, film.ctypes.data,
                                C.byref(stats), C.byref(tuning) if tuning else None))
        return film, stats.as_dict()

    def render_resident(self, camera, options, tuning=None, per_sample=False):
        """Film stays on the device; optionally returns every sample's radiance
        (samples, H, W, 3)."""
        stats = Stats()
        ps = None
        if per_sample:
            ps = np.zeros((options.samples, options.height, options.width, 3), np.float32)
        check(lib.cr_gpu_render_resident(self.handle, C.byref(camera), C.byref(options), C.byref(stats),
                                         C.byref(tuning) if tuning else None, None if ps is None else ps.ctypes.data))
        return stats.as_dict(), ps

    def environment_sample(self, count, alias=False, seed=1):
        """cr_gpu_environment_sample: (texel index, density) of `count` environment samples."""
        texels = np.zeros(count, np.uint32)
        dens = np.zeros(count, np.float32)
        check(lib.cr_gpu_environment_sample(self.handle, int(alias), seed, count, texels.ctypes.data, dens.ctypes.data))
        return texels, dens

    def trace_dump(self, camera, options, capacity, tuning=None):
        """cr_gpu_render_trace_dump: (rays traced, recorded records as traced_ray_dtype)."""
        rays = np.zeros(capacity, traced_ray_dtype)
        n = C.c_uint64(0)
        check(lib.cr_gpu_render_trace_dump(self.handle, C.byref(camera), C.byref(options),
                                           C.byref(tuning) if tuning else None, rays.ctypes.data if capacity else None,
                                           capacity, C.byref(n)))
        return n.value, rays[:min(n.value, capacity)]

    def film(self, width, height):
        out = np.zeros((height, width, 3), np.float32)
        check(lib.cr_gpu_film_download(self.handle, out.ctypes.data, out.size))
        return out

    def render_guided(self, camera, options, guide, train_samples=32, probability=0.5, batch=16384, epochs=4,
                      tuning=None):
        """cr_gpu_render_guided: returns (film, stats); `guide` is a Guide and keeps its training."""
        film = np.zeros((options.height, options.width, 3), np.float32)
        stats = Stats()
        go = GuideOptions(train_samples, probability, batch, epochs)
        check(lib.cr_gpu_render_guided(self.handle, C.byref(camera), C.byref(options), guide.handle, C.byref(go),
                                       film.ctypes.data, C.byref(stats), C.byref(tuning) if tuning else None))
        return film, stats.as_dict()

    def film_encode(self, fmt=ENCODE_SRGB8, exposure=0.0):
        """The last render's film encoded on the device (cr_gpu_film_encode): bytes."""
        size = C.c_uint64(0)
        check(lib.cr_gpu_film_encode(self.handle, fmt, exposure, None, 0, C.byref(size)))
        out = np.zeros(size.value, np.uint8)
        check(lib.cr_gpu_film_encode(self.handle, fmt, exposure, _ptr(out), size.value, C.byref(size)))
        return out[:size.value].tobytes()

    def render_progressive(self, camera, options, every, fmt=ENCODE_SRGB8, exposure=0.0, tuning=None):
        """cr_gpu_render_progressive: returns ([(samples_done, frame bytes)], film, stats)."""
        frames = []

        def on_frame(done, data, size, user):
            frames.append((done, C.string_at(data, size)))

        cb = FRAME_FN(on_frame)
        film = np.zeros((options.height, options.width, 3), np.float32)
        stats = Stats()
        check(lib.cr_gpu_render_progressive(self.handle, C.byref(camera), C.byref(options), every, fmt, exposure, cb, None,
                                            film.ctypes.data, C.byref(stats), C.byref(tuning) if tuning else None))
        return frames, film, stats.as_dict()


PHASES = ("camera", "closest-hit traversal", "occlusion traversal", "surface shading/maps", "BSDF sampling",
          "BSDF evaluation", "HDR importance sample+lookup+PDF")
phase_dtype = np.dtype([("seconds", "<f8"), ("calls", "<u8"), ("checksum", "<f8")])


def phase_benchmark(scene, camera, width=320, height=180, count=400000, seed=42):
    """cr_gpu_phase_benchmark: {phase: (seconds, calls, checksum)} in tests/benchmark.cpp's order."""
    out = np.zeros(len(PHASES), phase_dtype)
    check(lib.cr_gpu_phase_benchmark(scene.handle, C.byref(camera), width, height, count, seed, out.ctypes.data))
    return {name: (float(r["seconds"]), int(r["calls"]), float(r["checksum"])) for name, r in zip(PHASES, out)}


def display_thresholds(exposure=0.0):
    out = np.zeros(256, np.float32)
    check(lib.cr_display_thresholds(exposure, out.ctypes.data))
    return out


def encode(film, fmt=ENCODE_SRGB8, exposure=0.0, device=0):
    """A host film (H, W, 3) float32 encoded on the device (cr_gpu_encode): bytes."""
    film = np.ascontiguousarray(film, dtype=np.float32)
    h, w = film.shape[0], film.shape[1]
    size = C.c_uint64(0)
    check(lib.cr_gpu_encode(film.ctypes.data, w, h, fmt, exposure, device, None, 0, C.byref(size)))
    out = np.zeros(max(1, size.value), np.uint8)
    check(lib.cr_gpu_encode(film.ctypes.data, w, h, fmt, exposure, device, out.ctypes.data, size.value, C.byref(size)))
    return out[:size.value].tobytes()


def rel_mse(x, ref, eps=1e-2):
    """Relative MSE: mean over pixels and channels of (x - r)^2 / (r^2 + eps)."""
    x = np.asarray(x, np.float64)
    r = np.asarray(ref, np.float64)
    return float(np.mean((x - r) ** 2 / (r ** 2 + eps)))


def relative_l1(x, ref):
    """tests/image_metrics.cpp's score: sum |a - b| / sum a over RGB."""
    x = np.asarray(x, np.float64)
    r = np.asarray(ref, np.float64)
    return float(np.abs(x - r).sum() / max(1e-12, r.sum()))


class JobSpec:
    """A render job: scene, camera, options, optional progressive frames. After the job ends,
    .film (H, W, 3) float32 (when want_film), .frames [(samples_done, bytes)], .status,
    .error, .stats and the engine-clock times are filled in."""

    def __init__(self, scene, camera, options, every=0, fmt=ENCODE_SRGB8, exposure=0.0, want_film=True, keep_frames=True):
        self.scene, self.camera, self.options = scene, camera, options
        self.film = np.zeros((options.height, options.width, 3), np.float32) if want_film else None
        self.frames = []
        self.frame_times = []
        self.job = Job()
        j = self.job
        j.scene = scene.handle
        j.camera = camera
        j.options = options
        j.film_rgb = self.film.ctypes.data if want_film else None
        j.every_samples = every
        j.format = fmt
        j.exposure = exposure
        self._clock = None
        keep = keep_frames

        def on_frame(done, data, size, user):
            self.frames.append((done, C.string_at(data, size) if keep else size))

        self._cb = FRAME_FN(on_frame) if every else FRAME_FN(0)
        j.on_frame = self._cb

    @property
    def status(self):
        return self.job.status

    @property
    def error(self):
        return self.job.error.decode()

    @property
    def stats(self):
        return self.job.stats.as_dict()

    @property
    def times(self):
        j = self.job
        return {"submitted": j.submitted_at, "started": j.started_at, "first_frame": j.first_frame_at, "finished": j.finished_at}


def render_batch(specs, tuning=None):
    """cr_gpu_render_batch over JobSpecs; returns the engine stats (jobs report their own)."""
    arr = (Job * len(specs))()
    for i, sp in enumerate(specs):
        arr[i] = sp.job
    st = EngineStats()
    status = lib.cr_gpu_render_batch(C.cast(arr, C.c_void_p), len(specs), C.byref(tuning) if tuning else None, C.byref(st))
    for i, sp in enumerate(specs):
        sp.job = arr[i]
    if status != 0 and all(sp.job.status == 0 for sp in specs):  # an engine failure, not a job's
        raise CrError(status, last_error())
    return st.as_dict()


def autotune_batch(specs, base=None, trials=None):
    """cr_gpu_autotune_batch_trials: the chosen EngineTuning; the trials it ran (dicts) are
    appended to `trials` when a list is given."""
    arr = (Job * len(specs))()
    for i, sp in enumerate(specs):
        arr[i] = sp.job
    t = base if base is not None else EngineTuning.make()
    table = (AutotuneTrial * 64)()
    n = C.c_uint32(0)
    check(lib.cr_gpu_autotune_batch_trials(C.cast(arr, C.c_void_p), len(specs), C.byref(t), C.cast(table, C.c_void_p),
                                           len(table), C.byref(n)))
    if trials is not None:
        trials.extend(table[i].as_dict() for i in range(min(n.value, len(table))))
    return t


class Server:
    """cr_server: continuous batching on one device."""

    def __init__(self, device=0, tuning=None):
        h = C.c_void_p()
        check(lib.cr_server_create(device, C.byref(tuning) if tuning else None, C.byref(h)))
        self.handle = h
        self._live = {}

    def clock(self):
        return lib.cr_server_clock(self.handle)

    def submit(self, spec):
        t = C.c_uint64(0)
        check(lib.cr_server_submit(self.handle, C.byref(spec.job), C.byref(t)))
        self._live[t.value] = spec
        return t.value

    def wait(self, ticket, timeout=-1.0):
        st = lib.cr_server_wait(self.handle, ticket, timeout)
        if st != 7:
            self._live.pop(ticket, None)
        return st

    def stats(self):
        s = EngineStats()
        check(lib.cr_server_stats(self.handle, C.byref(s)))
        return s.as_dict()

    def close(self):
        if self.handle:
            lib.cr_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Guide:
    """cr_guide: the path-guiding network on a device."""

    def __init__(self, device=0, seed=1):
        h = C.c_void_p()
        check(lib.cr_guide_create(device, seed, C.byref(h)))
        self.handle = h
        self.count = lib.cr_guide_parameter_count()

    def parameters(self):
        out = np.zeros(self.count, np.float32)
        check(lib.cr_guide_get_parameters(self.handle, out.ctypes.data))
        return out

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.count
        check(lib.cr_guide_set_parameters(self.handle, p.ctypes.data))

    def evaluate(self, features):
        f = np.ascontiguousarray(features, np.float32).reshape(-1, 9)
        out = np.zeros((len(f), 40), np.float32)
        check(lib.cr_guide_evaluate(self.handle, f.ctypes.data, len(f), out.ctypes.data))
        return out

    def gradients(self, samples):
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 13)
        g = np.zeros(self.count, np.float32)
        loss = C.c_double(0)
        check(lib.cr_guide_gradients(self.handle, s.ctypes.data, len(s), g.ctypes.data, C.byref(loss)))
        return g, loss.value

    def train(self, samples, steps, batch=4096, lr=1e-3):
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 13)
        loss = C.c_float(0)
        check(lib.cr_guide_train(self.handle, s.ctypes.data, len(s), steps, batch, lr, C.byref(loss)))
        return loss.value

    def close(self):
        if self.handle:
            lib.cr_guide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
