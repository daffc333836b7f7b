"""ctypes binding of the reference itself (oracle/_ref/libcr_ref.so).

TEST INFRASTRUCTURE ONLY. This is the checker: the unmodified CPU-Renderer compiled from
its own sources (src/geometry.cpp, src/bsdf.cpp, src/render.cpp) plus oracle/ref_shim.cpp.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference arm use it.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "cpu-renderer_b200"))
from cr_types import (Camera, EnvDesc, Options, SceneDesc, Stats, hit_dtype, light_dtype, material_dtype,  # noqa: E402
                   node_dtype, ray_dtype, triangle_dtype, texture_dtype, Image, INF, NO_TRIANGLE)

LIB_PATH = os.path.join(HERE, "_ref", "libcr_ref.so")


def available():
    return os.path.exists(LIB_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError("reference library not built: " + LIB_PATH)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        sig = {
            "ref_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
            "ref_scene_new": (P, [C.POINTER(SceneDesc)]),
            "ref_scene_free": (None, [P]),
            "ref_scene_finalize": (C.c_int, [P, C.c_char_p, C.c_size_t]),
            "ref_scene_triangle_count": (C.c_uint64, [P]),
            "ref_scene_get_triangles": (None, [P, P]),
            "ref_bvh_new": (P, [P]),
            "ref_bvh_free": (None, [P]),
            "ref_bvh_node_count": (C.c_uint64, [P]),
            "ref_bvh_export": (None, [P, P, P]),
            "ref_intersect": (C.c_int, [P, P, P, C.c_uint64, C.c_int, C.c_uint32, P, P]),
            "ref_intersect_rays": (C.c_int, [P, P, P, P, C.c_uint64, C.c_int, P, P, C.c_int]),
            "ref_intersect_triangle": (C.c_int, [P, P, P]),
            "ref_bounds_intersect": (C.c_int, [P, P, P, C.POINTER(C.c_float)]),
            "ref_camera_generate": (C.c_int, [C.POINTER(Camera), P, P, C.c_uint64, C.c_int, C.c_int, P]),
            "ref_offset_ray": (C.c_int, [P, P, P, C.c_float, P]),
            "ref_sample_seed": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64]),
            "ref_env_new": (P, [C.POINTER(EnvDesc), C.c_float]),
            "ref_env_free": (None, [P]),
            "ref_env_export": (C.c_uint64, [P, P, P, P]),
            "ref_env_sample": (None, [P, C.POINTER(C.c_uint64), C.c_uint64, P, P]),
            "ref_env_eval": (None, [P, P, C.c_uint64, P, P]),
            "ref_sample_bsdf": (None, [P, P, C.POINTER(C.c_uint64), C.c_uint64, P]),
            "ref_evaluate_bsdf": (None, [P, P, P, C.c_uint64, P]),
            "ref_options_validate": (C.c_int, [C.POINTER(Options)]),
            "ref_render": (C.c_int, [P, P, C.POINTER(Camera), P, C.POINTER(Options), P, C.POINTER(Stats)]),
            "ref_write_png": (C.c_int, [C.c_char_p, C.c_int, C.c_int, P, C.c_float]),
            "ref_write_hdr": (C.c_int, [C.c_char_p, C.c_int, C.c_int, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


class RefError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


def _err(code):
    buf = C.create_string_buffer(4096)
    lib().ref_last_error(buf, len(buf))
    raise RefError(code, buf.value.decode())


def _ptr(a):
    return None if a is None or len(a) == 0 else a.ctypes.data


class RefScene:
    """cr::Scene (+ optional cr::Bvh) owned by the reference library."""

    def __init__(self, triangles, materials, lights=None, images=(), textures=None, finalize=True):
        t = np.ascontiguousarray(triangles, dtype=triangle_dtype)
        m = np.ascontiguousarray(materials, dtype=material_dtype)
        l = np.ascontiguousarray(lights if lights is not None else np.zeros(0, light_dtype), dtype=light_dtype)
        d = SceneDesc()
        d.triangles, d.triangle_count = _ptr(t), len(t)
        d.materials, d.material_count = _ptr(m), len(m)
        d.lights, d.light_count = _ptr(l), len(l)
        self._keep = [t, m, l]
        if images:
            arr = (Image * len(images))()
            for i, im in enumerate(images):
                im = np.ascontiguousarray(im, dtype=np.float32)
                self._keep.append(im)
                arr[i] = Image(im.shape[1], im.shape[0], im.ctypes.data)
            self._keep.append(arr)
            d.images, d.image_count = C.cast(arr, C.c_void_p).value, len(images)
        if textures is not None and len(textures):
            tx = np.ascontiguousarray(textures, dtype=texture_dtype)
            self._keep.append(tx)
            d.textures, d.texture_count = tx.ctypes.data, len(tx)
        self.handle = lib().ref_scene_new(C.byref(d))
        if not self.handle:
            _err(2)
        self.bvh = None
        self.warnings = []
        if finalize:
            buf = C.create_string_buffer(8192)
            code = lib().ref_scene_finalize(self.handle, buf, len(buf))
            if code:
                _err(code)
            w = buf.value.decode()
            self.warnings = w.split("\n") if w else []

    def triangles(self):
        n = lib().ref_scene_triangle_count(self.handle)
        out = np.zeros(n, triangle_dtype)
        if n:
            lib().ref_scene_get_triangles(self.handle, out.ctypes.data)
        return out

    def build_bvh(self):
        if self.bvh:
            lib().ref_bvh_free(self.bvh)
        self.bvh = lib().ref_bvh_new(self.handle)
        if not self.bvh:
            _err(2)
        return self

    def bvh_arrays(self):
        n = lib().ref_bvh_node_count(self.bvh)
        nodes = np.zeros(max(1, n), node_dtype)
        idx = np.zeros(max(1, lib().ref_scene_triangle_count(self.handle)), np.uint32)
        lib().ref_bvh_export(self.bvh, nodes.ctypes.data, idx.ctypes.data)
        return nodes[:n].copy(), idx[:lib().ref_scene_triangle_count(self.handle)].copy()

    def intersect(self, rays, any_hit=False, ignore=NO_TRIANGLE, hits=None):
        rays = np.ascontiguousarray(rays, dtype=ray_dtype)
        n = len(rays)
        if hits is None:
            hits = np.zeros(n, hit_dtype)
            hits["t"] = INF
        hits = np.ascontiguousarray(hits, dtype=hit_dtype).copy()
        found = np.zeros(n, np.uint8)
        code = lib().ref_intersect(self.handle, self.bvh, _ptr(rays), n, int(any_hit), ignore, _ptr(hits), _ptr(found))
        if code:
            _err(code)
        return found.astype(bool), hits

    def intersect_rays(self, rays, ignores, any_hit=False, threads=None):
        """Bvh::intersect of every ray with its own ignoreTriangle, on several host threads;
        the incoming hit is the reference's default (t = +inf)."""
        rays = np.ascontiguousarray(rays, dtype=ray_dtype)
        ignores = np.ascontiguousarray(ignores, dtype=np.uint32)
        n = len(rays)
        hits = np.zeros(n, hit_dtype)
        hits["t"] = INF
        found = np.zeros(n, np.uint8)
        code = lib().ref_intersect_rays(self.handle, self.bvh, _ptr(rays), _ptr(ignores), n, int(any_hit), _ptr(hits),
                                        _ptr(found), int(threads or os.cpu_count() or 1))
        if code:
            _err(code)
        return found.astype(bool), hits

    def render(self, camera, options, env):
        film = np.zeros((options.height, options.width, 3), np.float32)
        stats = Stats()
        code = lib().ref_render(self.handle, self.bvh, C.byref(camera), env.handle, C.byref(options), film.ctypes.data,
                                C.byref(stats))
        if code:
            _err(code)
        return film, stats.as_dict()

    def close(self):
        if self.bvh:
            lib().ref_bvh_free(self.bvh)
            self.bvh = None
        if self.handle:
            lib().ref_scene_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefEnvironment:
    def __init__(self, constant=(0, 0, 0), image=None, rotation_degrees=0.0, intensity=1.0):
        e = EnvDesc()
        e.constant[:] = [float(x) for x in constant]
        e.intensity = float(intensity)
        self._keep = None
        if image is not None:
            image = np.ascontiguousarray(image, dtype=np.float32)
            self._keep = image
            e.pixels = image.ctypes.data
            e.height, e.width = image.shape[0], image.shape[1]
        self.handle = lib().ref_env_new(C.byref(e), float(rotation_degrees))
        if not self.handle:
            _err(2)
        self.image = image

    def export(self):
        n = 0 if self.image is None else self.image.shape[0] * self.image.shape[1]
        cdf = np.zeros(max(1, n), np.float64)
        ws = np.zeros(2, np.float64)
        ri = np.zeros(2, np.float32)
        lib().ref_env_export(self.handle, cdf.ctypes.data, ws.ctypes.data, ri.ctypes.data)
        return cdf[:n], ws, ri

    def sample(self, state, n):
        s = C.c_uint64(state)
        dirs = np.zeros((n, 3), np.float32)
        pdfs = np.zeros(n, np.float32)
        lib().ref_env_sample(self.handle, C.byref(s), n, dirs.ctypes.data, pdfs.ctypes.data)
        return dirs, pdfs, s.value

    def eval(self, dirs):
        dirs = np.ascontiguousarray(dirs, dtype=np.float32)
        rad = np.zeros_like(dirs)
        pdfs = np.zeros(len(dirs), np.float32)
        lib().ref_env_eval(self.handle, dirs.ctypes.data, len(dirs), rad.ctypes.data, pdfs.ctypes.data)
        return rad, pdfs

    def __del__(self):
        try:
            if self.handle:
                lib().ref_env_free(self.handle)
                self.handle = None
        except Exception:
            pass


def camera_generate(camera, px, py, width, height):
    px = np.ascontiguousarray(px, np.float32)
    py = np.ascontiguousarray(py, np.float32)
    out = np.zeros(len(px), ray_dtype)
    code = lib().ref_camera_generate(C.byref(camera), px.ctypes.data, py.ctypes.data, len(px), width, height, out.ctypes.data)
    if code:
        _err(code)
    return out


def sample_seed(seed, pixel, sample):
    return lib().ref_sample_seed(seed, pixel, sample)


def intersect_triangle(tri, ray, hit=None):
    t = np.ascontiguousarray(np.atleast_1d(tri), dtype=triangle_dtype)
    r = np.ascontiguousarray(np.atleast_1d(ray), dtype=ray_dtype)
    if hit is None:
        hit = np.zeros(1, hit_dtype)
        hit["t"] = INF
    h = np.ascontiguousarray(np.atleast_1d(hit), dtype=hit_dtype).copy()
    ok = lib().ref_intersect_triangle(t.ctypes.data, r.ctypes.data, h.ctypes.data)
    return bool(ok), h[0]


def validate_options(options):
    code = lib().ref_options_validate(C.byref(options))
    if code:
        _err(code)


def write_png(path, film, exposure=0.0):
    """io::writePng (image.cpp:193-212) of a (H, W, 3) float film."""
    film = np.ascontiguousarray(film, dtype=np.float32)
    h, w = (film.shape[0], film.shape[1]) if film.ndim == 3 else (0, 0)
    rc = lib().ref_write_png(str(path).encode(), w, h, film.ctypes.data, exposure)
    if rc:
        _err(rc)


def write_hdr(path, film):
    """io::writeHdr (image.cpp:216-230) of a (H, W, 3) float film."""
    film = np.ascontiguousarray(film, dtype=np.float32)
    h, w = (film.shape[0], film.shape[1]) if film.ndim == 3 else (0, 0)
    rc = lib().ref_write_hdr(str(path).encode(), w, h, film.ctypes.data)
    if rc:
        _err(rc)
