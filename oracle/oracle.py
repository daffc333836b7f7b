"""ctypes binding of the CPU restatement (oracle/liboracle.so, built from oracle/cr_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg; nothing in the product imports it. The restatement takes the finalized
triangle array and, for BVH traversal, the node/index arrays of Bvh::build; both arrays are
pinned bit-identical to the reference's own by tests/test_host_parity.py. Brute-force mode
(test_geometry.cpp:396-407) needs neither.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "cpu-renderer_b200"))
from cr_types import (Camera, EnvDesc, Image, Options, SceneDesc, hit_dtype, light_dtype, material_dtype,  # noqa: E402
                   node_dtype, ray_dtype, texture_dtype, triangle_dtype, INF, NO_TRIANGLE)

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError("oracle not built: " + LIB_PATH)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.oracle_last_error.restype, L.oracle_last_error.argtypes = C.c_size_t, [C.c_char_p, C.c_size_t]
        L.oracle_intersect.restype = C.c_int
        L.oracle_intersect.argtypes = [C.POINTER(SceneDesc), C.c_int, P, C.c_uint64, C.c_int, C.c_uint32, P, P]
        L.oracle_render.restype = C.c_int
        L.oracle_render.argtypes = [C.POINTER(SceneDesc), C.POINTER(EnvDesc), C.POINTER(Camera), C.POINTER(Options), C.c_int,
                                    P, P, C.POINTER(C.c_uint64)]
        L.oracle_encode.restype = C.c_int
        L.oracle_encode.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_float, P, C.c_uint64, C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _err():
    buf = C.create_string_buffer(4096)
    lib().oracle_last_error(buf, len(buf))
    raise OracleError(buf.value.decode())


def _desc(triangles, materials, lights=None, images=(), textures=None, bvh=None):
    keep = []
    t = np.ascontiguousarray(triangles, dtype=triangle_dtype)
    m = np.ascontiguousarray(materials, dtype=material_dtype)
    l = np.ascontiguousarray(lights if lights is not None else np.zeros(0, light_dtype), dtype=light_dtype)
    keep += [t, m, l]
    d = SceneDesc()
    d.triangles, d.triangle_count = (t.ctypes.data if len(t) else None), len(t)
    d.materials, d.material_count = m.ctypes.data, len(m)
    d.lights, d.light_count = (l.ctypes.data if len(l) else None), len(l)
    if images:
        arr = (Image * len(images))()
        for i, im in enumerate(images):
            im = np.ascontiguousarray(im, dtype=np.float32)
            keep.append(im)
            arr[i] = Image(im.shape[1], im.shape[0], im.ctypes.data)
        keep.append(arr)
        d.images, d.image_count = C.cast(arr, C.c_void_p).value, len(images)
    if textures is not None and len(textures):
        tx = np.ascontiguousarray(textures, dtype=texture_dtype)
        keep.append(tx)
        d.textures, d.texture_count = tx.ctypes.data, len(tx)
    if bvh is not None:
        nodes = np.ascontiguousarray(bvh[0], dtype=node_dtype)
        idx = np.ascontiguousarray(bvh[1], dtype=np.uint32)
        keep += [nodes, idx]
        d.bvh_nodes, d.bvh_node_count = nodes.ctypes.data, len(nodes)
        d.bvh_indices, d.bvh_index_count = idx.ctypes.data, len(idx)
    return d, keep


def intersect(triangles, materials, rays, any_hit=False, ignore=NO_TRIANGLE, hits=None, bvh=None, images=(), textures=None):
    d, keep = _desc(triangles, materials, images=images, textures=textures, bvh=bvh)
    rays = np.ascontiguousarray(rays, dtype=ray_dtype)
    n = len(rays)
    if hits is None:
        hits = np.zeros(n, hit_dtype)
        hits["t"] = INF
    hits = np.ascontiguousarray(hits, dtype=hit_dtype).copy()
    found = np.zeros(n, np.uint8)
    if lib().oracle_intersect(C.byref(d), 0 if bvh is not None else 1, rays.ctypes.data, n, int(any_hit), ignore,
                              hits.ctypes.data, found.ctypes.data):
        _err()
    return found.astype(bool), hits


def render_arrays(triangles, materials, bvh, camera, options, env=None, lights=None, images=(), textures=None,
                  threads=None, per_sample=False):
    """cr::render restated; triangles must be finalized. Returns (film, per-sample or None, retries)."""
    d, keep = _desc(triangles, materials, lights=lights, images=images, textures=textures, bvh=bvh)
    e = env if env is not None else EnvDesc()
    film = np.zeros((options.height, options.width, 3), np.float32)
    ps = np.zeros((options.samples, options.height, options.width, 3), np.float32) if per_sample else None
    retries = C.c_uint64(0)
    n = threads or os.cpu_count() or 1
    if lib().oracle_render(C.byref(d), C.byref(e), C.byref(camera), C.byref(options), n, film.ctypes.data,
                           None if ps is None else ps.ctypes.data, C.byref(retries)):
        _err()
    return film, ps, retries.value


def render(sc, options, threads=None):
    """Convenience for a workload dict (triangles un-finalized): finalize and build the BVH
    with the host preparation pinned to the reference, then render."""
    import crgpu
    tris, _ = crgpu.finalize(sc["triangles"], sc["materials"], images=sc.get("images", ()), textures=sc.get("textures"))
    bvh = crgpu.build_bvh(tris)
    env = crgpu.env_desc(image=sc["env_image"]) if sc.get("env_image") is not None else None
    film, _, _ = render_arrays(tris, sc["materials"], bvh, sc["camera"], options, env=env, lights=sc.get("lights"),
                               images=sc.get("images", ()), textures=sc.get("textures"), threads=threads)
    return film


def encode(film, fmt=0, exposure=0.0):
    """io::writePng's pixels (fmt 0), RGBE quads (1) or io::writeHdr's file (2), restated."""
    film = np.ascontiguousarray(film, dtype=np.float32)
    h, w = (film.shape[0], film.shape[1]) if film.ndim == 3 else (0, 0)
    size = C.c_uint64(0)
    if lib().oracle_encode(film.ctypes.data, w, h, fmt, exposure, None, 0, C.byref(size)):
        _err()
    out = np.zeros(max(1, size.value), np.uint8)
    if lib().oracle_encode(film.ctypes.data, w, h, fmt, exposure, out.ctypes.data, size.value, C.byref(size)):
        _err()
    return out[:size.value].tobytes()
