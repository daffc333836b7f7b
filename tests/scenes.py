"""In-memory scene factories for the tests, following the shapes of the reference's own
fixtures (tests/test_geometry.cpp:42-62, tests/test_integrator.cpp:222-242,
tests/test_transport_edges.cpp:25-52). All arrays are plain cr_* records."""
import math

import numpy as np

from crgpu import (Camera, Options, new_lights, new_materials, new_triangles, ray_dtype, texture_dtype,
                   WRAP_CLAMP, WRAP_REPEAT, ALPHA_MASK, LIGHT_DIRECTIONAL, INF)

f32 = np.float32


def tri(a=(0, 0, 0), b=(1, 0, 0), c=(0, 1, 0), material=0):
    """test_geometry.cpp:42-49: positions, UV0 (0,0),(1,0),(0,1), UV1 = UV0."""
    t = new_triangles(1)
    for k, (p, uv) in enumerate(zip((a, b, c), ((0, 0), (1, 0), (0, 1)))):
        t[0]["v"][k]["position"] = p
        t[0]["v"][k]["uv"][0] = uv
        t[0]["v"][k]["uv"][1] = uv
    t[0]["material"] = material
    return t


def cat(*ts):
    return np.concatenate(ts)


def quad(a, b, c, d, material=0, uvs=True):
    """test_integrator.cpp:222-231: (a,b,c) + (a,c,d), flat normal cross(b-a, c-a)."""
    a, b, c, d = (np.asarray(p, f32) for p in (a, b, c, d))
    n = np.cross(b - a, c - a).astype(f32)
    n = (n / np.float32(np.sqrt(np.dot(n, n)))).astype(f32)
    out = new_triangles(2)
    for i, (verts, uv) in enumerate((((a, b, c), ((0, 0), (1, 0), (1, 1))), ((a, c, d), ((0, 0), (1, 1), (0, 1))))):
        for k in range(3):
            out[i]["v"][k]["position"] = verts[k]
            out[i]["v"][k]["normal"] = n
            if uvs:
                out[i]["v"][k]["uv"][0] = uv[k]
        out[i]["material"] = material
    return out


def cube(material, h=0.7):
    """test_integrator.cpp:233-240: closed, outward cube."""
    return cat(
        quad((-h, -h, h), (h, -h, h), (h, h, h), (-h, h, h), material),
        quad((h, -h, -h), (-h, -h, -h), (-h, h, -h), (h, h, -h), material),
        quad((-h, -h, -h), (-h, -h, h), (-h, h, h), (-h, h, -h), material),
        quad((h, -h, h), (h, -h, -h), (h, h, -h), (h, h, h), material),
        quad((-h, h, h), (h, h, h), (h, h, -h), (-h, h, -h), material),
        quad((-h, -h, -h), (h, -h, -h), (h, -h, h), (-h, -h, h), material))


def slab(h=100.0):
    """test_transport_edges.cpp:37-52: closed one-unit absorbing glass slab."""
    m = new_materials(1)
    m[0]["metallic"] = 0; m[0]["roughness"] = 0.6; m[0]["transmission"] = 1; m[0]["ior"] = 1.5
    m[0]["thickness"] = 1; m[0]["attenuation_distance"] = 1; m[0]["attenuation_color"] = (0.5, 0.8, 1)
    t = cat(quad((-h, -h, 1), (h, -h, 1), (h, h, 1), (-h, h, 1), uvs=False),
            quad((h, -h, 0), (-h, -h, 0), (-h, h, 0), (h, h, 0), uvs=False),
            quad((-h, -h, 0), (-h, -h, 1), (-h, h, 1), (-h, h, 0), uvs=False),
            quad((h, -h, 1), (h, -h, 0), (h, h, 0), (h, h, 1), uvs=False),
            quad((-h, h, 1), (h, h, 1), (h, h, 0), (-h, h, 0), uvs=False),
            quad((-h, -h, 0), (h, -h, 0), (h, -h, 1), (-h, -h, 1), uvs=False))
    return t, m


def rays(origins, directions, tmin=0.0, tmax=INF, low=None):
    origins = np.atleast_2d(np.asarray(origins, f32))
    directions = np.atleast_2d(np.asarray(directions, f32))
    n = max(len(origins), len(directions))
    r = np.zeros(n, ray_dtype)
    r["origin"] = origins
    r["direction"] = directions
    r["tmin"] = tmin
    r["tmax"] = tmax
    if low is not None:
        r["origin_low"] = low
    return r


def normalize(v):
    v = np.asarray(v, f32)
    return (v / np.sqrt(np.sum(v * v, axis=-1, keepdims=True))).astype(f32)


def frame_x(n):
    """math.h:95-99 Frame(n).x and .y in float32."""
    n = np.asarray(n, f32)
    helper = np.array((0, 0, 1), f32) if abs(n[2]) < f32(0.999) else np.array((0, 1, 0), f32)
    x = normalize(np.cross(helper, n).astype(f32))
    y = np.cross(n, x).astype(f32)
    return x, y


def bvh_random_scene(seed=0x75645321, count=450):
    """The mixed-material random-triangle family of test_geometry.cpp:533-550: two-sided,
    alpha-masked (2x2 linear Repeat texture with offset), one-sided, and transmissive."""
    rng = np.random.default_rng(seed)
    m = new_materials(4)
    m[0]["double_sided"] = 1
    m[1]["double_sided"] = 1
    m[1]["alpha_mode"] = ALPHA_MASK
    m[1]["base_color_texture"]["texture"] = 0
    m[1]["base_color_texture"]["offset"] = (-0.1, 0.2)
    m[3]["transmission"] = 0.8
    image = np.array([[[1, 1, 1, 0], [1, 1, 1, 1]], [[1, 1, 1, 1], [1, 1, 1, 0]]], f32)
    tex = np.zeros(1, texture_dtype)
    tex[0] = (0, WRAP_REPEAT, WRAP_REPEAT, 1)
    ts = []
    for i in range(count):
        center = rng.uniform(-10, 10, 3).astype(f32)
        n = normalize(rng.uniform(-1, 1, 3))
        fx, fy = frame_x(n)
        s = f32(rng.uniform(0.1, 2))
        ts.append(tri(center - fx * s - fy * s, center + fx * s, center + fy * s, i % 4))
    t = cat(*ts)
    return t, m, [image], tex


def bvh_random_rays(triangles, seed=7, count=6500):
    rng = np.random.default_rng(seed)
    out = np.zeros(count, ray_dtype)
    upper = np.full(count, INF)
    for i in range(count):
        o = rng.uniform(-15, 15, 3).astype(f32)
        d = normalize(rng.uniform(-1, 1, 3))
        if i % 2 == 0:
            t = triangles[i % len(triangles)]
            p = (t["v"][0]["position"] * f32(0.5) + t["v"][1]["position"] * f32(0.2) + t["v"][2]["position"] * f32(0.3)).astype(f32)
            d = normalize(p - o)
        if i % 5 == 0:
            d = (d * f32(3)).astype(f32)
        out[i]["origin"] = o
        out[i]["direction"] = d
        out[i]["tmin"] = 0.5 if i % 7 == 0 else 0
        out[i]["tmax"] = rng.uniform(1, 30) if i % 3 == 0 else INF
        if i % 11 == 0:
            upper[i] = 5
    return out, upper


def room_camera():
    """test_integrator.cpp:242."""
    return Camera.make(position=(0, 0, 4), forward=(0, 0, -1), yfov=0.65)


def directional(direction, intensity):
    l = new_lights(1)
    l[0]["type"] = LIGHT_DIRECTIONAL
    l[0]["direction"] = direction
    l[0]["intensity"] = intensity
    return l
