"""Seeded synthetic scenes for the two plain-tracer workloads.

room_scene          256x256, 16 spp, 8 bounces: a closed 2x2x2 room of 10 inward quads (20
                    triangles), two 0.4x0.4 emitter quads of radiance 15 (4 triangles) and 64
                    random triangles (edges 0.05-0.4), 70% GGX conductors (roughness U[0.05,1],
                    albedo U[0.2,0.9]^3, two-sided) and 30% thin smooth dielectrics (IOR 1.5).
                    No environment. 88 triangles.

sphere_grid_scene   1920x1080, 64 spp, 16 bounces: 20x20 closed, radially displaced spheres
                    (77 slices x 18 stacks = 2,618 triangles each, displacement amplitude 0.1)
                    over a 16x43-quad ground grid (1,376 triangles): 1,048,576 triangles in
                    total. Half the spheres are GGX conductors (roughness U[0.02,0.6]), half are
                    smooth closed dielectrics (IOR U[1.3,1.7]). A 2048x1024 RGB equirect sky of
                    log-normal (mu=0, sigma=1) texels plus a 0.5-degree sun disk of radiance 5e4.

cluttered_room_scene / uneven_scene_mix
                    the multi-scene mixes: config-1 rooms whose random triangles number from
                    10^3 to 2x10^6 (log-uniform over the mix; sizes shrink by sqrt(64/n) so the
                    clutter's area stays the room's, unless literal), drawn from a palette of 64
                    materials with the room's 70/30 conductor/dielectric split; each job draws
                    a resolution from {256^2, 512^2, 1024^2, 1920x1080}, samples from
                    {1, 4, 16, 64}, 12 bounces.

All draws come from numpy's PCG64 with fixed seeds, so every call returns identical arrays.
Triangles are returned un-finalized (Scene::finalize computes areas and normals).
"""
import math

import numpy as np

from cr_types import Camera, Options, new_materials, new_triangles

ROOM_SEED = 0x5EED0001
GRID_SEED = 0x5EED0002


def _quad(tris, a, b, c, d, material, inward=None):
    """Two triangles (a,b,c), (a,c,d), wound so that cross(b-a, c-a) points along `inward`."""
    a, b, c, d = (np.asarray(p, np.float32) for p in (a, b, c, d))
    n = np.cross(b - a, c - a)
    if inward is not None and np.dot(n, inward) < 0:
        b, d = d, b
        n = -n
    n = (n / np.linalg.norm(n)).astype(np.float32)
    for verts, uvs in (((a, b, c), ((0, 0), (1, 0), (1, 1))), ((a, c, d), ((0, 0), (1, 1), (0, 1)))):
        t = new_triangles(1)[0]
        for k in range(3):
            t["v"][k]["position"] = verts[k]
            t["v"][k]["normal"] = n
            t["v"][k]["uv"][0] = uvs[k]
            t["v"][k]["uv"][1] = uvs[k]
        t["material"] = material
        tris.append(t)


def room_scene(seed=ROOM_SEED):
    """Returns dict(triangles, materials, camera, options, env=None)."""
    rng = np.random.default_rng(seed)
    mats = new_materials(4)
    # 0 white walls, 1 red wall, 2 green wall, 3 emitter; random triangles get their own.
    for i, col in enumerate(((0.75, 0.75, 0.75), (0.7, 0.2, 0.15), (0.2, 0.6, 0.2))):
        mats[i]["base_color"][:3] = col
        mats[i]["metallic"] = 0.0
        mats[i]["roughness"] = 1.0
    mats[3]["base_color"][:3] = 0.0
    mats[3]["metallic"] = 0.0
    mats[3]["emission"] = 15.0
    tris = []
    lo, hi = -1.0, 1.0
    # floor, ceiling, left, right: two quads each (split at z=0); back and front: one each.
    for z0, z1 in ((lo, 0.0), (0.0, hi)):
        _quad(tris, (lo, 0, z0), (hi, 0, z0), (hi, 0, z1), (lo, 0, z1), 0, inward=(0, 1, 0))
        _quad(tris, (lo, 2, z0), (hi, 2, z0), (hi, 2, z1), (lo, 2, z1), 0, inward=(0, -1, 0))
        _quad(tris, (lo, 0, z0), (lo, 2, z0), (lo, 2, z1), (lo, 0, z1), 1, inward=(1, 0, 0))
        _quad(tris, (hi, 0, z0), (hi, 2, z0), (hi, 2, z1), (hi, 0, z1), 2, inward=(-1, 0, 0))
    _quad(tris, (lo, 0, lo), (hi, 0, lo), (hi, 2, lo), (lo, 2, lo), 0, inward=(0, 0, 1))
    _quad(tris, (lo, 0, hi), (hi, 0, hi), (hi, 2, hi), (lo, 2, hi), 0, inward=(0, 0, -1))
    # two 0.4 x 0.4 emitters just below the ceiling, facing down
    for cx in (-0.45, 0.45):
        y = 1.995
        _quad(tris, (cx - 0.2, y, -0.2), (cx + 0.2, y, -0.2), (cx + 0.2, y, 0.2), (cx - 0.2, y, 0.2), 3, inward=(0, -1, 0))
    # 64 random triangles inside the room
    extra = []
    ilo = np.array([-0.9, 0.1, -0.9]); ihi = np.array([0.9, 1.9, 0.9])
    while len(extra) < 64:
        v0 = rng.uniform(ilo, ihi)
        dirs = rng.normal(size=(2, 3))
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        lens = rng.uniform(0.05, 0.4, size=2)
        v1 = v0 + lens[0] * dirs[0]
        v2 = v0 + lens[1] * dirs[1]
        e = np.linalg.norm(v2 - v1)
        area = 0.5 * np.linalg.norm(np.cross(v1 - v0, v2 - v0))
        inside = np.all((np.stack([v1, v2]) > ilo) & (np.stack([v1, v2]) < ihi))
        if not (0.05 <= e <= 0.4) or area < 1e-4 or not inside:
            continue
        extra.append((v0, v1, v2))
    rand_mats = new_materials(64)
    kinds = rng.uniform(size=64) < 0.7
    for i in range(64):
        m = rand_mats[i]
        m["double_sided"] = 1
        if kinds[i]:  # GGX conductor
            m["metallic"] = 1.0
            m["roughness"] = rng.uniform(0.05, 1.0)
            m["base_color"][:3] = rng.uniform(0.2, 0.9, size=3)
        else:  # thin smooth dielectric
            m["metallic"] = 0.0
            m["transmission"] = 1.0
            m["ior"] = 1.5
            m["roughness"] = 0.0
            m["thickness"] = 0.0
            m["base_color"][:3] = 1.0
    for i, (v0, v1, v2) in enumerate(extra):
        t = new_triangles(1)[0]
        for k, p in enumerate((v0, v1, v2)):
            t["v"][k]["position"] = p.astype(np.float32)
        t["material"] = 4 + i
        tris.append(t)
    materials = np.concatenate([mats, rand_mats])
    triangles = np.array(tris, dtype=tris[0].dtype)
    camera = Camera.make(position=(0, 1, 0.98), forward=(0, 0, -1), right=(1, 0, 0), up=(0, 1, 0),
                         yfov=math.radians(60.0))
    options = Options.make(width=256, height=256, samples=16, bounces=8, threads=0, seed=42)
    return dict(triangles=triangles, materials=materials, lights=None, camera=camera, options=options, env=None,
                name="room-88tri-256x256-16spp-d8")


def _sphere_mesh(slices=77, stacks=18):
    """Unit lat-long sphere: poles plus (stacks-1) rings; 2*slices*(stacks-1) outward triangles."""
    rings = []
    for i in range(1, stacks):
        th = math.pi * i / stacks
        for j in range(slices):
            ph = 2 * math.pi * j / slices
            rings.append((math.sin(th) * math.cos(ph), math.cos(th), math.sin(th) * math.sin(ph)))
    verts = np.array([(0.0, 1.0, 0.0)] + rings + [(0.0, -1.0, 0.0)], np.float64)
    top, bottom = 0, len(verts) - 1
    ring = lambda i, j: 1 + (i * slices) + (j % slices)
    faces = []
    for j in range(slices):
        faces.append((top, ring(0, j + 1), ring(0, j)))
    for i in range(stacks - 2):
        for j in range(slices):
            a, b = ring(i, j), ring(i, j + 1)
            c, d = ring(i + 1, j), ring(i + 1, j + 1)
            faces.append((a, b, d))
            faces.append((a, d, c))
    for j in range(slices):
        faces.append((bottom, ring(stacks - 2, j), ring(stacks - 2, j + 1)))
    faces = np.array(faces, np.int64)
    # orient outward
    p = verts[faces]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    flip = np.einsum("ij,ij->i", n, p.mean(axis=1)) < 0
    faces[flip] = faces[flip][:, [0, 2, 1]]
    return verts, faces


def sky_image(width=2048, height=1024, seed=GRID_SEED + 1, sun_elevation_deg=35.0, sun_azimuth_deg=60.0,
              sun_diameter_deg=0.5, sun_radiance=5e4, background=True):
    """RGBA float32 (H, W, 4): log-normal(0, 1) grey texels (black without background) and a
    sun disk."""
    rng = np.random.default_rng(seed)
    img = np.ones((height, width, 4), np.float32)
    img[..., :3] = np.exp(rng.normal(0.0, 1.0, size=(height, width, 1))).astype(np.float32) if background else 0.0
    theta = (np.arange(height) + 0.5) / height * math.pi
    phi = ((np.arange(width) + 0.5) / width - 0.5) * 2 * math.pi
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    d = np.stack([st * np.cos(phi)[None, :], np.broadcast_to(ct, (height, width)), st * np.sin(phi)[None, :]], -1)
    el, az = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sun = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    inside = d @ sun >= math.cos(math.radians(sun_diameter_deg / 2))
    img[inside, :3] = sun_radiance
    return img


def sphere_grid_scene(seed=GRID_SEED, width=1920, height=1080, samples=64, bounces=16, sky=True):
    """Returns dict(triangles, materials, camera, options, env_image)."""
    rng = np.random.default_rng(seed)
    unit, faces = _sphere_mesh()
    grid, spacing, radius, amp = 20, 1.1, 0.38, 0.1
    mats = new_materials(grid * grid + 1)
    ground = grid * grid
    mats[ground]["metallic"] = 0.0
    mats[ground]["roughness"] = 0.8
    mats[ground]["base_color"][:3] = 0.5
    kinds = rng.uniform(size=grid * grid) < 0.5
    tri_blocks = []
    for k in range(grid * grid):
        i, j = divmod(k, grid)
        m = mats[k]
        if kinds[k]:
            m["metallic"] = 1.0
            m["roughness"] = rng.uniform(0.02, 0.6)
            m["base_color"][:3] = rng.uniform(0.3, 0.95, size=3)
        else:
            m["metallic"] = 0.0
            m["transmission"] = 1.0
            m["ior"] = rng.uniform(1.3, 1.7)
            m["roughness"] = 0.0
            m["thickness"] = 1.0
            m["base_color"][:3] = 1.0
        ph = rng.uniform(0, 2 * math.pi, size=3)
        fr = rng.uniform(2.0, 4.0, size=3)
        noise = np.sin(fr[0] * unit[:, 0] + ph[0]) * np.sin(fr[1] * unit[:, 1] + ph[1]) * np.sin(fr[2] * unit[:, 2] + ph[2])
        r = radius + amp * noise
        center = np.array([(i - (grid - 1) / 2) * spacing, radius + amp, (j - (grid - 1) / 2) * spacing])
        verts = unit * r[:, None] + center
        # smooth vertex normals: area-weighted face normals
        p = verts[faces]
        fn = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        vn = np.zeros_like(verts)
        for c in range(3):
            np.add.at(vn, faces[:, c], fn)
        vn /= np.linalg.norm(vn, axis=1, keepdims=True)
        t = new_triangles(len(faces))
        t["v"]["position"] = verts[faces].astype(np.float32)
        t["v"]["normal"] = vn[faces].astype(np.float32)
        t["material"] = k
        tri_blocks.append(t)
    # ground grid: 16 x 43 quads over the sphere footprint
    nx, nz = 16, 43
    ext = grid * spacing / 2 + 1.0
    xs = np.linspace(-ext, ext, nx + 1)
    zs = np.linspace(-ext, ext, nz + 1)
    g = new_triangles(2 * nx * nz)
    q = 0
    for a in range(nx):
        for b in range(nz):
            p00 = (xs[a], 0.0, zs[b]); p10 = (xs[a + 1], 0.0, zs[b])
            p11 = (xs[a + 1], 0.0, zs[b + 1]); p01 = (xs[a], 0.0, zs[b + 1])
            for tri in ((p00, p01, p11), (p00, p11, p10)):  # cross(b-a, c-a) = +y
                g[q]["v"]["position"] = np.array(tri, np.float32)
                g[q]["v"]["normal"] = (0.0, 1.0, 0.0)
                g[q]["material"] = ground
                q += 1
    tri_blocks.append(g)
    triangles = np.concatenate(tri_blocks)
    assert len(triangles) == 1 << 20
    camera = Camera.make(position=(0.0, 6.0, 17.0), forward=(0.0, -6.0, -17.0), right=(1, 0, 0), up=(0, 1, 0),
                         yfov=math.radians(40.0))
    options = Options.make(width=width, height=height, samples=samples, bounces=bounces, threads=0, seed=42)
    return dict(triangles=triangles, materials=mats, lights=None, camera=camera, options=options,
                env_image=sky_image() if sky else None,
                name="sphere-grid-1M-1920x1080-64spp-d16")


def caustic_scene(width=320, height=180, samples=64, bounces=16):
    """The learned-proposal workload: the sphere grid with every sphere a smooth closed
    dielectric of IOR 1.5 or a GGX conductor of roughness 0.05 (the same 50/50 draw), lit only
    by the sun disk (black sky). The ground keeps its rough, non-metallic material: it is the
    surface that receives the caustics (with every surface specular or near-specular, no light
    path through the dielectrics could end at a surface the camera sees diffusely)."""
    sc = sphere_grid_scene(width=width, height=height, samples=samples, bounces=bounces, sky=False)
    m = sc["materials"]
    spheres = len(m) - 1
    metal = m["metallic"][:spheres] == 1.0
    m["roughness"][:spheres][metal] = 0.05
    m["ior"][:spheres][~metal] = 1.5
    sc["env_image"] = sky_image(width=1024, height=512, background=False)
    sc["name"] = f"caustic-sphere-grid-{width}x{height}"
    return sc


def sunlit_room_scene(width=64, height=64, samples=64, bounces=8, hole=0.2):
    """A closed diffuse 2x2x2 room lit only by the sun disk through a square opening in the
    ceiling (half-width `hole`): the sun lands on a patch of the back wall and everything else
    is lit by that patch, the case where BSDF sampling rarely finds the light and a guide can."""
    mats = new_materials(2)
    for m, col in ((mats[0], 0.75), (mats[1], 0.6)):
        m["metallic"] = 0.0
        m["roughness"] = 1.0
        m["base_color"][:3] = col
    tris = []
    lo, hi = -1.0, 1.0
    _quad(tris, (lo, 0, lo), (hi, 0, lo), (hi, 0, hi), (lo, 0, hi), 1, inward=(0, 1, 0))      # floor
    _quad(tris, (lo, 0, lo), (lo, 2, lo), (lo, 2, hi), (lo, 0, hi), 0, inward=(1, 0, 0))      # left
    _quad(tris, (hi, 0, lo), (hi, 2, lo), (hi, 2, hi), (hi, 0, hi), 0, inward=(-1, 0, 0))     # right
    _quad(tris, (lo, 0, lo), (hi, 0, lo), (hi, 2, lo), (lo, 2, lo), 0, inward=(0, 0, 1))      # back
    _quad(tris, (lo, 0, hi), (hi, 0, hi), (hi, 2, hi), (lo, 2, hi), 0, inward=(0, 0, -1))     # front
    h = hole  # ceiling around the opening [-h, h]^2
    for (x0, x1, z0, z1) in ((lo, hi, lo, -h), (lo, hi, h, hi), (lo, -h, -h, h), (h, hi, -h, h)):
        _quad(tris, (x0, 2, z0), (x1, 2, z0), (x1, 2, z1), (x0, 2, z1), 0, inward=(0, -1, 0))
    camera = Camera.make(position=(0, 1, 0.98), forward=(0, 0, -1), right=(1, 0, 0), up=(0, 1, 0),
                         yfov=math.radians(70.0))
    options = Options.make(width=width, height=height, samples=samples, bounces=bounces, threads=0, seed=42)
    return dict(triangles=np.array(tris, dtype=tris[0].dtype), materials=mats, camera=camera, options=options,
                env_image=sky_image(width=1024, height=512, background=False), name="sunlit-room")


MIX_SEED = 0x5EED0003
MIX_RESOLUTIONS = ((256, 256), (512, 512), (1024, 1024), (1920, 1080))
MIX_SAMPLES = (1, 4, 16, 64)


def cluttered_room_scene(triangle_count, seed, literal=False):
    """A config-1 room (walls, two emitters) holding triangle_count - 24 random triangles
    (vertices in the interior) over a 64-material palette. The room's own random triangles
    have edges 0.05-0.4 and area >= 1e-4 for 64 of them; with `literal` every scene keeps
    those sizes, otherwise they shrink by sqrt(64 / n) so that n triangles cover the room's
    area of clutter (at 2x10^6 literal triangles thousands of triangles overlap every point
    of the room and every ray tests thousands of them)."""
    base = room_scene(seed)
    rng = np.random.default_rng(seed + 1)
    walls = base["triangles"][:24]
    n = max(0, int(triangle_count) - len(walls))
    k = 1.0 if literal or n <= 64 else math.sqrt(64.0 / n)
    ilo = np.array([-0.9, 0.1, -0.9]); ihi = np.array([0.9, 1.9, 0.9])
    chunks, have = [], 0
    while have < n:
        m = int((n - have) * 1.6) + 64
        v0 = rng.uniform(ilo, ihi, size=(m, 3))
        d = rng.normal(size=(m, 2, 3))
        d /= np.linalg.norm(d, axis=2, keepdims=True)
        lens = rng.uniform(0.05 * k, 0.4 * k, size=(m, 2, 1))
        v1 = v0 + lens[:, 0] * d[:, 0]
        v2 = v0 + lens[:, 1] * d[:, 1]
        e = np.linalg.norm(v2 - v1, axis=1)
        area = 0.5 * np.linalg.norm(np.cross(v1 - v0, v2 - v0), axis=1)
        inside = np.all((v1 > ilo) & (v1 < ihi) & (v2 > ilo) & (v2 < ihi), axis=1)
        ok = (e >= 0.05 * k) & (e <= 0.4 * k) & (area >= 1e-4 * k * k) & inside
        pts = np.stack([v0, v1, v2], axis=1)[ok][: n - have]
        chunks.append(pts)
        have += len(pts)
    pts = np.concatenate(chunks) if chunks else np.zeros((0, 3, 3))
    tris = new_triangles(len(walls) + n)
    tris[: len(walls)] = walls
    tris["v"]["position"][len(walls):] = pts.astype(np.float32)
    palette = base["materials"][4:]  # the room's 64 random materials: 70% conductors, 30% dielectrics
    tris["material"][len(walls):] = 4 + rng.integers(0, len(palette), size=n)
    return dict(triangles=tris, materials=base["materials"], camera=base["camera"], name=f"room-{len(tris)}tri")


def uneven_scene_mix(count=64, lo=1e3, hi=2e6, seed=MIX_SEED):
    """Triangle counts (log-uniform in [lo, hi]) and per-job draws for `count` scenes:
    returns [(triangle_count, scene_seed, (width, height), samples)]."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)
    res = rng.integers(0, len(MIX_RESOLUTIONS), size=count)
    spp = rng.integers(0, len(MIX_SAMPLES), size=count)
    return [(int(counts[i]), int(seed + 17 * (i + 1)), MIX_RESOLUTIONS[res[i]], MIX_SAMPLES[spp[i]]) for i in range(count)]


def request_stream(count=2000, rate=40.0, scenes=64, seed=MIX_SEED + 1):
    """A Poisson request stream over the mix: [(arrival seconds, scene index, (w, h), samples)]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    sc = rng.integers(0, scenes, size=count)
    res = rng.integers(0, len(MIX_RESOLUTIONS), size=count)
    spp = rng.integers(0, len(MIX_SAMPLES), size=count)
    return [(float(t[i]), int(sc[i]), MIX_RESOLUTIONS[res[i]], MIX_SAMPLES[spp[i]]) for i in range(count)]
