"""Seeded synthetic scenes for the benchmark configurations and the tests.

No public scene, dataset or benchmark suite is read: every scene is generated
from a fixed seed with the shapes and sizes its configuration names.

* :func:`cornell_box` - five 100-unit walls (Rectangle3F), a glass and a
  mirror sphere of radius 16.5, and a 30x30 light of radiance 12 under the
  ceiling.  The light is two Triangle3F with DiffuseAreaLights, because the
  CPU renderer can only sample area lights on spheres and triangles
  (geometry/Shape3F.java:104-108).
* :func:`terrain_spheres` - a fractal value-noise heightfield (8 octaves,
  amplitude 0.15 of the extent) with 2*n*n triangles, log-uniform spheres with
  matte/plastic/metal/glass materials (roughness U(0.05, 0.6)), lit by a Perez
  sun and sky.
"""
from __future__ import annotations

import math

import numpy as np

from . import model as M


def cornell_box(resolution=(512, 512), light_radiance=12.0) -> M.Scene:
    cam = M.Camera(eye=(50.0, 50.0, 220.0), look_at=(50.0, 50.0, 0.0), fov_x_deg=40.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="cornell")
    grey = M.Matte(kd=(0.75, 0.75, 0.75))
    red = M.Matte(kd=(0.75, 0.25, 0.25))
    green = M.Matte(kd=(0.25, 0.75, 0.25))
    walls = [
        (M.Rectangle((0, 0, 0), (0, 0, 100), (100, 0, 100)), grey),        # floor, normal +y
        (M.Rectangle((0, 100, 0), (100, 100, 0), (100, 100, 100)), grey),  # ceiling, normal -y
        (M.Rectangle((0, 0, 0), (100, 0, 0), (100, 100, 0)), grey),        # back, normal +z
        (M.Rectangle((0, 0, 0), (0, 100, 0), (0, 100, 100)), red),         # left, normal +x
        (M.Rectangle((100, 0, 0), (100, 0, 100), (100, 100, 100)), green),  # right, normal -x
    ]
    for shape, mat in walls:
        sc.add(M.Primitive(shape, mat))
    sc.add(M.Primitive(M.Sphere(), M.Glass(eta=1.5), M.Transform.translate_scale((30.0, 16.5, 45.0), 16.5)))
    sc.add(M.Primitive(M.Sphere(), M.Mirror(kr=(0.999, 0.999, 0.999)), M.Transform.translate_scale((72.0, 16.5, 70.0), 16.5)))
    black = M.Matte(kd=(0.0, 0.0, 0.0))
    y = 99.0
    tris = [M.Triangle((35, y, 35), (65, y, 35), (65, y, 65)), M.Triangle((35, y, 35), (65, y, 65), (35, y, 65))]
    for t in tris:
        light = M.DiffuseAreaLight(t, (light_radiance,) * 3)
        sc.lights.append(light)
        sc.add(M.Primitive(t, black, area_light=light))
    return sc


def _value_noise(xs: np.ndarray, zs: np.ndarray, octaves: int, rng: np.random.Generator) -> np.ndarray:
    """Fractal value noise on [0,1)^2, amplitude halving per octave, range about [-1, 1]."""
    out = np.zeros((zs.size, xs.size), dtype=np.float64)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        f = 4 * (2 ** o)
        lattice = rng.uniform(-1.0, 1.0, size=(f + 2, f + 2))
        gx, gz = xs * f, zs * f
        ix, iz = np.floor(gx).astype(np.int64), np.floor(gz).astype(np.int64)
        fx, fz = gx - ix, gz - iz
        sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
        a = lattice[np.ix_(iz, ix)]
        b = lattice[np.ix_(iz, ix + 1)]
        c = lattice[np.ix_(iz + 1, ix)]
        d = lattice[np.ix_(iz + 1, ix + 1)]
        top = a + (b - a) * sx[None, :]
        bot = c + (d - c) * sx[None, :]
        out += amp * (top + (bot - top) * sz[:, None])
        total += amp
        amp *= 0.5
    return out / total


def heightfield_mesh(cells: int, extent: float, seed: int, octaves: int = 8, amplitude_fraction: float = 0.15):
    """Returns (TriangleMesh, height function data) for a cells x cells grid centred at the origin (y up)."""
    rng = np.random.default_rng(seed)
    n = cells + 1
    t = np.linspace(0.0, 1.0, n, endpoint=False) + 0.5 / n
    h = _value_noise(t, t, octaves, rng) * (amplitude_fraction * extent)
    xs = np.linspace(-extent / 2, extent / 2, n)
    zs = np.linspace(-extent / 2, extent / 2, n)
    X, Z = np.meshgrid(xs, zs)
    P = np.stack([X, h, Z], axis=-1).reshape(-1, 3)
    # smooth vertex normals from central differences
    dhdx = np.gradient(h, xs, axis=1)
    dhdz = np.gradient(h, zs, axis=0)
    N = np.stack([-dhdx, np.ones_like(h), -dhdz], axis=-1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    N = N.reshape(-1, 3)
    U, V = np.meshgrid(np.linspace(0, 1, n), np.linspace(0, 1, n))
    UV = np.stack([U, V], axis=-1).reshape(-1, 2)
    i = np.arange(cells)
    I, J = np.meshgrid(i, i)  # J rows (z), I cols (x)
    v00 = (J * n + I).reshape(-1)
    v10 = v00 + 1
    v01 = v00 + n
    v11 = v01 + 1
    # counter-clockwise seen from +y so that the geometric normal points up
    idx = np.concatenate([np.stack([v00, v01, v10], 1), np.stack([v10, v01, v11], 1)], axis=0)
    mesh = M.TriangleMesh.from_positions(P.astype(np.float32), idx, uvs=UV.astype(np.float32), normals=N.astype(np.float32))
    return mesh, (xs, zs, h)


def _height_at(hf, x, z):
    xs, zs, h = hf
    fx = np.interp(x, xs, np.arange(xs.size))
    fz = np.interp(z, zs, np.arange(zs.size))
    ix, iz = np.clip(np.floor(fx).astype(int), 0, xs.size - 2), np.clip(np.floor(fz).astype(int), 0, zs.size - 2)
    tx, tz = fx - ix, fz - iz
    a, b, c, d = h[iz, ix], h[iz, ix + 1], h[iz + 1, ix], h[iz + 1, ix + 1]
    return (a * (1 - tx) + b * tx) * (1 - tz) + (c * (1 - tx) + d * tx) * tz


def terrain_spheres(cells=1024, n_spheres=2000, resolution=(1920, 1080), seed=2, extent=100.0, turbidity=2.5,
                    sun_elevation_deg=35.0, sun_azimuth_deg=40.0, kinds=(0, 1, 2, 3)) -> M.Scene:
    """kinds: allowed sphere materials, 0 matte, 1 plastic, 2 metal, 3 glass, 4 Disney (base colour, metallic
    and roughness uniform), drawn uniformly."""
    mesh, hf = heightfield_mesh(cells, extent, seed)
    rng = np.random.default_rng(seed + 1000)
    cam = M.Camera(eye=(0.0, 0.30 * extent, 0.62 * extent), look_at=(0.0, 0.0, -0.05 * extent), fov_x_deg=55.0,
                   resolution=resolution)
    sc = M.Scene(camera=cam, name="terrain_spheres")
    sc.add(M.Primitive(mesh, M.Matte(kd=(0.45, 0.42, 0.35))))
    radii = np.exp(rng.uniform(math.log(0.1), math.log(2.0), size=n_spheres))
    xs = rng.uniform(-0.45 * extent, 0.45 * extent, size=n_spheres)
    zs = rng.uniform(-0.45 * extent, 0.45 * extent, size=n_spheres)
    ys = _height_at(hf, xs, zs) + radii * 0.8
    kinds = np.asarray(kinds)[rng.integers(0, len(kinds), size=n_spheres)]
    for k in range(n_spheres):
        col = tuple(float(c) for c in rng.uniform(0.1, 0.9, size=3))
        rough = float(rng.uniform(0.05, 0.6))
        if kinds[k] == 0:
            mat = M.Matte(kd=col)
        elif kinds[k] == 1:
            mat = M.Plastic(kd=col, ks=(0.5, 0.5, 0.5), roughness=rough)
        elif kinds[k] == 2:
            mat = M.Metal(roughness_u=rough, roughness_v=rough)
        elif kinds[k] == 3:
            mat = M.Glass(eta=1.5, roughness_u=rough, roughness_v=rough)
        else:
            mat = M.Disney(color=col, metallic=float(rng.uniform(0.0, 1.0)), roughness=rough)
        sc.add(M.Primitive(M.Sphere(), mat, M.Transform.translate_scale((xs[k], ys[k], zs[k]), radii[k])))
    el, az = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sun = (math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az))
    sc.lights.append(M.PerezLight(turbidity=turbidity, sun_direction_world=sun))
    return sc


def small_mixed_scene(resolution=(96, 64), seed=7, cells=24, n_spheres=24, with_lights=True) -> M.Scene:
    """A small scene that exercises every supported shape, material and light type."""
    sc = terrain_spheres(cells=cells, n_spheres=n_spheres, resolution=resolution, seed=seed, extent=20.0)
    rng = np.random.default_rng(seed + 5)
    sc.add(M.Primitive(M.Rectangle((-6, 0.5, -6), (-6, 4.5, -6), (-2, 4.5, -6)), M.Matte(kd=(0.6, 0.6, 0.2), angle=20.0)))
    sc.add(M.Primitive(M.Triangle((2, 1, -5), (6, 1, -5), (4, 5, -5)), M.Mirror(kr=(0.9, 0.9, 0.9))))
    sc.add(M.Primitive(M.Plane(), M.Matte(kd=(0.3, 0.3, 0.3)), M.Transform.from_matrix(
        np.array([[1, 0, 0, 0], [0, 0, 1, -3.0], [0, -1, 0, 0], [0, 0, 0, 1]], dtype=np.float64))))
    sc.add(M.Primitive(M.Sphere(), M.Glass(eta=1.5), M.Transform.translate_scale((0.0, 3.0, 0.0), 1.5)))
    if with_lights:
        sc.lights.append(M.PointLight((3.0, 8.0, 4.0), (60.0, 60.0, 60.0)))
        sc.lights.append(M.SpotLight((-4.0, 9.0, 3.0), (0.0, 0.0, 0.0), (80.0, 70.0, 60.0), 25.0, 5.0))
        sc.lights.append(M.DirectionalLight((0.3, 1.0, 0.2), (0.8, 0.8, 0.8)))
        tri = M.Triangle((-2, 7, -2), (2, 7, -2), (2, 7, 2))
        al = M.DiffuseAreaLight(tri, (6.0, 6.0, 6.0))
        sc.lights.append(al)
        sc.add(M.Primitive(tri, M.Matte(kd=(0.0, 0.0, 0.0)), area_light=al))
        sl = M.DiffuseAreaLight(M.Sphere(), (4.0, 3.0, 2.0), transform=M.Transform.translate_scale((5.0, 6.0, 1.0), 0.7))
        sc.lights.append(sl)
        sc.add(M.Primitive(sl.shape, M.Matte(kd=(0.0, 0.0, 0.0)), M.Transform.translate_scale((5.0, 6.0, 1.0), 0.7), area_light=sl))
    del rng
    return sc


def disney_scene(resolution=(96, 72), with_lights=True) -> M.Scene:
    """Spheres of DisneyMaterial covering every lobe combination the material
    builds (DisneyMaterial.java:1121-1210): diffuse + retro, sheen, metallic and
    anisotropic specular, clear coat, rough transmission, the scatter-distance
    specular transmission, and thin sheets with flatness and diffuse
    transmission; on a matte ground plane, lit by a point light, a spherical
    area light and a triangle area light."""
    cam = M.Camera(eye=(0.0, 3.0, 10.0), look_at=(0.0, 1.0, 0.0), fov_x_deg=60.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="disney")
    mats = [
        M.Disney(color=(0.8, 0.3, 0.2), roughness=0.5),
        M.Disney(color=(0.2, 0.6, 0.8), roughness=0.3, sheen=1.0, sheen_tint=0.7),
        M.Disney(color=(0.9, 0.7, 0.3), metallic=1.0, roughness=0.25, anisotropic=0.6),
        M.Disney(color=(0.3, 0.8, 0.3), roughness=0.4, clear_coat=1.0, clear_coat_gloss=0.8, specular_tint=0.5),
        M.Disney(color=(0.9, 0.9, 0.9), roughness=0.2, specular_transmission=0.9, eta=1.5),
        M.Disney(color=(0.7, 0.5, 0.9), roughness=0.4, scatter_distance=(0.5, 0.5, 0.5)),
        M.Disney(color=(0.6, 0.8, 0.4), roughness=0.6, thin=True, flatness=0.5, diffuse_transmission=0.8, sheen=0.5),
        M.Disney(color=(0.8, 0.8, 0.6), roughness=0.3, thin=True, specular_transmission=0.5, metallic=0.2, clear_coat=0.5),
    ]
    for k, m in enumerate(mats):
        x = -5.25 + 1.5 * k
        sc.add(M.Primitive(M.Sphere(), m, M.Transform.translate_scale((x, 0.7, 0.0), 0.7)))
    sc.add(M.Primitive(M.Plane(), M.Matte(kd=(0.5, 0.5, 0.5)), _rot_x(-90.0, (0.0, 0.0, 0.0))))
    if with_lights:
        sc.lights.append(M.PointLight((2.0, 6.0, 5.0), (40.0, 40.0, 40.0)))
        sl = M.DiffuseAreaLight(M.Sphere(), (6.0, 5.0, 4.0), transform=M.Transform.translate_scale((-3.0, 5.0, 3.0), 0.6))
        sc.lights.append(sl)
        sc.add(M.Primitive(sl.shape, M.Matte(kd=(0.0, 0.0, 0.0)), M.Transform.translate_scale((-3.0, 5.0, 3.0), 0.6), area_light=sl))
        tri = M.Triangle((3, 5, -2), (5, 5, -2), (4, 6, 1))
        al = M.DiffuseAreaLight(tri, (5.0, 5.0, 5.0))
        sc.lights.append(al)
        sc.add(M.Primitive(tri, M.Matte(kd=(0.0, 0.0, 0.0)), area_light=al))
    return sc


def materials_scene(resolution=(96, 72), with_lights=True) -> M.Scene:
    """Spheres of ClearCoatMaterial, GlossyMaterial, SubstrateMaterial,
    TranslucentMaterial (reflection and transmission) and UberMaterial (opaque;
    partly transparent with specular reflection and transmission) on a matte
    ground plane, lit by a point light and a spherical area light."""
    cam = M.Camera(eye=(0.0, 3.0, 10.0), look_at=(0.0, 1.0, 0.0), fov_x_deg=60.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="materials")
    mats = [
        M.ClearCoat(kd=(0.6, 0.2, 0.2), ks=(1.0, 1.0, 1.0)),
        M.Glossy(kr=(0.8, 0.6, 0.3), roughness=0.15),
        M.Substrate(kd=(0.2, 0.5, 0.7), ks=(0.4, 0.4, 0.4), roughness_u=0.2, roughness_v=0.1),
        M.Translucent(kd=(0.6, 0.7, 0.3), ks=(0.3, 0.3, 0.3), roughness=0.2),
        M.Uber(kd=(0.5, 0.3, 0.6), ks=(0.3, 0.3, 0.3)),
        M.Uber(kd=(0.2, 0.2, 0.2), kr=(0.5, 0.5, 0.5), kt=(0.6, 0.6, 0.6), opacity=(0.6, 0.7, 0.8), eta=1.4),
        M.Translucent(kd=(0.8, 0.4, 0.2), ks=(0.0, 0.0, 0.0), reflectance=(0.0, 0.0, 0.0), transmittance=(0.9, 0.9, 0.9)),
    ]
    for k, m in enumerate(mats):
        x = -4.5 + 1.5 * k
        sc.add(M.Primitive(M.Sphere(), m, M.Transform.translate_scale((x, 0.7, 0.0), 0.7)))
    sc.add(M.Primitive(M.Plane(), M.Matte(kd=(0.5, 0.5, 0.5)), _rot_x(-90.0, (0.0, 0.0, 0.0))))
    if with_lights:
        sc.lights.append(M.PointLight((2.0, 6.0, 5.0), (40.0, 40.0, 40.0)))
        sl = M.DiffuseAreaLight(M.Sphere(), (6.0, 5.0, 4.0), transform=M.Transform.translate_scale((-3.0, 5.0, 3.0), 0.6))
        sc.lights.append(sl)
        sc.add(M.Primitive(sl.shape, M.Matte(kd=(0.0, 0.0, 0.0)), M.Transform.translate_scale((-3.0, 5.0, 3.0), 0.6), area_light=sl))
    return sc


def environment_image(width=4096, height=2048, seed=5, sun_direction_world=(0.4, 0.6, -0.7), sun_radiance=5.0e4,
                      sun_diameter_deg=0.5) -> np.ndarray:
    """A seeded HDR environment for ImageLight, (height, width, 3) float32 in
    the light's spherical texture layout (row y is theta = pi (y + 0.5) /
    height, column x is phi = 2 pi (x + 0.5) / width, object space): a
    low-frequency value-noise sky (blue-ish, brighter towards the zenith) and a
    sun disk of the given angular diameter and radiance.  Pixels whose centre
    lies inside the disk are set to the sun radiance; the nearest pixel always
    is, so the sun survives at low resolutions."""
    from .perez import SKY_WORLD_TO_OBJECT
    rng = np.random.default_rng(seed)
    xs = (np.arange(width) + 0.5) / width
    ys = (np.arange(height) + 0.5) / height
    noise = _value_noise(xs, ys, 3, rng)  # (height, width), about [-1, 1]
    theta = np.pi * ys[:, None]
    phi = 2.0 * np.pi * xs[None, :]
    up = np.cos(theta) * np.ones_like(phi)  # object z; the sky transform maps object z to world y
    base = np.stack([0.35 + 0.15 * noise, 0.45 + 0.15 * noise, 0.75 + 0.2 * noise], axis=-1)
    img = base * (0.6 + 0.4 * np.clip(up, 0.0, 1.0))[..., None]
    img = np.maximum(img, 0.02)
    sw = np.asarray(sun_direction_world, dtype=np.float64)
    so = SKY_WORLD_TO_OBJECT[:3, :3].astype(np.float64) @ (sw / np.linalg.norm(sw))
    so /= np.linalg.norm(so)
    d = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi)], axis=-1)
    cosang = d @ so
    disk = cosang >= math.cos(math.radians(sun_diameter_deg / 2.0))
    sp = math.atan2(so[1], so[0]) % (2.0 * math.pi)
    st = math.acos(max(-1.0, min(1.0, so[2])))
    disk[min(int(st / np.pi * height), height - 1), min(int(sp / (2.0 * np.pi) * width), width - 1)] = True
    img[disk] = sun_radiance
    return img.astype(np.float32)


def image_light_scene(resolution=(96, 72), env=(256, 128), seed=9) -> M.Scene:
    """Spheres (matte, metal, glass, Disney) on a matte ground under an ImageLight
    of a seeded environment with a small sun."""
    cam = M.Camera(eye=(0.0, 2.5, 8.0), look_at=(0.0, 0.8, 0.0), fov_x_deg=60.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="image_light")
    mats = [M.Matte(kd=(0.7, 0.6, 0.5)), M.Metal(roughness_u=0.2, roughness_v=0.2), M.Glass(eta=1.5),
            M.Disney(color=(0.3, 0.6, 0.8), roughness=0.4, clear_coat=0.5)]
    for k, m in enumerate(mats):
        sc.add(M.Primitive(M.Sphere(), m, M.Transform.translate_scale((-3.0 + 2.0 * k, 0.8, 0.0), 0.8)))
    sc.add(M.Primitive(M.Plane(), M.Matte(kd=(0.5, 0.5, 0.5)), _rot_x(-90.0, (0.0, 0.0, 0.0))))
    img = environment_image(env[0], env[1], seed=seed, sun_radiance=200.0, sun_diameter_deg=4.0)
    sc.lights.append(M.ImageLight(img, angle_deg=30.0))
    return sc


def blob_mesh(subdivisions: int = 4, seed: int = 21, amplitude: float = 0.3):
    """A seeded blob: an icosphere of 20 * 4^subdivisions triangles (5,120 for
    4) with its vertices pushed along their directions by smooth noise."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.asarray(x, dtype=np.float64) / np.linalg.norm(x) for x in verts]
    f = list(faces)
    for _ in range(subdivisions):
        cache, nf = {}, []

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[k] = len(v) - 1
            return cache[k]
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    V = np.array(v)
    rng = np.random.default_rng(seed)
    k = rng.normal(size=(6, 3))
    ph = rng.uniform(0, 2 * np.pi, size=6)
    disp = sum(np.sin(V @ k[i] * (1.5 + 0.5 * i) + ph[i]) / (1.0 + i) for i in range(6))
    P = V * (1.0 + amplitude * disp / np.abs(disp).max())[:, None]
    return M.TriangleMesh.from_positions(P.astype(np.float32), np.array(f, dtype=np.int64))


def large_scene(cells=2236, instances=50000, blob_subdivisions=4, resolution=(3840, 2160), env=(4096, 2048), seed=4,
                extent=400.0) -> M.Scene:
    """The large single scene: a fractal heightfield of 2 * cells^2 triangles
    (2236 -> 9,999,392), `instances` instanced copies of one seeded blob mesh
    (5,120 triangles) standing on it with random scale and rotation, every
    copy with its own DisneyMaterial (base colour, metallic and roughness
    uniform), lit by an ImageLight of a seeded env[0] x env[1] HDR
    environment with a 0.5 degree sun disk of radiance 5e4."""
    terrain, hf = heightfield_mesh(cells, extent, seed)
    blob = blob_mesh(blob_subdivisions, seed=seed + 1)
    cam = M.Camera(eye=(0.0, 0.12 * extent, 0.45 * extent), look_at=(0.0, 0.0, 0.0), fov_x_deg=60.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="large")
    rng = np.random.default_rng(seed + 2)
    sc.add(M.Primitive(terrain, M.Disney(color=(0.45, 0.42, 0.35), roughness=0.7)))
    xs = rng.uniform(-0.45 * extent, 0.45 * extent, size=instances)
    zs = rng.uniform(-0.45 * extent, 0.45 * extent, size=instances)
    scale = rng.uniform(0.5, 2.0, size=instances)
    ys = _height_at(hf, xs, zs) + 0.6 * scale
    ang = rng.uniform(0.0, 2.0 * np.pi, size=instances)
    cols = rng.uniform(0.05, 0.95, size=(instances, 3))
    met = rng.uniform(0.0, 1.0, size=instances)
    rough = rng.uniform(0.05, 0.95, size=instances)
    for k in range(instances):
        c, s_ = math.cos(ang[k]), math.sin(ang[k])
        m = np.eye(4)
        m[:3, :3] = np.array([[c, 0, s_], [0, 1, 0], [-s_, 0, c]]) * scale[k]
        m[:3, 3] = (xs[k], ys[k], zs[k])
        mat = M.Disney(color=tuple(float(x) for x in cols[k]), metallic=float(met[k]), roughness=float(rough[k]))
        sc.add(M.Primitive(blob, mat, M.Transform.from_matrix(m)))
    sc.lights.append(M.ImageLight(environment_image(env[0], env[1], seed=seed + 3)))
    return sc


def _rot_x(deg, position, scale=1.0):
    """Object-to-world: rotate about x by `deg`, scale, then translate."""
    c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
    m = np.eye(4)
    m[:3, :3] = np.array([[1, 0, 0], [0, c, -s], [0, s, c]]) * float(scale)
    m[:3, 3] = position
    return M.Transform.from_matrix(m)


def quadrics_scene(resolution=(128, 96), with_lights=True) -> M.Scene:
    """Disk, cylinder, cone, paraboloid, hyperboloid, rectangular cuboid, torus
    (full and partial sweeps) and polygons standing on a ground plane, z-up objects turned
    upright, lit by a point light, a directional light and a spherical area light."""
    cam = M.Camera(eye=(0.0, 3.8, 9.0), look_at=(0.0, 1.0, 0.0), fov_x_deg=70.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="quadrics")
    up = -90.0  # object z -> world y
    shapes = [
        (M.Disk(300.0, 0.4, 1.2, 0.0), M.Matte(kd=(0.7, 0.3, 0.3)), _rot_x(up, (-6.0, 0.01, 2.0))),
        (M.Cylinder(360.0, 0.8, 2.0, 0.0), M.Plastic(kd=(0.2, 0.5, 0.7), ks=(0.3, 0.3, 0.3), roughness=0.2), _rot_x(up, (-3.0, 0.0, 0.0))),
        (M.Cylinder(270.0, 0.6, 1.5, 0.0), M.Metal(roughness_u=0.3, roughness_v=0.3), _rot_x(up, (-6.0, 0.0, -3.0))),
        (M.Cone(360.0, 1.0, 2.5), M.Matte(kd=(0.8, 0.7, 0.2)), _rot_x(up, (0.0, 0.0, -2.0))),
        (M.Paraboloid(360.0, 1.0, 2.0, 0.0), M.Matte(kd=(0.3, 0.8, 0.4)), _rot_x(up, (3.0, 0.0, 0.0))),
        (M.Hyperboloid(360.0, (0.3, 0.3, 0.0), (1.0, 0.2, 2.0)), M.Plastic(kd=(0.6, 0.3, 0.7), ks=(0.2, 0.2, 0.2), roughness=0.4),
         _rot_x(up, (6.0, 0.0, -2.0))),
        (M.RectangularCuboid((-0.7, -0.7, 0.0), (0.7, 0.7, 1.4)), M.Matte(kd=(0.5, 0.5, 0.8)), _rot_x(up, (1.5, 0.0, 3.0))),
        (M.Torus(0.35, 1.0), M.Metal(roughness_u=0.15, roughness_v=0.15), _rot_x(-60.0, (-1.5, 1.4, 3.5))),
        (M.Torus(0.25, 0.8), M.Matte(kd=(0.9, 0.5, 0.1)), _rot_x(0.0, (4.5, 2.2, 3.0))),
        # a concave pentagon and a hexagon standing upright (Polygon3F)
        (M.Polygon([(0, 0, 0), (1.6, 0, 0), (1.6, 1.4, 0), (0.8, 0.6, 0), (0, 1.4, 0)]), M.Matte(kd=(0.3, 0.4, 0.9)),
         M.Transform.from_matrix(np.array([[1, 0, 0, -4.6], [0, 1, 0, 0.0], [0, 0, 1, 3.0], [0, 0, 0, 1]], dtype=np.float64))),
        (M.Polygon([(math.cos(k * math.pi / 3), math.sin(k * math.pi / 3), 0.0) for k in range(6)]), M.Plastic(kd=(0.8, 0.8, 0.3)),
         M.Transform.from_matrix(np.array([[1, 0, 0, 0.0], [0, 1, 0, 4.4], [0, 0, 1, 0.5], [0, 0, 0, 1]], dtype=np.float64))),
    ]
    for shp, mat, tr in shapes:
        sc.add(M.Primitive(shp, mat, tr))
    sc.add(M.Primitive(M.Plane(), M.Matte(kd=(0.6, 0.6, 0.6)), _rot_x(-90.0, (0.0, 0.0, 0.0))))
    if with_lights:
        sc.lights.append(M.PointLight((4.0, 9.0, 6.0), (90.0, 90.0, 90.0)))
        sc.lights.append(M.DirectionalLight((-0.4, 1.0, 0.5), (0.6, 0.6, 0.6)))
        sl = M.DiffuseAreaLight(M.Sphere(), (8.0, 7.0, 6.0), transform=M.Transform.translate_scale((-4.0, 7.0, 4.0), 0.8))
        sc.lights.append(sl)
        sc.add(M.Primitive(sl.shape, M.Matte(kd=(0.0, 0.0, 0.0)), M.Transform.translate_scale((-4.0, 7.0, 4.0), 0.8), area_light=sl))
    return sc


def ldr_image(width: int, height: int, seed: int) -> np.ndarray:
    """A seeded packed-ARGB image (alpha 255): smooth colour gradients plus blocks of noise."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:height, 0:width]
    r = (x * 255 // max(width - 1, 1)).astype(np.uint32)
    g = (y * 255 // max(height - 1, 1)).astype(np.uint32)
    b = rng.integers(0, 256, size=(height, width), dtype=np.uint32)
    return ((np.uint32(255) << 24) | (r << 16) | (g << 8) | b).reshape(-1).astype(np.uint32)


def normal_map_image(width: int, height: int, seed: int) -> np.ndarray:
    """A seeded tangent-space normal map: unit normals tilted up to ~35 degrees, packed ARGB."""
    rng = np.random.default_rng(seed)
    t = rng.normal(0.0, 0.35, size=(height * width, 2))
    n = np.concatenate([t, np.ones((height * width, 1))], axis=1)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    c = np.clip(np.round((n + 1.0) * 0.5 * 255.0), 0, 255).astype(np.uint32)
    return ((np.uint32(255) << 24) | (c[:, 0] << 16) | (c[:, 1] << 8) | c[:, 2]).astype(np.uint32)


def textures_scene(resolution=(128, 72), with_lights=True, point_light_only=False) -> M.Scene:
    """Every texture the compiled scene format carries (checkerboard, polka dot,
    bullseye, marble, simplex fBm, LDR image, blend, surface normal, dot product,
    UV, constant), both shading-normal modifiers, the three composite materials,
    textured float parameters (Disney roughness and metallic, Matte angle) and a
    textured emission, on spheres over a ground plane with a composite material.
    With ``point_light_only`` the first-bounce radiance is the same per sample
    on every renderer that shares the random numbers (no light is sampled)."""
    cam = M.Camera(eye=(0.0, 4.2, 6.8), look_at=(0.0, 0.4, -0.6), fov_x_deg=62.0, resolution=resolution)
    sc = M.Scene(camera=cam, name="textures")
    checker = M.CheckerboardTexture(a=(0.85, 0.2, 0.15), b=(0.15, 0.25, 0.85), angle_deg=30.0, scale=(8.0, 4.0))
    polka = M.PolkaDotTexture(a=(0.9, 0.9, 0.2), b=(0.2, 0.5, 0.3), angle_deg=15.0, cell_resolution=6.0, radius=0.3)
    bull = M.BullseyeTexture(a=(0.8, 0.4, 0.1), b=M.UVTexture(), origin=(0.3, 0.5, 0.2), scale=3.0)  # object space: off-centre rings
    marble = M.MarbleTexture(color_a=(0.8, 0.8, 0.8), color_b=(0.4, 0.2, 0.1), color_c=(0.06, 0.04, 0.02), frequency=2.0, scale=5.0, octaves=4)
    fbm = M.SimplexFBMTexture(color=(0.75, 0.5, 0.75), frequency=1.5, gain=0.5, octaves=4)
    image = M.LDRImageTexture(resolution_x=16, resolution_y=8, image=ldr_image(16, 8, seed=3), angle_deg=10.0, scale=(2.0, 1.0))
    blend = M.BlendTexture(a=checker, b=M.BlendTexture(a=M.UVTexture(), b=marble, t=(0.5, 0.5, 0.5)), t=(0.3, 0.5, 0.7))
    nmap = M.NormalMapLDRImageModifier(resolution_x=8, resolution_y=8, image=normal_map_image(8, 8, seed=4), scale=(4.0, 2.0))
    mats = [
        M.Matte(kd=checker),
        M.Matte(kd=polka, angle=M.CheckerboardTexture(a=(0.0, 0.0, 0.0), b=(30.0, 30.0, 30.0), scale=(4.0, 4.0))),
        M.Matte(kd=bull),
        M.Matte(kd=marble),
        M.Plastic(kd=fbm, ks=(0.3, 0.3, 0.3), roughness=0.2),
        M.Matte(kd=image),
        M.Matte(kd=blend),
        M.Matte(kd=M.SurfaceNormalTexture()),
        M.Matte(kd=M.DotProductTexture()),
        M.Disney(color=marble, roughness=M.CheckerboardTexture(a=(0.2, 0.2, 0.2), b=(0.7, 0.7, 0.7), scale=(6.0, 3.0)),
                 metallic=M.PolkaDotTexture(a=(1.0, 1.0, 1.0), b=(0.0, 0.0, 0.0), cell_resolution=5.0, radius=0.35)),
        M.Matte(kd=(0.7, 0.7, 0.7), modifier=nmap),
        M.Plastic(kd=(0.3, 0.5, 0.8), ks=(0.4, 0.4, 0.4), roughness=0.1, modifier=M.SimplexNoiseNormalMapModifier(frequency=4.0, scale=1.0)),
        M.CheckerboardMaterial(a=M.Matte(kd=(0.9, 0.2, 0.2)), b=M.Glass(), scale=(6.0, 3.0)),
        M.PolkaDotMaterial(a=M.Matte(kd=(0.95, 0.95, 0.95)), b=M.Metal(roughness_u=0.2, roughness_v=0.2), cell_resolution=5.0, radius=0.3),
        M.Matte(kd=(0.2, 0.2, 0.2), emission=M.CheckerboardTexture(a=(2.0, 1.5, 0.5), b=(0.0, 0.0, 0.0), scale=(10.0, 5.0))),
    ]
    for k, m in enumerate(mats):  # three rows of five
        x = -3.4 + 1.7 * (k % 5)
        z = 1.4 - 1.9 * (k // 5)
        sc.add(M.Primitive(M.Sphere(), m, M.Transform.translate_scale((x, 0.7, z), 0.7)))
    ground = M.BullseyeMaterial(a=M.Matte(kd=(0.55, 0.55, 0.55)), b=M.Plastic(kd=(0.3, 0.3, 0.35), ks=(0.3, 0.3, 0.3), roughness=0.3),
                                origin=(0.0, 0.0, 0.0), scale=0.5)
    sc.add(M.Primitive(M.Plane(), ground, _rot_x(-90.0, (0.0, 0.0, 0.0))))
    if with_lights:
        sc.lights.append(M.PointLight((2.0, 8.0, 6.0), (60.0, 60.0, 60.0)))
        if not point_light_only:
            sl = M.DiffuseAreaLight(M.Sphere(), (6.0, 5.0, 4.0), transform=M.Transform.translate_scale((-4.0, 6.0, 4.0), 0.6))
            sc.lights.append(sl)
            sc.add(M.Primitive(sl.shape, M.Matte(kd=(0.0, 0.0, 0.0)), M.Transform.translate_scale((-4.0, 6.0, 4.0), 0.6), area_light=sl))
    return sc


# ---- batched-job mix: eight seeded scenes and a job list over them --------------
# Sphere counts 10 .. 10k and heightfield sizes 10k .. 2M triangles, each spaced
# evenly in log scale over the eight scenes and paired in a shuffled order.
JOB_MIX_SPHERES = [10, 27, 72, 193, 518, 1389, 3728, 10000]
JOB_MIX_CELLS = [71, 103, 151, 220, 321, 468, 684, 1000]  # 2 * cells^2 = 10,082 .. 2,000,000 triangles
JOB_MIX_CELL_ORDER = [3, 7, 0, 5, 1, 6, 2, 4]


def job_mix_scene(index: int, seed: int = 300, resolution=(512, 512), kinds=(0, 1, 2, 3, 4)) -> M.Scene:
    """Scene `index` (0..7) of the batched-job mix: a fractal heightfield and
    log-uniform spheres of random matte/plastic/metal/glass/Disney materials, lit by a
    point light, a spot light and a rectangular area light made of two
    triangles (the CPU renderer samples area lights on triangles and spheres
    only)."""
    extent = 100.0
    cells = JOB_MIX_CELLS[JOB_MIX_CELL_ORDER[index]]
    sc = terrain_spheres(cells=cells, n_spheres=JOB_MIX_SPHERES[index], resolution=resolution, seed=seed + 17 * index,
                         extent=extent, kinds=kinds)
    sc.name = "job_mix_%d" % index
    sc.lights = []
    rng = np.random.default_rng(seed + 31 * index)
    px, pz = rng.uniform(-0.3 * extent, 0.3 * extent, size=2)
    sc.lights.append(M.PointLight((float(px), 0.45 * extent, float(pz)), (4000.0, 3800.0, 3500.0)))
    sx, sz = rng.uniform(-0.3 * extent, 0.3 * extent, size=2)
    sc.lights.append(M.SpotLight((float(sx), 0.5 * extent, float(sz)), (0.0, 0.0, 0.0), (9000.0, 8000.0, 7000.0), 35.0, 8.0))
    y, h = 0.42 * extent, 0.08 * extent
    a, b, c, d = (-h, y, -h), (h, y, -h), (h, y, h), (-h, y, h)
    for tri in (M.Triangle(a, c, b), M.Triangle(a, d, c)):  # facing down
        al = M.DiffuseAreaLight(tri, (25.0, 25.0, 25.0))
        sc.lights.append(al)
        sc.add(M.Primitive(tri, M.Matte(kd=(0.0, 0.0, 0.0)), area_light=al))
    return sc


def job_mix(n_jobs: int = 256, seed: int = 301, n_scenes: int = 8, min_side: int = 64, max_side: int = 1024,
            spp_choices=(1, 4, 16, 64), bounce_choices=(4, 8, 20)):
    """The batched workload: n_jobs jobs with square resolutions log-uniform
    from min_side^2 to max_side^2, spp uniform over spp_choices, maximum bounce
    uniform over bounce_choices, a uniformly drawn scene and a per-job seed.
    Returns a list of dicts with keys scene, width, height, samples,
    maximum_bounce, seed."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_jobs):
        side = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        jobs.append({"scene": int(rng.integers(0, n_scenes)), "width": side, "height": side,
                     "samples": int(spp_choices[rng.integers(0, len(spp_choices))]),
                     "maximum_bounce": int(bounce_choices[rng.integers(0, len(bounce_choices))]),
                     "seed": int(rng.integers(1, 2 ** 31))})
    return jobs
