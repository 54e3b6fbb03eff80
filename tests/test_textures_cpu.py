"""Textures, modifiers and composite materials on the CPU: the oracle's noise
against the reference's own noise known-answer tests, and the compiled
records against the layouts of scene/compiler/CompiledTextureCache.java,
CompiledModifierCache.java and CompiledMaterialCache.java."""
import math

import numpy as np
import pytest

from dayflower_b200.scene import generators as G
from dayflower_b200.scene import model as M
from dayflower_b200.scene.compiler import compile_scene
from oracle import dfo


def _unpack16(f):
    v = int(f)
    return (v >> 16) & 0xFFFF, v & 0xFFFF


def test_noise_known_answers():
    L = dfo.lib()
    # PerlinNoiseFUnitTests.java:88-92, SimplexNoiseFUnitTests.java:234-238: zero at lattice points and for NaN
    assert L.dfo_perlin(1.0, 2.0, 3.0) == 0.0
    assert L.dfo_simplex(1.0, 2.0, 3.0) == 0.0
    for args in ((math.nan, 0.0, 0.0), (0.0, math.nan, 0.0), (0.0, 0.0, math.nan)):
        assert L.dfo_perlin(*args) == 0.0
        assert L.dfo_simplex(*args) == 0.0


def test_noise_ranges_and_variation():
    L = dfo.lib()
    rng = np.random.default_rng(3)
    pts = rng.uniform(-50.0, 50.0, size=(2000, 3))
    p = np.array([L.dfo_perlin(*q) for q in pts])
    s = np.array([L.dfo_simplex(*q) for q in pts])
    # PerlinNoiseFUnitTests.java:85, SimplexNoiseFUnitTests.java:231: within [-1, 1]
    assert np.all(np.abs(p) <= 1.0) and np.all(np.abs(s) <= 1.0)
    assert p.std() > 0.1 and s.std() > 0.1  # not constant
    # turbulenceXYZ(x, y, z, octaves) sums |noise| / 2^i: within [0, 2) (PerlinNoiseFUnitTests.java:126)
    t = np.array([L.dfo_perlin_turbulence(*q, 8) for q in pts[:300]])
    assert np.all(t >= 0.0) and np.all(t <= 2.0)
    # fractionalBrownianMotionXYZ maps into [minimum, maximum] (SimplexNoiseFUnitTests.java:167)
    f = np.array([L.dfo_simplex_fbm(*q, 1.5, 0.5, -0.25, 0.25, 16) for q in pts[:300]])
    assert np.all(f >= -0.25) and np.all(f <= 0.25)
    # continuity: a tiny step changes the noise a little
    q = pts[0]
    assert abs(L.dfo_perlin(*q) - L.dfo_perlin(q[0] + 1e-3, q[1], q[2])) < 0.02


def test_texture_records():
    img = G.ldr_image(4, 2, seed=1)
    a = M.CheckerboardTexture(a=(1, 0, 0), b=(0, 0, 1), angle_deg=30.0, scale=(8.0, 4.0))
    tex = M.BlendTexture(a=a, b=M.LDRImageTexture(resolution_x=4, resolution_y=2, image=img, scale=(2.0, 1.0)), t=(0.25, 0.5, 0.75))
    sc = M.Scene(camera=M.Camera((0, 0, 5), (0, 0, 0), resolution=(8, 8)))
    sc.add(M.Primitive(M.Sphere(), M.Matte(kd=tex, emission=M.UVTexture())))
    arr = compile_scene(sc).arrays
    # the Matte record: slot 0 (emission texture, modifier), slot 1 (angle, KD), 8-bit packed (Ints.java:258)
    rec = arr["materialMatteMaterialArray"].view(np.uint32)
    e_id, e_off, m_id, m_off = rec[0] & 0xFF, (rec[0] >> 8) & 0xFF, (rec[0] >> 16) & 0xFF, rec[0] >> 24
    assert (e_id, e_off, m_id, m_off) == (M.TEX_UV, 0, M.MOD_NOOP, 0)
    kd_id, kd_off = (rec[1] >> 16) & 0xFF, rec[1] >> 24
    assert kd_id == M.TEX_BLEND
    blend = arr["textureBlendTextureArray"].reshape(-1, 8)[kd_off]
    assert _unpack16(blend[0])[0] == M.TEX_CHECKERBOARD and _unpack16(blend[1]) == (M.TEX_LDR_IMAGE, 0)
    assert list(blend[2:5]) == [0.25, 0.5, 0.75]
    chk = arr["textureCheckerboardTextureArray"].reshape(-1, 8)[_unpack16(blend[0])[1]]
    assert chk[0] == 30.0 and abs(chk[1] - math.radians(30.0)) < 1e-7 and list(chk[4:6]) == [8.0, 4.0]
    assert _unpack16(chk[2])[0] == M.TEX_CONSTANT and _unpack16(chk[3])[0] == M.TEX_CONSTANT
    c = arr["textureConstantTextureArray"].reshape(-1, 4)
    assert list(c[_unpack16(chk[2])[1], :3]) == [1, 0, 0] and list(c[_unpack16(chk[3])[1], :3]) == [0, 0, 1]
    # LDRImageTexture: angle, scale, resolution, pixels, padded to a multiple of 8; relative offset via the offset array
    off = arr["textureLDRImageTextureOffsetArray"]
    ldr = arr["textureLDRImageTextureArray"]
    assert list(off) == [0] and ldr.size == 16 and list(ldr[1:5]) == [2.0, 1.0, 4.0, 2.0]
    assert np.array_equal(ldr[5:13].astype(np.int64).astype(np.int32).view(np.uint32), img)


def test_modifier_and_composite_records():
    nm = M.NormalMapLDRImageModifier(resolution_x=2, resolution_y=2, image=G.normal_map_image(2, 2, seed=1))
    inner_a = M.Matte(kd=(0.5, 0.5, 0.5), modifier=nm)
    inner_b = M.Plastic(modifier=M.SimplexNoiseNormalMapModifier(frequency=8.0, scale=0.5))
    outer = M.CheckerboardMaterial(a=M.PolkaDotMaterial(a=inner_a, b=inner_b, cell_resolution=3.0, radius=0.2), b=inner_a,
                                   angle_deg=45.0, scale=(2.0, 3.0))
    sc = M.Scene(camera=M.Camera((0, 0, 5), (0, 0, 0), resolution=(8, 8)))
    sc.add(M.Primitive(M.Sphere(), outer))
    for lv in (1, 2):
        arr = compile_scene(sc, layout_version=lv).arrays
        prim = arr["primitiveArray"]
        assert prim[4] == M.MAT_CHECKERBOARD
        assert arr["materialCheckerboardMaterialArray"].dtype == np.float32  # composite records are float arrays
        chk = arr["materialCheckerboardMaterialArray"][prim[5]:prim[5] + 8]
        assert chk[0] == 45.0 and list(chk[4:6]) == [2.0, 3.0]
        a_id, a_off = _unpack16(chk[2])
        b_id, b_off = _unpack16(chk[3])
        assert (a_id, b_id) == (M.MAT_POLKA_DOT, M.MAT_MATTE)
        pd = arr["materialPolkaDotMaterialArray"][a_off:a_off + 8]
        assert list(pd[4:6]) == [3.0, np.float32(0.2)]
        assert _unpack16(pd[2]) == (M.MAT_MATTE, b_off) and _unpack16(pd[3])[0] == M.MAT_PLASTIC
        # modifiers: slot 0 texture B of the record, relative offsets
        matte = arr["materialMatteMaterialArray"]
        mid, moff = (int(matte[b_off + 2]), int(matte[b_off + 3])) if lv == 2 else \
            ((int(matte.view(np.uint32)[b_off]) >> 16) & 0xFF, int(matte.view(np.uint32)[b_off]) >> 24)
        assert (mid, moff) == (M.MOD_NORMAL_MAP_LDR_IMAGE, 0)
        assert list(arr["modifierNormalMapLDRImageModifierOffsetArray"]) == [0]
        assert list(arr["modifierSimplexNoiseNormalMapModifierArray"]) == [8.0, 0.5]


def test_packed_colours_and_layout_limit():
    sc = M.Scene(camera=M.Camera((0, 0, 5), (0, 0, 0), resolution=(8, 8)))
    sc.add(M.Primitive(M.Sphere(), M.Matte(kd=M.MarbleTexture(color_a=(1.0, 0.5, 0.0)))))
    arr = compile_scene(sc).arrays
    argb = int(arr["textureMarbleTextureArray"][0]) & 0xFFFFFFFF  # Color3F.pack(): ARGB, alpha 255
    assert argb == (255 << 24) | (255 << 16) | (128 << 8) | 0
    # layout 1 packs texture offsets in 8 bits
    sc = M.Scene(camera=M.Camera((0, 0, 5), (0, 0, 0), resolution=(8, 8)))
    for k in range(300):
        sc.add(M.Primitive(M.Sphere(), M.Matte(kd=(k / 300.0, 0.5, 0.5)), M.Transform.translate_scale((k, 0, 0), 0.4)))
    with pytest.raises(ValueError):
        compile_scene(sc, layout_version=1)
    compile_scene(sc, layout_version=2)


def test_textures_scene_compiles_and_oracle_renders():
    from dayflower_b200 import RenderingAlgorithm as RA
    cs = compile_scene(G.textures_scene(resolution=(48, 27)))
    o = dfo.OracleScene(cs).render(RA.PATH_TRACING, spp=2, max_bounce=3, threads=4)
    img = o["sum"] / np.maximum(o["count"], 1)[..., None]
    assert np.all(np.isfinite(img)) and img.mean() > 0.02
