"""The resolve (resolve.wgsl:1378-1466, its three lanes: sky and opaque
surfaces with shade_hit_legacy_cached, water with water_ctx / water_compose
and the half-resolution water_sec legs or per-pixel legs, glass with its
transmission and reflection; the fog blend with sun shafts, sky_color with
clouds) against the oracle's restatement.

The kernel and the oracle share the float contract of the march but not
the colour arithmetic: the kernel divides, exponentiates and takes logs and
powers at the accuracy WGSL specifies for the engine's shaders (approximate
reciprocal, exp2 and log2 units), the oracle with IEEE division and the
host's libm, so colours are compared within a tolerance: 2e-4 absolute plus
1e-3 relative at 99.9% of the pixels, and 0.05 absolute at every pixel (a
last-bit difference can move a texture-level or a smoothstep edge, or a
water_sec leg across a binary16 rounding step).

CPU: the material builders (atlas format and mips, the engine's face table),
the sun-visibility rounding and oracle properties.  GPU: frames of the small
world with the engine's default look, with probes, the shaft envelope, a
soft-shadow mask, non-uniform light bricks, every resolve override the
kernel reads, and the whole 1920x1080 frame of the 1024x256x1024 terrain."""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle, engine_atlas
from voxelcraft_menu_b200 import look as LK
from voxelcraft_menu_b200 import world as W

ABS, REL, FRAC, WORST = 2e-4, 1e-3, 1e-3, 0.05


def within(got, want, what):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    assert np.array_equal(got[:, 3], want[:, 3]), f"{what}: lane masks differ"
    d = np.abs(got[:, :3] - want[:, :3])
    tol = ABS + REL * np.abs(want[:, :3])
    bad = np.any(d > tol, axis=1)
    assert np.isfinite(got).all(), f"{what}: non-finite colour"
    assert bad.mean() <= FRAC, f"{what}: {bad.sum()} of {len(bad)} pixels outside tolerance (max {d.max():.3g})"
    assert d.max() <= WORST, f"{what}: largest difference {d.max():.3g}"


@pytest.fixture(scope="module")
def small():
    w = W.World.generate(W.recipe_small_terrain())
    return w, w.pools()


def look_camera(width=480, height=270, flags=0, **kw):
    return W.small_terrain_camera(width=width, height=height,
                                  flags=W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | LK.LOOK_FLAGS | flags, **kw)


def look_view(w, cam, seed=1):
    v = w.view(cam)
    LK.apply_defaults(v.frame, seed)
    v.frame.time = 37.5
    return v


# ---------------------------------------------------------------- CPU -----

def test_atlas_layout_and_mips():
    a = LK.atlas(3)
    assert a.size == LK.TEX_COUNT * 340 * 4
    mip0 = a[: LK.TEX_COUNT * 256 * 4].reshape(LK.TEX_COUNT, 16, 16, 4)
    mip1 = a[LK.TEX_COUNT * 256 * 4: LK.TEX_COUNT * 320 * 4].reshape(LK.TEX_COUNT, 8, 8, 4)
    # alpha is the tint mask of grass tops and leaves, 0 for stone and dirt
    assert (mip0[2, :, :, 3] == 255).all() and (mip0[8, :, :, 3] == 255).all()
    assert (mip0[0, :, :, 3] == 0).all() and (mip0[1, :, :, 3] == 0).all()
    # each mip is the 2x2 box average of the one above (alpha linear)
    want = mip0[:, :, :, 3].reshape(LK.TEX_COUNT, 8, 2, 8, 2).astype(np.float64).mean(axis=(2, 4))
    assert np.abs(mip1[:, :, :, 3] - want).max() <= 0.5 + 1e-9
    assert not np.array_equal(LK.atlas(3), LK.atlas(4))


def test_engine_atlas_layout():
    """The oracle's restatement of the engine's atlas: tint masks on grass tops
    and leaves, tuft layers fully transparent or opaque, mips in sequence."""
    a = engine_atlas()
    assert a.size == LK.TEX_COUNT * 340 * 4
    mip0 = a[: LK.TEX_COUNT * 256 * 4].reshape(LK.TEX_COUNT, 16, 16, 4)
    assert (mip0[2, :, :, 3] == 255).all() and (mip0[8, :, :, 3] == 255).all()
    assert (mip0[0, :, :, 3] == 0).all() and (mip0[14, :, :, 3] == 0).all()
    for layer in (19, 25, 26):
        al = mip0[layer, :, :, 3]
        assert set(np.unique(al)) <= {0, 255} and 0.3 < (al > 0).mean() < 0.8
        assert (al[-1] > 0).any() and not (al[0] > 0).all()      # blades grow from the bottom row
    mip3 = a[LK.TEX_COUNT * 336 * 4:].reshape(LK.TEX_COUNT, 2, 2, 4)
    assert 0 < int(mip3[19, :, :, 3].mean()) < 255
    assert not np.array_equal(engine_atlas(), engine_atlas(tint_balance=True))


def test_block_faces_follow_the_engine_table():
    f = LK.block_faces().reshape(26, 8)
    layer, perm = f & 0xFFFF, f >> 16
    # src/block.rs:136-170: grass = column(GRASS_SIDE 3, DIRT 1, GRASS_TOP 2), log = column(6, 7, 7)
    assert layer[3].tolist() == [3, 3, 1, 2, 3, 3, 3, 3]
    assert layer[6].tolist() == [6, 6, 7, 7, 6, 6, 6, 6]
    assert layer[23].tolist() == [24, 24, 1, 20, 24, 24, 24, 24]       # meadow-side
    assert (layer[1] == 0).all() and (layer[13] == 14).all() and (layer[25] == 26).all()
    # perm classes (src/block.rs:74-92): D4 on dirt / grass top / leaves, FLIP_U on grass side
    assert perm[2].tolist() == [2] * 8 and perm[7].tolist() == [2] * 8
    assert perm[3].tolist() == [1, 1, 2, 2, 1, 1, 1, 1]
    assert (perm[1] == 0).all() and (perm[18] == 0).all()


def test_sun_visibility_rounds_to_the_8bit_target():
    sh = np.array([0.0, 3.5, 0.0, 12.0], np.float32)
    assert LK.sun_visibility(sh).tolist() == [1.0, 0.0, 1.0, 0.0]
    m = np.array([0.0, 0.5, 0.999, 1.2, -0.1, 0.00196], np.float32)
    got = LK.sun_visibility(sh[:1].repeat(6), mask=m)
    assert np.array_equal(got * np.float32(255.0), np.round(np.clip(m, 0, 1) * 255.0).astype(np.float32))
    frac = np.array([0.25, 1.0], np.float32)
    assert LK.sun_visibility(frac, soft_rays=True).tolist() == pytest.approx([0.74901962, 0.0])


def test_oracle_resolve_properties(small):
    w, pools = small
    v = look_view(w, look_camera(160, 90))
    o = Oracle(v, *pools)
    vis = o.frame_vis()[0]
    sh = o.shadow(vis)
    sv = LK.sun_visibility(sh)
    atlas, faces = LK.atlas(1), LK.block_faces()
    c = o.resolve(vis, sv, atlas, faces, spec_hi=LK.HI_DEFAULT)
    assert np.isfinite(c).all()
    sky = vis == 0
    assert sky.any() and (~sky).any()
    assert (c[sky, 3] == 1.0).all()
    # water and glass pixels: their lanes' colour (water_compose, shade_glass)
    ids = np.array([o.block_at(int(k >> 24) & 0x1FFF, [(int(k) >> 16) & 63, (int(k) >> 8) & 63, int(k) & 63])
                    if k else 0 for k in vis])
    lane = (~sky) & ((ids == 13) | (ids == 10))
    assert lane.any() and (c[:, 3] == 1.0).all()
    assert (c[lane, :3] > 0.0).all() and (c[ids == 13, 2] > c[ids == 13, 0]).mean() > 0.9   # water is blue
    # the half-resolution legs and per-pixel legs agree where a block is flat water
    own = o.resolve(vis, sv, atlas, faces, spec_hi=LK.HI_DEFAULT & ~LK.HI_WATER_SEC)
    water = ids == 13
    assert np.abs(own[water, :3] - c[water, :3]).mean() < 0.02
    assert np.array_equal(own[~water], c[~water])
    # a part of the range equals the same pixels of the whole frame
    part = o.resolve(vis, sv, atlas, faces, spec_hi=LK.HI_DEFAULT, pix=(3000, 5000))
    assert np.array_equal(part, c[3000:5000])
    # shadowed surfaces are darker than the same frame fully lit
    lit = o.resolve(vis, np.ones_like(sv), atlas, faces, spec_hi=LK.HI_DEFAULT)
    shadowed = (sv == 0.0) & (~lane) & (~sky)
    assert shadowed.any()
    assert (lit[shadowed, :3].sum(1) >= c[shadowed, :3].sum(1)).all()
    assert (lit[shadowed, :3].sum(1) > c[shadowed, :3].sum(1)).mean() > 0.5


def test_oracle_sky_without_clouds_is_sky_base(small):
    """With no clouds, no god rays and no scatter lobe the sky is sky_base's
    gradient and sun disk (common.wgsl:1370-1395), restated here in float64."""
    w, pools = small
    v = look_view(w, look_camera(64, 36, pitch=math.radians(40.0)))
    v.frame.cloud_cover = 0.0
    v.frame.godray_strength = 0.0
    v.frame.fog_scatter = 0.0
    o = Oracle(v, *pools)
    c = o.resolve(np.zeros(o.npix, np.uint64), np.ones(o.npix, np.float32), LK.atlas(1), LK.block_faces())
    day = float(v.frame.daylight)
    hor = np.array([0.0049, 0.0060, 0.0134]) * (1 - day) + np.array([0.4480, 0.6210, 0.8900]) * day
    zen = np.array([0.0008, 0.0015, 0.0039]) * (1 - day) + np.array([0.0637, 0.2140, 0.8276]) * day
    sun = np.array(v.frame.sun_dir, np.float64)

    def smooth(e0, e1, x):
        t = min(max((x - e0) / (e1 - e0), 0.0), 1.0)
        return t * t * (3 - 2 * t)

    for pix in range(0, o.npix, 7):
        rd = o.ray_dir(pix % 64 + 0.5, pix // 64 + 0.5).astype(np.float64)
        up = min(max(rd[1], 0.0), 1.0)
        g = up ** 0.55
        col = hor * (1 - g) + zen * g
        col = col + np.array([1.0, 0.8276, 0.5225]) * smooth(0.9975, 0.9990, float(rd @ sun)) * max(day, 0.2)
        k = smooth(0.0, -0.35, rd[1])
        col = col * (1 - k) + hor * 0.26 * k
        assert np.allclose(c[pix, :3], col, rtol=2e-4, atol=2e-6), pix   # float32 rd . sun at the disk edge


def test_oracle_heat_map_and_debug_view_properties(small):
    """heat (resolve.wgsl:36-44): no iterations -> blue, 300 or more -> red;
    SURFACE_DEBUG 1 (resolve.wgsl:579): n * 0.5 + 0.5 without the fog blend,
    so a +Y face reads (0.5, 1, 0.5) and the sky keeps its colour."""
    w, pools = small
    v = look_view(w, look_camera(64, 36, pitch=math.radians(-30.0)))
    o = Oracle(v, *pools)
    heat = o.resolve_heat(np.array([0, 150, 300, 5000] + [0] * (o.npix - 4), np.uint32))
    assert np.allclose(heat[0], [0.0, 0.0, 1.0, 1.0]) and np.allclose(heat[2], [1.0, 0.0, 0.0, 1.0])
    assert np.array_equal(heat[2], heat[3]) and 0.0 < heat[1, 1] <= 1.0
    vis = o.frame_vis()[0]
    sv = np.ones(o.npix, np.float32)
    look = (LK.atlas(1), LK.block_faces())
    dbg = o.resolve(vis, sv, *look, spec_hi=LK.HI_DEFAULT | (1 << 23))
    plain = o.resolve(vis, sv, *look, spec_hi=LK.HI_DEFAULT)
    top = (vis != 0) & (((vis >> np.uint64(37)) & np.uint64(7)) == 3)    # +Y faces (NORMAL_PY)
    blocks = np.array([o.block_at((int(k) >> 24) & 0x1FFF, [(int(k) >> 16) & 63, (int(k) >> 8) & 63, int(k) & 63])
                       for k in vis[top]])
    dry = np.flatnonzero(top)[(blocks != 13) & (blocks != 10)]
    assert dry.size > 100
    assert np.allclose(dbg[dry, :3], [0.5, 1.0, 0.5])
    assert np.array_equal(dbg[vis == 0], plain[vis == 0])


# ---------------------------------------------------------------- GPU -----

def light_bricks(v, bricks, seed):
    """Non-uniform light volumes for every chunk of the view, appended to the
    brick pool in the engine's format (light.rs pack_bricks: 4096 cell words,
    uniform cells UNIFORM_BIT | packed, others a pointer to 32 words of two
    16-bit voxels)."""
    rng = np.random.default_rng(seed)
    extra = []
    base = bricks.size
    chunks = v.chunks.copy()
    for i in range(len(chunks)):
        cells = np.empty(4096, np.uint32)
        words = []
        for cell in range(4096):
            if rng.random() < 0.6:
                sky = int(rng.integers(0, 16))
                rgb = rng.integers(0, 16, 3) * (rng.random() < 0.2)
                cells[cell] = 0x80000000 | (sky << 12) | (int(rgb[0]) << 8) | (int(rgb[1]) << 4) | int(rgb[2])
            else:
                vox = (rng.integers(0, 16, 64) << 12) | (rng.integers(0, 16, 64) * (rng.random(64) < 0.3))
                vox = vox.astype(np.uint32)
                cells[cell] = base + 4096 + sum(len(x) for x in words)
                words.append((vox[0::2] | (vox[1::2] << 16)).astype(np.uint32))
        chunks[i]["light_base"] = base
        chunks[i]["light_flags"] = 0
        blob = np.concatenate([cells] + words)
        extra.append(blob)
        base += blob.size
    return chunks, np.concatenate([bricks] + extra)


def gpu_resolve(v, pools, look, spec_hi, soften=None, spec=None):
    from voxelcraft_menu_b200.march import Marcher
    m = Marcher(v.res[0], v.res[1])
    try:
        if spec is not None:
            m.set_spec(spec)
        m.upload_world(*pools)
        m.upload_view(v)
        m.upload_look(*look)
        m.render()
        mask = None
        if soften is not None:
            m.soften_shadows(*soften)
            mask = m.read_shadow_mask()
        m.resolve(spec_hi)
        return m.read_vis(), m.read_shadow(), mask, m.read_color()
    finally:
        m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["default", "engine_atlas", "probes_shaft", "plain_flags", "legacy_lighting",
                                  "reflect_legs", "per_pixel_legs", "probe_tap", "probe_ambient", "water_look"])
def test_resolve_matches_the_oracle(small, case):
    w, pools = small
    cam = look_camera()
    v = look_view(w, cam)
    probes = shaft = None
    spec_hi = LK.HI_DEFAULT
    if case == "probes_shaft":
        probes = LK.probe_field(5)
        shaft = LK.shaft_envelope(w.recipe, v.frame.sun_dir, v.frame.shaft_origin, 4.0)
    elif case == "plain_flags":
        v.frame.flags &= ~(LK.FLAG_LIGHT_RGB | LK.FLAG_SKY_TINT | LK.FLAG_AO | LK.FLAG_TEX_VARIATION | LK.FLAG_TINT)
        spec_hi = 0
    elif case == "legacy_lighting":
        spec_hi = LK.HI_DEFAULT | LK.HI_LEGACY_LIGHTING
    elif case == "reflect_legs":
        v.frame.flags |= W.FLAG_WATER_REFLECT | W.FLAG_WAVES
        spec_hi = LK.HI_DEFAULT | LK.HI_GLASS_REFLECT
    elif case == "per_pixel_legs":
        v.frame.flags |= W.FLAG_WATER_REFLECT
        v.frame.flags &= ~LK.FLAG_FLAT_SECONDARY
        spec_hi = LK.HI_DEFAULT & ~LK.HI_WATER_SEC
    elif case == "water_look":
        # SPEC_WATER_LOOK (resolve.wgsl:995-1008,1138-1153,1178-1183): ripples on
        # the mirror normal, murk and a shallow tint in the refracted colour
        v.frame.flags |= W.FLAG_WAVES
        spec_hi = LK.HI_DEFAULT | LK.HI_WATER_LOOK
    elif case in ("probe_tap", "probe_ambient"):
        # SPEC_PROBE_TAP / SPEC_PROBE_AMBIENT (resolve.wgsl:500-505): the probe
        # field through the clamped linear sampler scales, or replaces, the ambient
        probes = LK.probe_field(5)
        v.frame.flags |= LK.FLAG_PROBE_TAP if case == "probe_tap" else LK.FLAG_PROBE_AMBIENT
    atlas = engine_atlas() if case == "engine_atlas" else LK.atlas(2)
    look = (atlas, LK.block_faces(), probes, shaft)
    vis, sh, _, got = gpu_resolve(v, pools, look, spec_hi)
    o = Oracle(v, *pools)
    want_vis = o.frame_vis()[0]
    assert np.array_equal(vis, want_vis)
    want = o.resolve(vis, LK.sun_visibility(sh), *look, spec_hi=spec_hi)
    within(got, want, case)


@pytest.mark.gpu
def test_resolve_with_light_bricks_soft_mask_and_overrides(small):
    w, pools = small
    cam = look_camera(flags=0)
    v = look_view(w, cam, seed=11)
    v.frame.haze_warm, v.frame.zenith_deep, v.frame.cloud_patch, v.frame.cloud_relief = 0.6, 0.4, 0.5, 0.7
    v.frame.daylight = 0.7
    chunks, bricks = light_bricks(v, pools[2], seed=4)
    v.chunks = chunks
    lp = (pools[0], pools[1], bricks)
    probes = LK.probe_field(9)
    shaft = LK.shaft_envelope(w.recipe, v.frame.sun_dir, v.frame.shaft_origin, 4.0)
    look = (LK.atlas(5), LK.block_faces(), probes, shaft)
    spec_hi = (LK.HI_DEFAULT | LK.HI_SKY_LOOK | LK.HI_SKY_COOL | LK.HI_FOLIAGE_RICH | LK.HI_CANOPY_RELIEF |
               LK.HI_CAUSTICS | LK.HI_TINT_BALANCE)
    vis, sh, mask, got = gpu_resolve(v, lp, look, spec_hi, soften=(4, 1.5))
    o = Oracle(v, *lp)
    want = o.resolve(vis, LK.sun_visibility(sh, mask=mask), *look, spec_hi=spec_hi)
    within(got, want, "light bricks + overrides")


@pytest.mark.gpu
def test_resolve_rejects_unbuilt_variants(small):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    v = look_view(w, look_camera(64, 36))
    m = Marcher(64, 36)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        m.render()
        with pytest.raises(RuntimeError):
            m.resolve(LK.HI_DEFAULT)                      # no atlas yet
        m.upload_look(LK.atlas(1), LK.block_faces())
        with pytest.raises(RuntimeError):
            m.read_color()                                # no resolve yet
        m.resolve(LK.HI_DEFAULT)
        assert m.read_color().shape == (64 * 36, 4)
        v.frame.flags |= W.FLAG_HEATMAP
        m.upload_view(v)
        m.render()
        with pytest.raises(RuntimeError):
            m.resolve(LK.HI_DEFAULT)          # a heat map needs the engine passes' iteration counts
    finally:
        m.close()


FLAG_SNELL = 8388608   # the engine's FLAG_SNELL frame flag (src/render/mod.rs)


@pytest.mark.gpu
@pytest.mark.parametrize("snell", [False, True])
def test_underwater_resolve_matches_the_oracle(small, snell):
    """An underwater frame (resolve.wgsl:1396-1464): the fog path starts at the
    sea surface (water_path), no sun shafts, and every pixel ends with
    surface_from_below (with FLAG_SNELL the waved sea surface seen from below,
    Fresnel-weighted against the water body) and the camera ray's water
    medium (resolve.wgsl:1321-1376)."""
    w, pools = small
    # the deepest sea floor away from the world's edge, the camera 4 above it
    h, x, z = min((W.surface_height(w.recipe, x, z), x, z) for x in range(32, 224, 4) for z in range(32, 224, 4))
    assert h + 4 < w.recipe.water_level - 3                 # deeper than SNELL_MIN_DEPTH
    flags = (W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_UNDERWATER | W.FLAG_WATER_FAR | W.FLAG_WAVES |
             LK.LOOK_FLAGS | (FLAG_SNELL if snell else 0))
    cam = W.Camera(pos=(x + 0.5, h + 4.0, z + 0.5), pitch=math.radians(25.0), width=320, height=200, flags=flags)
    v = look_view(w, cam)
    look = (LK.atlas(1), LK.block_faces(), LK.probe_field(5),
            LK.shaft_envelope(w.recipe, v.frame.sun_dir, v.frame.shaft_origin, 4.0))
    vis, sh, _, got = gpu_resolve(v, pools, look, LK.HI_DEFAULT)
    o = Oracle(v, *pools)
    assert np.array_equal(vis, o.frame_vis()[0])
    want = o.resolve(vis, LK.sun_visibility(sh), *look, spec_hi=LK.HI_DEFAULT)
    within(got, want, f"underwater, snell {snell}")
    assert (vis == 0).any() and (vis != 0).any()


@pytest.mark.gpu
def test_heat_map_view_matches_the_oracle(small):
    """FLAG_HEATMAP (resolve.wgsl:36-44,1389-1394): after the engine passes
    (tile_select, march), every pixel's colour is heat(iterations / 300)."""
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    v = w.view(W.small_terrain_camera(width=320, height=180, flags=W.FLAG_HEATMAP))
    m = Marcher(320, 180)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        m.select()
        m.march()
        m.resolve(0)
        got = m.read_color()
        it = m.read_heatmap()
    finally:
        m.close()
    o = Oracle(v, *pools)
    assert np.array_equal(it, o.frame_vis(heat=True)[3])
    assert it.max() > 0
    within(got, o.resolve_heat(it), "heat map")


@pytest.mark.gpu
@pytest.mark.parametrize("view", range(1, 8))
def test_surface_debug_views_match_the_oracle(small, view):
    """SURFACE_DEBUG = (FLAG_HI_* >> 23) & 7 (resolve.wgsl:579-582,1200-1202,
    1449-1464): 1 normal, 2 sun visibility, 3 sun, 4 ambient of the surface
    lanes, 5 normal, 6 reflected, 7 refracted colour of the water lane, no
    fog blend."""
    w, pools = small
    v = look_view(w, look_camera())
    v.frame.flags |= W.FLAG_WAVES
    look = (LK.atlas(1), LK.block_faces(), LK.probe_field(5),
            LK.shaft_envelope(w.recipe, v.frame.sun_dir, v.frame.shaft_origin, 4.0))
    hi = LK.HI_DEFAULT | (view << 23)
    vis, sh, _, got = gpu_resolve(v, pools, look, hi)
    want = Oracle(v, *pools).resolve(vis, LK.sun_visibility(sh), *look, spec_hi=hi)
    within(got, want, f"debug view {view}")


@pytest.mark.gpu
def test_compact_shade_hit_gives_the_legacy_colours(small):
    """SPEC_COMPACT_SHADE_HIT (FLAG_HI_COMPACT_SHADE_HIT): shade_hit_compact
    and shade_hit_compact_cached (resolve.wgsl:587-851,1790-2054) run the
    legacy variants' statements with the material block after the light
    block, the light times face_scale = 1.0: the same colours, bit for bit."""
    w, pools = small
    v = look_view(w, look_camera())
    v.frame.flags |= W.FLAG_WATER_REFLECT | W.FLAG_WAVES   # legs shade through the non-cached variant too
    look = (LK.atlas(1), LK.block_faces(), LK.probe_field(5),
            LK.shaft_envelope(w.recipe, v.frame.sun_dir, v.frame.shaft_origin, 4.0))
    hi = LK.HI_DEFAULT | LK.HI_GLASS_REFLECT
    _, _, _, legacy = gpu_resolve(v, pools, look, hi)
    vis, sh, _, compact = gpu_resolve(v, pools, look, hi | LK.HI_COMPACT_SHADE_HIT)
    assert np.array_equal(compact, legacy)
    want = Oracle(v, *pools).resolve(vis, LK.sun_visibility(sh), *look, spec_hi=hi | LK.HI_COMPACT_SHADE_HIT)
    within(compact, want, "compact")


@pytest.mark.gpu
def test_resolve_replays_from_a_cuda_graph(small):
    """vm_resolve forks its water and glass lanes onto streams of the context
    with events and joins them back into the caller's stream: recorded into a
    stream capture the caller owns (a torch CUDA graph) and replayed, it
    writes the colours of a direct call, bit for bit."""
    import torch
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    v = look_view(w, look_camera())
    look = (LK.atlas(1), LK.block_faces(), LK.probe_field(5),
            LK.shaft_envelope(w.recipe, v.frame.sun_dir, v.frame.shaft_origin, 4.0))
    m = Marcher(v.res[0], v.res[1])
    try:
        side = torch.cuda.Stream()
        m.set_stream(side.cuda_stream)
        m.upload_world(*pools)
        m.upload_view(v)
        m.upload_look(*look)
        m.render()
        m.resolve(LK.HI_DEFAULT)          # sizes the resolve's buffers and streams outside the capture
        want = m.read_color()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side, capture_error_mode="thread_local"):
            m.resolve(LK.HI_DEFAULT)
        torch.cuda.synchronize()
        m.resolve(0)                      # another look over the colour buffer before each replay
        plain = m.read_color()
        assert not np.array_equal(plain, want)
        for _ in range(2):
            with torch.cuda.stream(side):     # the replay follows the direct calls on the caller's stream
                g.replay()
            assert np.array_equal(m.read_color(), want)
            m.resolve(0)
        del g
    finally:
        m.close()


@pytest.mark.gpu
def test_full_hd_frame_resolve_matches_the_oracle():
    rec = W.recipe_large_terrain()
    w = W.World.generate(rec)
    pools = w.pools()
    cam = W.large_terrain_camera(rec, flags=W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | LK.LOOK_FLAGS)
    v = w.view(cam)
    LK.apply_defaults(v.frame, rec.seed)
    probes = LK.probe_field(rec.seed)
    shaft = LK.shaft_envelope(rec, v.frame.sun_dir, v.frame.shaft_origin, 4.0)
    look = (LK.atlas(rec.seed), LK.block_faces(), probes, shaft)
    vis, sh, _, got = gpu_resolve(v, pools, look, LK.HI_DEFAULT)
    o = Oracle(v, *pools)
    want = o.resolve(vis, LK.sun_visibility(sh), *look, spec_hi=LK.HI_DEFAULT)
    within(got, want, "1080p")
