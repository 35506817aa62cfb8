"""Frame assembly for hq renders: the camera (crates/lumenwright/src/scene/camera.rs), `hq_params`
(crates/lumenwright/src/request.rs:1153-1225) and the benchmark configurations, each as a seeded
synthetic world drawn through the reference's frame set-up (request.rs:640-653, 751-930).
"""

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import anvil as AN
from . import gamesky as G
from . import layout as L
from . import sky as SK
from . import synth as S
from .hqbuild import build_hq
from .scene import HqFrame, HqScene

F32 = np.float32


@dataclass
class Camera:
    """`Camera` (camera.rs:5-16): eye position (f64 world coordinates), Minecraft yaw and pitch in
    degrees, vertical field of view."""

    pos: tuple
    yaw: float
    pitch: float
    fov_y: float = 70.0

    def forward(self):
        """camera.rs:20-23 (f32)."""
        y, p = np.radians(F32(self.yaw), dtype=F32), np.radians(F32(self.pitch), dtype=F32)
        return SK.normalize32([-np.sin(y) * np.cos(p), -np.sin(p), np.cos(y) * np.cos(p)])

    def basis(self):
        """camera.rs:26-37: (forward, right, up)."""
        f = self.forward()
        r = np.cross(f, np.array([0, 1, 0], F32)).astype(F32)
        if float(r @ r) < 1e-8:
            y = np.radians(F32(self.yaw), dtype=F32)
            r = np.array([-np.cos(y), 0.0, -np.sin(y)], F32)
        r = SK.normalize32(r)
        u = SK.normalize32(np.cross(r, f).astype(F32))
        return f, r, u

    @staticmethod
    def look_at(frm, to):
        """camera.rs:40-45: yaw and pitch from `frm` towards `to` (f64)."""
        d = np.asarray(to, np.float64) - np.asarray(frm, np.float64)
        d = d / math.sqrt(float(d @ d))
        pitch = math.degrees(math.asin(-d[1]))
        yaw = math.degrees(math.atan2(-d[0], d[2]))
        return F32(yaw), F32(pitch)


def hq_params(width, height, hq: HqScene, eye, cam: Camera, s: SK.HqSky, *, spp_seed=0, max_bounces=4,
              emitter_intensity=SK.DEFAULT_EMITTER_INTENSITY, emitter_sampling=L.EMITTER_SAMPLING_ONE,
              prevent_normal_emitter=False, turbidity=2.5) -> np.ndarray:
    """`hq_params` (request.rs:1153-1225)."""
    f, r, u = cam.basis()
    tan_half = F32(math.tan(math.radians(cam.fov_y) * 0.5))
    aspect = F32(width) / F32(height)
    sky = SK.Preetham(s.sun_dir, turbidity)
    su, sv = SK.sun_texture_axes(s.sun_dir)
    p = L.new_params()
    f4 = lambda v, w: [F32(v[0]), F32(v[1]), F32(v[2]), F32(w)]  # noqa: E731
    p["cam_pos"] = f4(eye, tan_half)
    p["cam_fwd"] = f4(f, aspect)
    p["cam_right"] = f4(r, 0.0)
    p["cam_up"] = f4(u, 0.0)
    p["sun_dir"] = f4(s.sun_dir, math.cos(float(SK.SUN_RADIUS)))
    p["sun_color"] = f4(s.sun_color, SK.SUN_RADIUS)
    p["sky_sun"] = f4(sky.sun, s.sky_light)
    p["sky_zenith"] = f4(sky.zenith, 0.0)
    for k, name in enumerate(("perez_a", "perez_b", "perez_c", "perez_d", "perez_e")):
        p[name] = f4(sky.perez[k], 0.0)
    p["water_color"] = [0.42, 0.16, 0.10, 1.333]
    p["misc_f"] = [emitter_intensity, 1e-3, SK.SKY_CACHE_RESOLUTION, 0.0]
    d = hq.dims
    p["grid_dims"] = [d[0], d[1], d[2], d[0] * d[1] * d[2]]
    p["off"] = list(hq.offsets[:4])
    p["off2"] = [hq.offsets[4], hq.atlas_size[0], hq.atlas_size[1], hq.quads.size]
    p["frame"] = [width, height, 0, max_bounces]
    p["misc_u"] = [spp_seed, 1, hq.models.size, hq.emitter_count]
    p["see_through"] = [hq.see_through[0], hq.see_through[1], 0, 0]
    strategy = emitter_sampling if float(emitter_intensity) > 0.0 else L.EMITTER_SAMPLING_NONE
    p["emitter"] = [strategy, int(prevent_normal_emitter), 0, 0]
    p["sun_su"] = f4(su, SK.SUN_TEXTURE_BRIGHTNESS)
    p["sun_sv"] = f4(sv, F32(4.0) * SK.SUN_RADIUS)
    p["sun_sprite"] = list(hq.sun_sprite) if hq.sun_sprite else [0.0] * 4
    p["sky_map"] = [0.0] * 4
    p["water_plane"] = [0.0] * 4
    return p


def water_plane_height(sea_level: float) -> float:
    """request.rs:206-208: a source block's surface (8/9 high) in the layer below the sea level."""
    return sea_level - 1.0 + 8.0 / 9.0


@dataclass
class Config:
    """One benchmark configuration (synthetic world + render settings)."""

    name: str
    chunks: int
    width: int
    height: int
    spp: int
    bounces: int
    time: int
    look: str  # "chunky" or "game"
    emitters: bool = False
    water_plane: Optional[float] = None
    seed: int = 1
    eye: tuple = (32.0, 100.0, 32.0)
    target: tuple = (0.0, 64.0, 0.0)
    origin_x: float = 0.0  # world x of the grid's first column (the world is translated by it)
    notes: dict = field(default_factory=dict)


CONFIGS = {
    # Plain hq path trace, CPU-runnable.
    "c1": Config("c1", 4, 256, 144, 16, 4, 4000, "chunky"),
    # Drop-in scale: 12x12 chunks with emitters and the water plane, game sky at dusk.
    "c2": Config("c2", 12, 1280, 720, 1024, 8, 12800, "game", emitters=True, water_plane=63.0),
    # Differentiation world.
    "c4": Config("c4", 8, 512, 288, 64, 4, 4000, "chunky"),
    # Precision: 32x32 chunks translated to x = 1,000,000, the camera at a fractional position
    # there; the host rebases it to the grid in f64 before the f32 cast.
    "c5": Config("c5", 32, 3840, 2160, 4096, 8, 4000, "chunky", emitters=True, water_plane=63.0,
                 eye=(1_000_256.37, 120.61, 256.29), target=(1_000_128.5, 70.0, 128.5), origin_x=1_000_000.0),
}


def config_world(cfg: Config) -> S.World:
    """The configuration's seeded world, its first column at x = ``cfg.origin_x``."""
    world = S.generate_world(cfg.chunks, cfg.seed, emitters=cfg.emitters)
    world.origin = (cfg.origin_x, world.origin[1], world.origin[2])
    return world


def write_save(cfg: Config, path: str) -> list:
    """Writes the configuration's world as an Anvil save in `path` (``level.dat`` and
    ``region/``, `anvil.write_world`): its chunks where the frame places them, the day time the
    frame's, the spawn under the eye. Returns the region files written."""
    spawn = (math.floor(cfg.eye[0]), 64, math.floor(cfg.eye[2]))
    return AN.write_world(config_world(cfg), path, name=f"Lumenwright {cfg.name}", spawn=spawn, day_time=cfg.time)


def make_frame(cfg: Config, sky_backend=None, width=None, height=None, spp=None, save: Optional[str] = None) -> HqFrame:
    """The hq frame of a configuration, as `render()` assembles it (request.rs:640-653, 751-930).

    ``sky_backend`` builds the sky inputs: an object with ``build_sky_cache(params, n)`` (`sky_cache`,
    crates/lumenwright/src/render/sky.rs:593-611), ``draw_sky_map(quick_sky, stars, w, h, atlas,
    atlas_w)`` (`draw_map`, sky.rs:861-878: the game sky's maps, from the stated sky of the tick,
    ``gamesky.stated_sky``) and ``blend_chunky_sky(params, cache, maps, sizes, weight)``
    (sky.rs:836-850); by default the library's device kernels on device 0.

    ``save`` names an Anvil save to load the world from (`anvil.read_world`, the configuration's
    chunks, as `World::open` and `load_area` load them, world/mod.rs:297-491) instead of
    generating it; `write_save` writes the configuration's own.
    """
    width = width or cfg.width
    height = height or cfg.height
    spp = spp or cfg.spp
    own = None
    if sky_backend is None:
        from .native import Context
        own = sky_backend = Context(0)
    try:
        if save is None:
            world = config_world(cfg)
        else:
            world = AN.read_world(save, (int(cfg.origin_x) // 16, 0), (cfg.chunks, cfg.chunks))
        atlas = S.build_atlas(cfg.seed)
        hq = build_hq(world, atlas)
        yaw, pitch = Camera.look_at(cfg.eye, cfg.target)
        cam = Camera(cfg.eye, float(yaw), float(pitch), 70.0)
        origin = world.origin
        eye64 = tuple(float(cfg.eye[i]) - float(origin[i]) for i in range(3))
        eye = [F32(e) for e in eye64]  # f64 difference, then f32
        sun_dir = SK.sun_direction_from_angle(SK.celestial_angle(cfg.time))
        weight = F32(1.0) if cfg.look == "chunky" else SK.dusk_day_weight(cfg.time)
        intensity = SK.default_emitter_intensity(False, weight)
        p = hq_params(width, height, hq, eye, cam, SK.hq_sky(sun_dir), max_bounces=cfg.bounces,
                      emitter_intensity=intensity)
        if cfg.water_plane is not None:
            p["water_plane"] = [F32(water_plane_height(cfg.water_plane) - origin[1]), 1.0, 0.0, 0.0]
        cache = sky_backend.build_sky_cache(p, int(p["misc_f"][2]))
        if weight >= 1.0:
            sky = cache
        else:
            desc, factor, colour = G.stated_sky(cfg.time, hq.sun_sprite)
            maps, sizes, _ = G.game_sky_maps(sky_backend, desc, factor, colour, hq.atlas, hq.atlas_size[0])
            if weight > 0.0:
                maps = sky_backend.blend_chunky_sky(p, cache, maps, sizes, weight)
                p["sun_color"][:3] = p["sun_color"][:3] * weight
                p["sun_su"][3] = p["sun_su"][3] * weight
            else:
                p["sun_color"][:3] = 0.0
                p["sun_sprite"] = [0.0] * 4
            p["sky_map"] = sizes
            p["misc_f"][2] = 0.0
            sky = maps
    finally:
        if own is not None:
            own.close()
    cfg.notes.update(dict(weight=float(weight), emitter_intensity=float(intensity), stats=vars(hq.stats),
                          emitters=world.emitters_placed, solid=world.solid_blocks))
    return HqFrame(scene=hq, params=p, spp=spp, sky=sky, eye64=eye64)


def with_chunk_frames(frame: HqFrame) -> HqFrame:
    """The same frame rendered with chunk-origin rebasing (the precision form's option): the eye,
    relative to the grid origin in f64, split by `lw_rebase_camera` into the chunk corner nearest
    it and an f32 remainder of at most 8 blocks per axis; the kernels then hold every path origin
    relative to its own nearest chunk corner. The scene, sky and random streams are unchanged."""
    from .native import rebase_camera
    if frame.eye64 is None:
        raise ValueError("chunk frames need the frame's f64 eye")
    return HqFrame(scene=frame.scene, params=rebase_camera(frame.params, frame.eye64), spp=frame.spp, sky=frame.sky,
                   eye64=frame.eye64)
