"""Hand-built scenes of the reference kernel tests (`crates/lumenwright-kernel/src/tests.rs`),
restated as flat buffers. The oracle tests and the CUDA parity tests run on the same
fixtures, so each known answer pins both.
"""

import numpy as np

from lumenwright_b200 import layout as L

INF = float("inf")


def norm(v):
    v = np.asarray(v, dtype=np.float32)
    n = np.float32(np.sqrt(np.float32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))
    return (v * (np.float32(1.0) / n)).astype(np.float32)


def quad(p0, eu, ev, flags):
    """tests.rs:13-22: a 2x1 atlas quad (texel 0 opaque white, texel 1 transparent)."""
    return L.make_quad(p0, eu, ev, flags=flags, tint=0xFFFF_FFFF, emittance=0.0,
                       uv=(0.0, 0.0, 2.0, 0.0), uvt=(0.0, 1.0))


def cube(flags):
    """tests.rs:25-35: unit cube faces in block-local space, normal = ev x eu outward."""
    x, y, z = np.array([1.0, 0, 0]), np.array([0, 1.0, 0]), np.array([0, 0, 1.0])
    return [
        quad((1, 1, 0), -x, -y, flags),  # north
        quad((0, 1, 1), x, -y, flags),   # south
        quad((1, 1, 1), -z, -y, flags),  # east
        quad((0, 1, 0), z, -y, flags),   # west
        quad((0, 1, 0), x, z, flags),    # up
        quad((0, 0, 1), x, -z, flags),   # down
    ]


class KScene:
    """A `KScene` (tests.rs:37-46): params plus the seven buffers plus the sky."""

    def __init__(self, params, grid, models, quads, atlas, emitters, emitter_grid, sky=None):
        self.params = params
        self.grid = np.asarray(grid, dtype=np.uint32)
        self.models = models
        self.quads = quads
        self.atlas = np.asarray(atlas, dtype=np.uint32)
        self.emitters = emitters
        self.emitter_grid = np.asarray(emitter_grid, dtype=np.uint32)
        self.sky = np.zeros(0, np.float32) if sky is None else np.asarray(sky, dtype=np.float32)

    def buffers(self):
        return (self.params, self.grid, self.models, self.quads, self.atlas, self.emitters,
                self.emitter_grid, self.sky)


def models_array(rows):
    m = np.zeros(len(rows), dtype=L.MODEL_DTYPE)
    for i, (off, cnt) in enumerate(rows):
        m[i]["quad_offset"] = off
        m[i]["quad_count"] = cnt
    return m


def emitters_array(rows):
    """rows of (x, y, z, first_quad, faces)."""
    e = np.zeros(max(len(rows), 1), dtype=L.EMITTER_DTYPE)
    w = e.view("<u4").reshape(-1, 8)
    for i, (x, y, z, fq, faces) in enumerate(rows):
        w[i, 0:3] = np.array([x, y, z], dtype="<f4").view("<u4")
        w[i, 3] = fq
        w[i, 4] = faces
    return e


def basic_scene(entity: bool) -> KScene:
    """tests.rs:49-112: 3x1x1 bricks; brick 0 empty, brick 1 one cube at local (4,5,5),
    brick 2 uniform cubes; with ``entity`` an overlay quad in brick 0 at x = 8.5."""
    quads = cube(L.ALPHA_OPAQUE)
    models = models_array([(0, 0), (0, 6)])
    nb = 3
    top = [L.EMPTY, 0, L.UNIFORM | 1]
    brick = np.zeros(L.BRICK_WORDS, np.uint32)
    local = (5 * 16 + 5) * 16 + 4
    brick[local >> 1] |= 1 << ((local & 1) * 16)
    ov_top = [L.EMPTY] * nb
    ov_cells, ov_quads = [], []
    if entity:
        quads.append(quad((8.5, 6.0, 5.0), (0, 0, 1.0), (0, -1.0, 0), L.ALPHA_CUTOUT))
        ov_top[0] = 0
        ov_cells = np.zeros(L.OV_CELL_WORDS, np.uint32)
        cell = (5 * 16 + 5) * 16 + 8
        ov_cells[cell * 2] = 0
        ov_cells[cell * 2 + 1] = 1
        ov_quads = [6]
    grid = list(top)
    off_bricks = len(grid)
    grid += list(brick)
    off_ov_top = len(grid)
    grid += ov_top
    off_ov_cells = len(grid)
    grid += list(ov_cells)
    off_ov_quads = len(grid)
    grid += ov_quads
    grid.append(0)
    p = L.new_params()
    p["grid_dims"] = [3, 1, 1, nb]
    p["off"] = [0, off_bricks, off_ov_top, off_ov_cells]
    p["off2"] = [off_ov_quads, 2, 1, len(quads)]
    p["misc_f"] = [1.0, 1e-3, 0.0, 0.0]
    return KScene(p, grid, models, L.quads_array(quads), [0xFFFF_FFFF, 0x0000_0000],
                     emitters_array([]), [0] * L.EMITTER_GRID_HEADER)


def hollow_scene() -> KScene:
    """3x1x1 bricks holding a model without quads (a fluid block inside its fluid): brick 0 is a
    uniform brick of it, brick 1 is full of it but for one cube at local (8, 5, 5) and one air voxel
    at (3, 9, 9), brick 2 is uniform cubes. The traversal re-lays the model as air."""
    quads = cube(L.ALPHA_OPAQUE)
    models = models_array([(0, 0), (0, 6), (6, 0)])
    nb = 3
    top = [L.UNIFORM | 2, 0, L.UNIFORM | 1]
    ids = np.full(4096, 2, np.uint32)
    ids[(5 * 16 + 5) * 16 + 8] = 1
    ids[(9 * 16 + 9) * 16 + 3] = 0
    brick = (ids[0::2] | (ids[1::2] << 16)).astype(np.uint32)
    grid = list(top)
    off_bricks = len(grid)
    grid += list(brick)
    off_ov_top = len(grid)
    grid += [L.EMPTY] * nb
    off_ov_cells = len(grid)
    off_ov_quads = len(grid)
    grid.append(0)
    p = L.new_params()
    p["grid_dims"] = [3, 1, 1, nb]
    p["off"] = [0, off_bricks, off_ov_top, off_ov_cells]
    p["off2"] = [off_ov_quads, 2, 1, len(quads)]
    p["misc_f"] = [1.0, 1e-3, 0.0, 0.0]
    return KScene(p, grid, models, L.quads_array(quads), [0xFFFF_FFFF, 0x0000_0000],
                  emitters_array([]), [0] * L.EMITTER_GRID_HEADER)


LAMP_EMITTANCE = 0.5  # tests.rs:301
LAMP_INTENSITY = 13.0  # tests.rs:303


def lamp_scene(strategy: int, decoy: bool) -> KScene:
    """tests.rs:310-395: a 16^3 floor of white cubes at y = 0 and a lamp quad facing down at
    (7, 4, 7); with ``decoy`` a second emitter at (2, 0, 2) the floor never sees."""
    quads = cube(L.ALPHA_OPAQUE)
    quads.append(L.make_quad((0, 0, 0), (0, 0, 1.0), (1.0, 0, 0), flags=L.ALPHA_OPAQUE,
                             emittance=LAMP_EMITTANCE, uv=(0, 0, 2.0, 0), uvt=(0, 1.0)))
    quads.append(L.make_quad((0, 0, 0), (1.0, 0, 0), (0, 0, 1.0), flags=L.ALPHA_OPAQUE,
                             emittance=LAMP_EMITTANCE, uv=(0, 0, 2.0, 0), uvt=(0, 1.0)))
    qa = L.quads_array(quads)
    qa["uv"][:, 2] = 1.0  # white texels only
    models = models_array([(0, 0), (0, 6), (6, 1), (7, 1)])
    brick = np.zeros(L.BRICK_WORDS, np.uint32)

    def put(x, y, z, m):
        local = (y * 16 + z) * 16 + x
        brick[local >> 1] |= m << ((local & 1) * 16)

    for z in range(16):
        for x in range(16):
            if not (decoy and x == 2 and z == 2):
                put(x, 0, z, 1)
    put(7, 4, 7, 2)
    if decoy:
        put(2, 0, 2, 3)
    grid = [0] + list(brick)
    off_bricks = 1
    off_ov_top = len(grid)
    grid.append(L.EMPTY)
    off_ov_cells = len(grid)
    off_ov_quads = len(grid)
    grid.append(0)
    em = [(7.0, 4.0, 7.0, 6, 1)]
    if decoy:
        em.append((2.0, 0.0, 2.0, 7, 1))
    eg = [16, 1, 1, 1, 0, 0, 0, 0, 0, len(em)] + list(range(len(em)))
    p = L.new_params()
    p["grid_dims"] = [1, 1, 1, 1]
    p["off"] = [0, off_bricks, off_ov_top, off_ov_cells]
    p["off2"] = [off_ov_quads, 2, 1, len(quads)]
    p["misc_f"] = [LAMP_INTENSITY, 1e-3, 0.0, 0.0]
    p["misc_u"] = [7, 1, 4, len(em)]
    p["emitter"] = [strategy, 0, 0, 0]
    p["frame"] = [8, 8, 0, 3]
    p["sun_dir"] = [0.0, -1.0, 0.0, 1.0]
    return KScene(p, grid, models, qa, [0xFFFF_FFFF, 0x0000_0000], emitters_array(em), eg)


# tests.rs:592-600: Preetham at altitude 45 degrees, turbidity 2.5.
PREETHAM_45_ZENITH = [0.29624206, 0.30751193, 8.306274, 0.0]
PREETHAM_PEREZ = [
    [-0.30745, -0.30255, -1.01625, 0.0],
    [-0.16545, -0.2283, -0.461, 0.0],
    [0.2115, 0.19045, 5.26835, 0.0],
    [-1.05915, -1.76395, -2.2756, 0.0],
    [0.03695, 0.02565, 0.2028, 0.0],
]


def set_preetham_45(p):
    p["sky_sun"] = [0.5, np.float32(np.sqrt(0.5)), 0.5, 1.0]
    p["sky_zenith"] = PREETHAM_45_ZENITH
    for k, name in enumerate(("perez_a", "perez_b", "perez_c", "perez_d", "perez_e")):
        p[name] = PREETHAM_PEREZ[k]


def wall_scene() -> KScene:
    """tests.rs:607-654: 16 bricks along x, a stray cube in each of bricks 0-14, a wall of
    front-only cubes at x = 250 in brick 15."""
    quads = L.quads_array(cube(L.ALPHA_OPAQUE | L.FLAG_FRONT_ONLY))
    models = models_array([(0, 0), (0, 6)])
    nb = 16
    top = [0] * nb
    top[15] = 1
    stray = np.zeros(L.BRICK_WORDS, np.uint32)
    corner = (15 * 16 + 15) * 16
    stray[corner >> 1] |= 1 << ((corner & 1) * 16)
    wall = np.zeros(L.BRICK_WORDS, np.uint32)
    for y in range(16):
        for z in range(16):
            local = (y * 16 + z) * 16 + (250 - 240)
            wall[local >> 1] |= 1 << ((local & 1) * 16)
    grid = top + list(stray) + list(wall)
    off_bricks = nb
    off_ov_top = len(grid)
    grid += [L.EMPTY] * nb
    off_ov_cells = len(grid)
    grid.append(0)
    p = L.new_params()
    p["grid_dims"] = [16, 1, 1, nb]
    p["off"] = [0, off_bricks, off_ov_top, off_ov_cells]
    p["off2"] = [off_ov_cells, 2, 1, len(quads)]
    return KScene(p, grid, models, quads, [0xFFFF_FFFF, 0], emitters_array([]),
                     [0] * L.EMITTER_GRID_HEADER)


def wall_rays():
    """The 4096 rays of tests.rs:658-677, as f32 (o, d) pairs."""
    rays = []
    for i in range(64):
        for j in range(64):
            o = np.array([np.float32(0.137) + np.float32(i) * np.float32(0.0131),
                          np.float32(1.1) + np.float32(i) * np.float32(0.03),
                          np.float32(1.3) + np.float32(j) * np.float32(0.05)], dtype=np.float32)
            d = norm([np.float32(1.0),
                      np.float32(0.04) + np.float32(0.002) * (np.float32(j) - np.float32(32.0)) / np.float32(32.0),
                      np.float32(0.03) + np.float32(0.002) * (np.float32(i) - np.float32(32.0)) / np.float32(32.0)])
            rays.append((o, d))
    return rays


def map_scene() -> KScene:
    """tests.rs:725-741: lens map 4x2 holding (i, j, 1), light map 2x2 holding (10+i, 10+j, 2)."""
    s = basic_scene(False)
    s.params["sky_map"] = [4.0, 2.0, 2.0, 2.0]
    sky = []
    for j in range(2):
        for i in range(4):
            sky += [i, j, 1.0]
    for j in range(2):
        for i in range(2):
            sky += [10.0 + i, 10.0 + j, 2.0]
    s.sky = np.array(sky, dtype=np.float32)
    return s


def sky_dir(turns, el):
    """tests.rs:744-747."""
    az = np.float32(turns) * np.float32(2 * np.pi)
    el = np.float32(el)
    return np.array([np.cos(el) * np.cos(az), np.sin(el), np.cos(el) * np.sin(az)], dtype=np.float32)


SUN_ATLAS = (40, 40)  # sky.rs:1153-1163: a 32x32 sun sprite at (3, 5) in a 40x40 atlas
SUN_SPRITE = (3, 5, 32, 32)


def sun_texel(x, y):
    """sky.rs:1155-1157: every texel of the sprite differs."""
    return 0xFF00_0000 | (x * 7 + 3) | ((y * 7 + 3) << 8) | (((x + y) * 3) << 16)


def sun_atlas():
    w, h = SUN_ATLAS
    sx, sy, sw, sh = SUN_SPRITE
    atlas = np.zeros(w * h, np.uint32)
    for y in range(sh):
        for x in range(sw):
            atlas[(y + sy) * w + x + sx] = sun_texel(x, y)
    return atlas


def sun_sprite_params(p, sun):
    """The sun-texture fields of `Params` for a sun direction, as `hq_params` sets them
    (request.rs:1153-1225): `sun_su`/`sun_sv` from `sun_texture_axes` with the brightness and
    half-width in w, the sprite's rectangle in the atlas."""
    from lumenwright_b200 import sky as SK
    su, sv = SK.sun_texture_axes(sun)
    p["sun_dir"] = [sun[0], sun[1], sun[2], np.float32(np.cos(SK.SUN_RADIUS))]
    p["sun_su"] = [su[0], su[1], su[2], SK.SUN_TEXTURE_BRIGHTNESS]
    p["sun_sv"] = [sv[0], sv[1], sv[2], np.float32(4.0) * SK.SUN_RADIUS]
    p["sun_sprite"] = [float(v) for v in SUN_SPRITE]
    return su, sv
