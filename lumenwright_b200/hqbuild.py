"""The hq grid build: `voxel::build_hq` (crates/lumenwright/src/scene/voxel.rs:111-491) and
`emitter_list` (:542-607) for a block volume of the synthetic block set, vectorised per section.

The output buffers are the reference's word for word: the same instance numbering (phase 1's
per-section first-occurrence palettes interned in brick order, phase 2), the same buried and
uniform collapses, the same u16 packing (even voxel in the low half) and the same emitter list
and grid. ``tests/test_hqbuild.py`` checks them against a plain restatement of voxel.rs.
"""

import numpy as np

from . import layout as L
from . import synth as S
from .scene import HqScene, HqStats

EMITTER_CELL = 10  # voxel.rs:532


def fluid_face_masks(blocks: np.ndarray) -> np.ndarray:
    """`Scene::fluid_face_mask` (crates/lumenwright/src/scene/mod.rs:586-609) for every voxel,
    water: bit 7 and the Up bit when water is above; each other face's bit when its neighbour is
    water or occludes. Outside the volume is air."""
    water = blocks == S.WATER
    occl = np.zeros_like(water)
    for sid, info in enumerate(S.BLOCKS):
        if info.occludes:
            occl |= blocks == sid
    pad_w = np.pad(water, 1, constant_values=False)
    pad_o = np.pad(occl, 1, constant_values=False)
    Y, Z, X = blocks.shape

    def nb(arr, d):
        dx, dy, dz = S.DIR_OFFSET[d]
        return arr[1 + dy:1 + dy + Y, 1 + dz:1 + dz + Z, 1 + dx:1 + dx + X]

    mask = np.zeros(blocks.shape, np.uint16)
    mask |= np.where(nb(pad_w, S.UP), 0x80 | (1 << S.UP), 0).astype(np.uint16)
    for d in (S.DOWN, S.NORTH, S.SOUTH, S.WEST, S.EAST):
        mask |= np.where(nb(pad_w, d) | nb(pad_o, d), 1 << d, 0).astype(np.uint16)
    return mask


def emitter_list(models: np.ndarray, sites):
    """`emitter_list` (voxel.rs:542-607): the emitters and the emitter grid from (voxel corner,
    model id) sites, in site order."""
    if len(sites) == 0:
        grid = np.zeros(L.EMITTER_GRID_HEADER, np.uint32)
        grid[0] = EMITTER_CELL
        return np.zeros(1, L.EMITTER_DTYPE), grid
    c = np.array([s[0] for s in sites], np.int64)
    m = np.array([s[1] for s in sites], np.int64)
    em = np.zeros(len(sites), L.EMITTER_DTYPE)
    w = em.view("<u4").reshape(-1, 8)
    w[:, 0:3] = c.astype("<f4").view("<u4")
    w[:, 3] = models["quad_offset"][m]
    w[:, 4] = models["quad_count"][m]
    g = np.floor_divide(c, EMITTER_CELL)
    lo, hi = g.min(0), g.max(0)
    offset = lo - 1
    size = hi - lo + 3
    ncells = int(size[0] * size[1] * size[2])
    counts = np.zeros(ncells, np.int64)
    entries = []  # (cell, emitter) in Chunky's insertion order: emitter-major, then dy, dz, dx
    for dy in (-1, 0, 1):
        for dz in (-1, 0, 1):
            for dx in (-1, 0, 1):
                l = g + np.array([dx, dy, dz]) - offset
                entries.append(((l[:, 1] * size[2] + l[:, 2]) * size[0] + l[:, 0]))
    cells = np.stack(entries, 1)  # (n_sites, 27)
    flat_cell = cells.ravel()
    flat_em = np.repeat(np.arange(len(sites)), 27)
    order = np.argsort(flat_cell, kind="stable")  # stable: per cell, emitters in site order
    np.add.at(counts, flat_cell, 1)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    head = np.array([EMITTER_CELL, size[0], size[1], size[2], offset[0] & 0xFFFFFFFF, offset[1] & 0xFFFFFFFF,
                     offset[2] & 0xFFFFFFFF, 0], np.uint64).astype(np.uint32)
    pairs = np.stack([starts, counts], 1).astype(np.uint32).ravel()
    grid = np.concatenate([head, pairs, flat_em[order].astype(np.uint32)])
    return em, grid


def build_hq(world: "S.World", atlas: "S.Atlas") -> HqScene:
    """`build_hq` (voxel.rs:111-491) for a synthetic world. The grid spans the whole volume:
    ``dims = (chunks_x, 24, chunks_z)`` bricks, brick index ``(y * dz + z) * dx + x``."""
    blocks = world.blocks
    Y, Z, X = blocks.shape
    dims = (X // 16, Y // 16, Z // 16)
    nb = dims[0] * dims[1] * dims[2]
    stats = HqStats()
    occludes = np.array([b.occludes for b in S.BLOCKS])
    simple = np.array([b.simple for b in S.BLOCKS])
    invisible = np.array([b.invisible for b in S.BLOCKS])
    fmask = fluid_face_masks(blocks)
    # Instance key per voxel: the state alone for a simple state; for water, with its fluid mask
    # (the synthetic set has one biome, deterministic models and no self-culling blocks, so the
    # other key fields are the same for every voxel of a state). 0 is air.
    key = blocks.astype(np.int64) * 256
    key += np.where(blocks == S.WATER, fmask, 0)
    key[invisible[blocks]] = 0
    # Sections in brick order (y, z, x), each as its 4096 keys in voxel order (y, z, x).
    sec = key.reshape(dims[1], 16, dims[2], 16, dims[0], 16).transpose(0, 2, 4, 1, 3, 5).reshape(nb, 4096)
    sec_blocks = blocks.reshape(dims[1], 16, dims[2], 16, dims[0], 16).transpose(0, 2, 4, 1, 3, 5).reshape(nb, 4096)
    # Phase 0 (voxel.rs:119-131): a section of occluding blocks only (an all-air section is None).
    all_occluding = np.array([bool(s.any()) and bool(occludes[np.unique(s)].all()) for s in sec_blocks])

    def brick_index(b):
        bx, by, bz = b
        if bx < 0 or by < 0 or bz < 0 or bx >= dims[0] or by >= dims[1] or bz >= dims[2]:
            return None
        return (by * dims[2] + bz) * dims[0] + bx

    model_rows = [(0, 0)]
    quads = []
    model_emits = [False]
    instance_ids = {}
    top = np.full(nb, L.EMPTY, np.uint64)
    bricks = []
    sites = []
    for bi in range(nb):
        k = sec[bi]
        if not k.any():
            continue
        # Phase 1 (voxel.rs:171-260): the section's palette in first-occurrence order.
        uniq, first = np.unique(k, return_index=True)
        keep = uniq != 0
        uniq, first = uniq[keep], first[keep]
        order = np.argsort(first, kind="stable")
        uniq, first = uniq[order], first[order]
        # Phase 2 (voxel.rs:274-343): intern globally in brick order.
        gids = np.zeros(len(uniq), np.int64)
        for i, kk in enumerate(uniq.tolist()):
            iid = instance_ids.get(kk)
            if iid is None:
                state, fm = kk >> 8, kk & 0xFF
                qs = S.block_quads(atlas, state, fm)
                off = len(quads)
                for q in qs:
                    if not (int(q[3]) & L.FLAG_WATER):
                        q = q.copy()
                        q[3] |= L.FLAG_FRONT_ONLY
                    quads.append(q)
                model_emits.append(len(qs) > 0 and S.BLOCKS[state].emittance > 0.0)
                model_rows.append((off, len(qs)))
                iid = len(model_rows) - 1
                instance_ids[kk] = iid
            gids[i] = iid
        if len(model_rows) > 0x10000:
            raise ValueError("more than 65535 distinct block model instances in view")
        lut = np.zeros(int(uniq.max()) + 1, np.int64)
        lut[uniq] = gids
        ids = lut[k]
        by, rem = divmod(bi, dims[0] * dims[2])
        bz, bx = divmod(rem, dims[0])
        buried = all_occluding[bi] and all(
            (n := brick_index((bx + o[0], by + o[1], bz + o[2]))) is not None and all_occluding[n]
            for o in S.DIR_OFFSET.values())
        emits = np.array(model_emits)[ids]
        for local in np.nonzero(emits)[0]:
            lx, ly, lz = local & 15, local >> 8, (local >> 4) & 15
            sites.append(((bx * 16 + lx, by * 16 + ly, bz * 16 + lz), int(ids[local])))
        if buried:
            stats.buried_bricks += 1
            nz = ids[ids != 0]
            top[bi] = L.UNIFORM | (int(nz[0]) if len(nz) else 1)
            continue
        if np.all(ids == ids[0]):
            stats.uniform_bricks += 1
            top[bi] = L.UNIFORM | int(ids[0])
            continue
        top[bi] = len(bricks)
        bricks.append((ids[0::2] | (ids[1::2] << 16)).astype(np.uint32))
        stats.bricks += 1
    stats.instances = len(model_rows) - 1
    models = np.zeros(len(model_rows), L.MODEL_DTYPE)
    models["quad_offset"] = [r[0] for r in model_rows]
    models["quad_count"] = [r[1] for r in model_rows]
    quads_arr = L.quads_array(quads) if quads else L.quads_array([np.zeros(20, np.uint32)])
    emitters, egrid = emitter_list(models, sites)
    stats.emitters = len(sites)
    top = top.astype(np.uint32)
    brick_words = np.concatenate(bricks) if bricks else np.zeros(0, np.uint32)
    ov_top = np.full(nb, L.EMPTY, np.uint32)
    off_bricks = nb
    off_ov_top = off_bricks + brick_words.size
    off_ov_cells = off_ov_top + nb
    off_ov_quads = off_ov_cells
    grid = np.concatenate([top, brick_words, ov_top, np.zeros(1, np.uint32)])
    n_real_quads = len(quads)
    sun = atlas.sprites["sun"]
    return HqScene(
        grid=grid, models=models, quads=quads_arr, atlas=atlas.pixels.ravel(), atlas_size=atlas.size,
        dims=dims, offsets=(0, off_bricks, off_ov_top, off_ov_cells, off_ov_quads),
        see_through=(n_real_quads, 0), emitters=emitters, emitter_count=len(sites), emitter_grid=egrid,
        sun_sprite=(sun.x, sun.y, sun.w, sun.h), stats=stats)
