"""Plain restatement of the reference's hq grid build, for the bit-exact check of the product's.

TEST INFRASTRUCTURE (see oracle/oracle.py). Follows, loop for loop:
  `build_hq`      crates/lumenwright/src/scene/voxel.rs:111-491
  `add_instance`  voxel.rs:494-528
  `emitter_list`  voxel.rs:542-607
  `fluid_face_mask` crates/lumenwright/src/scene/mod.rs:586-609
over a block volume of the synthetic block set, whose block models (`Scene::block_quads`) come
from ``lumenwright_b200.synth`` (the scene side the reference reads from its jar). Per-voxel
Python loops: meant for worlds of a few chunks.
"""

import numpy as np

from lumenwright_b200 import layout as L
from lumenwright_b200 import synth as S

EMITTER_CELL = 10
DIRS = [S.DOWN, S.UP, S.NORTH, S.SOUTH, S.WEST, S.EAST]  # Dir::ALL


def build_hq_ref(world, atlas):
    b = world.blocks
    Y, Z, X = b.shape
    cx, sy, cz = X // 16, Y // 16, Z // 16
    nb = cx * sy * cz
    blocks = S.BLOCKS

    def block(x, y, z):
        if 0 <= x < X and 0 <= y < Y and 0 <= z < Z:
            return int(b[y, z, x])
        return S.AIR

    def brick_xyz(i):  # voxel.rs:132-139
        return (i % cx, i // (cx * cz), (i // cx) % cz)

    def brick_index(bb):  # voxel.rs:140-150
        if min(bb) < 0 or bb[0] >= cx or bb[1] >= sy or bb[2] >= cz:
            return None
        return (bb[1] * cz + bb[2]) * cx + bb[0]

    def section(i):
        bx, by, bz = brick_xyz(i)
        return b[by * 16:(by + 1) * 16, bz * 16:(bz + 1) * 16, bx * 16:(bx + 1) * 16]

    # Phase 0 (voxel.rs:119-131).
    all_occluding = []
    for i in range(nb):
        s = section(i)
        if not s.any():
            all_occluding.append(False)
        else:
            all_occluding.append(all(blocks[int(p)].occludes for p in set(s.ravel().tolist())))

    def fluid_face_mask(pos):  # scene/mod.rs:586-609, water
        x, y, z = pos
        same = lambda o: block(x + o[0], y + o[1], z + o[2]) == S.WATER  # noqa: E731
        occl = lambda o: blocks[block(x + o[0], y + o[1], z + o[2])].occludes  # noqa: E731
        mask = 0
        if same((0, 1, 0)):
            mask |= 0x80 | (1 << S.UP)
        for d in (S.DOWN, S.NORTH, S.SOUTH, S.WEST, S.EAST):
            o = S.DIR_OFFSET[d]
            if same(o) or occl(o):
                mask |= 1 << d
        return mask

    # Phase 1 (voxel.rs:171-260).
    keyed = []
    for bi in range(nb):
        s = section(bi)
        if not s.any():
            keyed.append(None)
            continue
        bx, by, bz = brick_xyz(bi)
        local, keys, ids = {}, [], [0] * 4096
        for ly in range(16):
            for lz in range(16):
                for lx in range(16):
                    sid = int(s[ly, lz, lx])
                    info = blocks[sid]
                    if sid == 0 or info.invisible:
                        continue
                    pos = (bx * 16 + lx, by * 16 + ly, bz * 16 + lz)
                    if info.simple:
                        key = (sid, (0xFFFFFFFF,) * 8, 0, 0, 0)
                    else:
                        models = (0xFFFFFFFF,) * 8 if info.fluid else (sid,) + (0xFFFFFFFF,) * 7
                        fm = fluid_face_mask(pos) if info.fluid else 0
                        tint_pos = 0  # one biome
                        key = (sid, models, tint_pos, 0, fm)
                    if key not in local:
                        keys.append((key, pos))
                        local[key] = len(keys)
                    ids[(ly * 16 + lz) * 16 + lx] = local[key]
        keyed.append((keys, ids))

    # Phase 2 (voxel.rs:262-343).
    models = [(0, 0)]
    quads = []
    model_emits = [False]
    instance_ids = {}
    top = [L.EMPTY] * nb
    bricks = []
    sites = []
    for bi, sk in enumerate(keyed):
        if sk is None or not sk[0]:
            continue
        keys, lids = sk
        mp = [0] * (len(keys) + 1)
        for i, (key, pos) in enumerate(keys):
            if key in instance_ids:
                mp[i + 1] = instance_ids[key]
            else:
                qs = S.block_quads(atlas, key[0], key[4])  # add_instance (voxel.rs:494-528)
                off = len(quads)
                for q in qs:
                    q = np.array(q, np.uint32)
                    if not (int(q[3]) & L.FLAG_WATER):
                        q[3] = int(q[3]) | L.FLAG_FRONT_ONLY
                    quads.append(q)
                model_emits.append(len(qs) > 0 and blocks[key[0]].emittance > 0.0)
                models.append((off, len(qs)))
                iid = len(models) - 1
                instance_ids[key] = iid
                mp[i + 1] = iid
        ids = [mp[l] for l in lids]
        bx, by, bz = brick_xyz(bi)
        buried = all_occluding[bi]
        if buried:
            for d in DIRS:
                o = S.DIR_OFFSET[d]
                n = brick_index((bx + o[0], by + o[1], bz + o[2]))
                if n is None or not all_occluding[n]:
                    buried = False
                    break
        for loc, iid in enumerate(ids):
            if model_emits[iid]:
                sites.append(((bx * 16 + (loc & 15), by * 16 + (loc >> 8), bz * 16 + ((loc >> 4) & 15)), iid))
        if buried:
            nz = [i for i in ids if i != 0]
            top[bi] = L.UNIFORM | (nz[0] if nz else 1)
            continue
        if all(i == ids[0] for i in ids):
            top[bi] = L.UNIFORM | ids[0]
            continue
        top[bi] = len(bricks) // L.BRICK_WORDS
        for k in range(0, 4096, 2):
            bricks.append(ids[k] | (ids[k + 1] << 16))

    emitters, egrid = emitter_list_ref(models, sites)
    grid = top + bricks + [L.EMPTY] * nb + [0]
    return dict(grid=np.array(grid, np.uint32), models=models, quads=quads, emitters=emitters,
                emitter_grid=np.array(egrid, np.uint32), offsets=(0, nb, nb + len(bricks), 2 * nb + len(bricks),
                                                               2 * nb + len(bricks)))


def emitter_list_ref(models, sites):
    """voxel.rs:542-607."""
    if not sites:
        return [], [EMITTER_CELL] + [0] * 7
    emitters = [(c, models[m][0], models[m][1]) for c, m in sites]
    cell_of = lambda c: tuple(v // EMITTER_CELL for v in c)  # noqa: E731  (div_euclid)
    lo = [min(cell_of(c)[a] for c, _ in sites) for a in range(3)]
    hi = [max(cell_of(c)[a] for c, _ in sites) for a in range(3)]
    offset = [v - 1 for v in lo]
    size = [hi[a] - lo[a] + 3 for a in range(3)]

    def index(g):
        l = [g[a] - offset[a] for a in range(3)]
        return (l[1] * size[2] + l[2]) * size[0] + l[0]

    cells = [[] for _ in range(size[0] * size[1] * size[2])]
    for i, (c, _) in enumerate(sites):
        g = cell_of(c)
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    cells[index((g[0] + dx, g[1] + dy, g[2] + dz))].append(i)
    grid = [EMITTER_CELL, size[0], size[1], size[2]] + [v & 0xFFFFFFFF for v in offset] + [0]
    lst = []
    for c in cells:
        grid += [len(lst), len(c)]
        lst += c
    return emitters, grid + lst
