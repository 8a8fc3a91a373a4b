"""The compressed eight-wide BVH, on the host (rtg_host_scene_layout: the layout a
scene gets at upload, computed without a GPU).

Checks, for the benchmark scenes, mix scenes and builder edge cases:
  * every quantised child box, decoded exactly, encloses the fp32 boxes the
    binary tree stores for the leaves beneath that child (so the eight-wide walk
    culls nothing the binary walk would visit);
  * the leaves of the eight-wide tree cover every primitive slot exactly once, a
    leaf's slots end at its last-in-leaf mark, and the binary and four-wide trees
    still reach the same leaves after the slots were reordered;
  * the slot -> primitive map is a permutation and the slot records moved with it;
  * a restatement of the kernel's walk (groups of children visited in slot XOR
    octant order, leaves tested at once) finds the same hits as a brute-force
    loop over the slots, in float32, on random rays.
"""
import json

import numpy as np
import pytest

import rtg
import workloads

LAST = 0x40000000
SPHERE = 0x80000000


def _scene(objects, planes=()):
    return {"materials": {"m": {"type": "lambertian"}}, "objects": list(planes) + list(objects)}


def _spheres(centres, r=0.3):
    return [{"type": "sphere", "center": [float(x) for x in c], "radius": r, "material": "m"} for c in centres]


def _chains(n, length, rng):
    """Clusters of nearly coincident spheres: deep trees and long leaves."""
    base = rng.uniform(-5, 5, (n, 3))
    return np.concatenate([b + np.arange(length)[:, None] * 1e-7 for b in base])


_rng = np.random.default_rng(7)
SCENES = {
    "cornell": workloads.cornell(),
    "spheres": workloads.sphere_field(),
    "mesh": workloads.mesh_stress(),
    "mix_4": workloads.mix_scene(4),
    "mix_9": workloads.mix_scene(9),
    "one_sphere": _scene(_spheres([[0, 0, 0]])),
    "nine_spheres": _scene(_spheres(_rng.uniform(-3, 3, (9, 3)))),
    "planes_only": _scene([], [{"type": "plane", "point": [0, 0, 0], "normal": [0, 1, 0], "material": "m"}]),
    "coincident_chains": _scene(_spheres(_chains(30, 40, _rng), r=0.1)),
    "identical_spheres": _scene(_spheres(np.zeros((300, 3)) + 0.5, r=0.5)),
}


def _words_to_bytes(words):
    return np.ascontiguousarray(words, dtype="<u4").view(np.uint8).reshape(len(words), -1)


def decode(n8):
    """Per node: origin p (3), scale (3), imask, child_base, prim_base, meta[8],
    decoded child boxes lo/hi (8 x 3, float64, exact)."""
    n8 = np.asarray(n8, dtype=np.uint32)
    p = n8[:, 0:3].view(np.float32).astype(np.float64)
    ew = n8[:, 3]
    e = np.stack([(ew >> (8 * k)) & 0xFF for k in range(3)], 1).astype(np.int64)
    scale = np.ldexp(1.0, e - 127)
    imask = (ew >> 24) & 0xFF
    child_base, prim_base = n8[:, 4], n8[:, 5]
    meta = _words_to_bytes(n8[:, 6:8])
    q = _words_to_bytes(n8[:, 8:20]).reshape(-1, 6, 8).astype(np.float64)  # lo x,y,z then hi x,y,z
    lo = p[:, None, :] + scale[:, None, :] * np.moveaxis(q[:, 0:3, :], 1, 2)
    hi = p[:, None, :] + scale[:, None, :] * np.moveaxis(q[:, 3:6, :], 1, 2)
    used = ~((q[:, 0:3, :] == 255).all(1) & (q[:, 3:6, :] == 0).all(1))
    return dict(p=p, scale=scale, imask=imask, child_base=child_base, prim_base=prim_base, meta=meta, lo=lo, hi=hi,
                used=used)


def leaf_slots(first, word):
    k = first
    while not (word[k] & LAST):
        k += 1
    return list(range(first, k + 1))


def walk_leaves(d, root, word):
    """(node, slot) -> slots under that child, and every leaf's slot list."""
    under = {}
    leaves = []

    def visit(node):
        out = []
        for s in range(8):
            if not d["used"][node, s]:
                continue
            if (d["imask"][node] >> s) & 1:
                idx = int(d["child_base"][node]) + bin(int(d["imask"][node]) & ((1 << s) - 1)).count("1")
                got = visit(idx)
            else:
                got = leaf_slots(int(d["prim_base"][node]) + int(d["meta"][node, s]), word)
                leaves.append(got)
            under[(node, s)] = got
            out += got
        return out

    visit(root)
    return under, leaves


@pytest.mark.parametrize("name", list(SCENES))
def test_wide8_layout_invariants(name):
    host = rtg.parse_scene(json.dumps(SCENES[name]))
    roots = host.device_layout("roots")[0]
    root, root4, n_slots, root8 = int(roots[0]), int(roots[1]), int(roots[2]), int(roots[4])
    prims = host.device_layout("prims")
    slot_prim = host.device_layout("slot_prim").reshape(-1)
    assert len(slot_prim) == n_slots and len(set(slot_prim.tolist())) == n_slots
    word = np.asarray(prims, np.float32).reshape(-1, 3, 4)[:, 0, 3].view(np.uint32)
    assert np.array_equal(word & 0x3FFFFFFF, slot_prim)  # the records moved with the map
    n8 = host.device_layout("nodes8")
    if n_slots == 0:
        assert root8 == -2 ** 31 and len(n8) == 0
        return
    if root8 < 0:
        assert len(n8) == 0 and leaf_slots(~root8, word) == list(range(n_slots))
        return
    d = decode(n8)
    under, leaves = walk_leaves(d, root8, word)
    covered = sorted(s for leaf in leaves for s in leaf)
    assert covered == list(range(n_slots))
    # The fp32 box of every binary leaf, as its binary parent stores it: what the
    # eight-wide boxes are quantised from and must enclose.
    nodes_f = host.device_layout("nodes").reshape(-1, 16)
    links_b = nodes_f.view(np.int32)[:, 12:14]
    leaf_lo, leaf_hi = {}, {}
    for i in range(len(nodes_f)):
        f = nodes_f[i]
        boxes = [((f[0], f[2], f[8]), (f[1], f[3], f[9])), ((f[4], f[6], f[10]), (f[5], f[7], f[11]))]
        for c in range(2):
            if links_b[i, c] < 0:
                leaf_lo[~int(links_b[i, c])] = np.array(boxes[c][0], np.float64)
                leaf_hi[~int(links_b[i, c])] = np.array(boxes[c][1], np.float64)
    for (node, s), slots in under.items():
        starts = [k for k in slots if k in leaf_lo]
        blo = np.min([leaf_lo[k] for k in starts], 0)
        bhi = np.max([leaf_hi[k] for k in starts], 0)
        assert (d["lo"][node, s] <= blo).all() and (d["hi"][node, s] >= bhi).all(), (node, s)
    # The binary and four-wide trees reach the same leaves (links moved with the slots).
    leaf_starts = {leaf[0] for leaf in leaves}
    assert set(leaf_lo) == leaf_starts
    nodes = host.device_layout("nodes").view(np.int32)
    links = np.concatenate([nodes[:, 12:14].reshape(-1), host.device_layout("nodes4").view(np.int32)[:, 24:28].reshape(-1),
                            [root, root4]])
    starts = {~int(x) for x in links if x < 0 and x != -2 ** 31}
    assert starts == leaf_starts


def _tri_hit(o, dvec, v0, e1, e2, tmin, tmax):
    pv = np.cross(dvec, e2)
    det = np.dot(e1, pv)
    if abs(det) < 1e-14:
        return None
    inv = np.float32(1) / det
    tv = o - v0
    u = np.dot(tv, pv) * inv
    if u < -1e-6 or u > 1 + 1e-6:
        return None
    qv = np.cross(tv, e1)
    v = np.dot(dvec, qv) * inv
    if v < -1e-6 or u + v > 1 + 1e-6:
        return None
    t = np.dot(e2, qv) * inv
    return t if tmin < t < tmax else None


def _sphere_hit(o, dvec, c, r, tmin, tmax):
    oc = c - o
    a = np.dot(dvec, dvec)
    h = np.dot(dvec, oc)
    cc = np.dot(oc, oc) - r * r
    perp = oc - (h / a) * dvec
    disc = a * (r * r - np.dot(perp, perp))
    if disc < 0:
        return None
    q = h + np.copysign(np.sqrt(disc), h)
    t0, t1 = (cc / q, q / a) if q != 0 else (h / a, h / a)
    t0, t1 = min(t0, t1), max(t0, t1)
    for t in (t0, t1):
        if tmin < t < tmax:
            return t
    return None


def _test_slot(rows, k, o, dvec, tmin, tmax):
    w = rows[k, 0, 3:4].view(np.uint32)[0]
    if w & SPHERE:
        return _sphere_hit(o, dvec, rows[k, 0, :3], rows[k, 1, 0], tmin, tmax)
    return _tri_hit(o, dvec, rows[k, 0, :3], rows[k, 1, :3], rows[k, 2, :3], tmin, tmax)


def walk8(d, root8, rows, word, o, dvec, tmin=np.float32(1e-6)):
    """The kernel's closest-hit walk, restated: a group is (child_base, imask,
    visit bits); a ray visits slot pos ^ octant for visit positions in order."""
    inv = np.float32(1) / np.where(np.abs(dvec) < 1e-20, np.copysign(np.float32(1e-20), dvec), dvec)
    oct_ = int(inv[0] < 0) | int(inv[1] < 0) << 1 | int(inv[2] < 0) << 2
    best_t, best = np.float32(3e38), -1
    stack = [(root8, (1 << oct_) | (1 << 8))]
    while stack:
        base, mask = stack.pop()
        while mask & 0xFF:
            pos = (mask & -mask).bit_length() - 1
            mask &= ~(1 << pos)
            slot = pos ^ oct_
            node = base + bin((mask >> 8) & ((1 << slot) - 1)).count("1")
            if mask & 0xFF:
                stack.append((base, mask))
            lo = ((d["lo"][node] - o) * inv).astype(np.float32)
            hi = ((d["hi"][node] - o) * inv).astype(np.float32)
            tn = np.maximum(np.minimum(lo, hi).max(1), tmin)
            tf = np.minimum(np.maximum(lo, hi).min(1), best_t)
            hit = (tn <= tf) & d["used"][node]
            inner = leaves = 0
            for j in range(8):
                if hit[j]:
                    if (d["imask"][node] >> j) & 1:
                        inner |= 1 << (j ^ oct_)
                    else:
                        leaves |= 1 << (j ^ oct_)
            while leaves:
                lp = (leaves & -leaves).bit_length() - 1
                leaves &= leaves - 1
                ls = lp ^ oct_
                for k in leaf_slots(int(d["prim_base"][node]) + int(d["meta"][node, ls]), word):
                    t = _test_slot(rows, k, o, dvec, tmin, best_t)
                    if t is not None:
                        best_t, best = np.float32(t), k
            base, mask = int(d["child_base"][node]), inner | (int(d["imask"][node]) << 8)
    return best, best_t


@pytest.mark.parametrize("name", ["cornell", "nine_spheres", "mix_4"])
def test_restated_walk_matches_brute_force(name):
    host = rtg.parse_scene(json.dumps(SCENES[name]))
    root8 = int(host.device_layout("roots")[0][4])
    rows = host.device_layout("prims").reshape(-1, 3, 4).astype(np.float32)
    word = rows[:, 0, 3].view(np.uint32)
    d = decode(host.device_layout("nodes8"))
    rays = workloads.random_rays(host.view(), 150, seed=5)
    for r in rays:
        o, dvec = r[0:3].astype(np.float32), r[4:7].astype(np.float32)
        best, bt = walk8(d, root8, rows, word, o, dvec)
        bb, bbt = -1, np.float32(3e38)
        for k in range(len(rows)):
            t = _test_slot(rows, k, o, dvec, np.float32(1e-6), bbt)
            if t is not None:
                bb, bbt = k, np.float32(t)
        assert (best < 0) == (bb < 0)
        if best >= 0:
            assert best == bb or abs(bt - bbt) <= 1e-6 * abs(bbt), (best, bb, bt, bbt)
