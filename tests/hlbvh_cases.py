"""Seeded HLBVH parity cases shared by the fixture script and the oracle test:
name -> (mesh maker, Morton bits, Morton SAH bits). Meshes are scaled into
[0, 1]^3 as the reference's scene loader does (rt/scene/SceneLoader.cpp:136-140)."""
import numpy as np

import hippie_b200 as hp


def _singleton():
    """A uniform mesh plus one triangle alone beyond its maximum corner: the last
    sorted key is a leaf cluster of its own."""
    v, t = hp.gen.uniform_mesh(5, 400)
    lo, hi = v.min(0), v.max(0)
    far = hi + 0.5 * (hi - lo) + np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.01, 0]], np.float32)
    v = np.concatenate([v, far.astype(np.float32)])
    t = np.concatenate([t, np.array([[len(v) - 3, len(v) - 2, len(v) - 1]], np.int32)])
    return v, t


CASES = {
    "uniform_15": (lambda: hp.gen.uniform_mesh(91, 3000), 60, 15),
    "clustered_9": (lambda: hp.gen.clustered_mesh(92, 4000, 16, 0.05, 0.01), 60, 9),
    "clustered_6": (lambda: hp.gen.clustered_mesh(93, 2500, 8, 0.05, 0.01), 60, 6),
    "uniform_12_bits30": (lambda: hp.gen.uniform_mesh(94, 5000), 30, 12),
    "singleton_15": (_singleton, 60, 15),
}


def mesh(name):
    v, t = CASES[name][0]()
    lo, hi = v.min(0), v.max(0)
    return ((v - lo) / (hi - lo).max()).astype(np.float32), np.ascontiguousarray(t, np.int32)


def canonical(nodes, tri_idx, sorted_tri=None):
    """Depth-first structure of a binary BVH (boxes, sizes, leaf triangle sets).

    With sorted_tri (the Morton order), the node whose children are the
    single-triangle leaf of the last sorted triangle and the subtree holding the
    first one is written with the first one's side on the left: the reference
    orders that pair, its object-median fallback, by atomic arrival."""
    first = last = None
    if sorted_tri is not None:
        first, last = int(sorted_tri[0]), int(sorted_tri[-1])
    holds_first = set()
    if first is not None:
        parent = {}
        for i in range(nodes.shape[0]):
            c0, c1, size, _ = nodes[i, 12:16]
            if size >= 0:
                parent[~c0 if c0 < 0 else c0] = i
                parent[~c1 if c1 < 0 else c1] = i
        for i in range(nodes.shape[0]):
            c0, c1, size, _ = nodes[i, 12:16]
            if size < 0 and first in tri_idx[c0:c1].tolist():
                j = i
                while j in parent or j == 0:
                    holds_first.add(j)
                    if j == 0:
                        break
                    j = parent[j]
                break

    def is_last_leaf(i):
        c0, c1, size, _ = nodes[i, 12:16]
        return size < 0 and c1 - c0 == 1 and int(tri_idx[c0]) == last

    out = []
    stack = [0]
    while stack:
        if len(out) > nodes.shape[0]:
            raise AssertionError("a node is reached twice: not a tree")
        i = stack.pop()
        c0, c1, size, _ = nodes[i, 12:16]
        if size < 0:
            out.append(("L", tuple(nodes[i, :12].tolist()), tuple(sorted(tri_idx[c0:c1].tolist()))))
            continue
        a, b = (~c0 if c0 < 0 else c0), (~c1 if c1 < 0 else c1)
        box = nodes[i, :12].tolist()
        if first is not None and is_last_leaf(a) and b in holds_first:
            a, b = b, a
            box = box[4:8] + box[0:4] + box[10:12] + box[8:10]
        out.append(("I", tuple(box), int(size)))
        stack.append(b)
        stack.append(a)
    return out
