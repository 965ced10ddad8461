"""CPU oracle of the coarse/fine interface lists of an AMR mesh (test
infrastructure only: nothing in the product imports this file).

The reference rebuilds its coarse/fine pairs incrementally inside every
regrid (AMR::PerformAdaptive, AMR.cpp:6-209): TagRefineGhost marks, around
each box it refines, the first restriction layer (tag 1: a box with an
unrefined box among its 27 neighbours), the second (tag 2: an unrefined box
two steps away along an axis) and the prolongation boxes (tag -2: unrefined
neighbours of refined boxes) (AMRGhost_refine.cpp:30-98); AdjustMesh and the
pair bookkeeping of AMRLevel.cpp / AMRGhost_*.cpp then keep the lists
f_res_ghost[0..1], f_pro_ghost and g_pro (AMRLevel.H:320-329) as the mesh
changes.  On the finished mesh those lists are a function of the leaf cells
of every level alone, which this module states (2-D, one block):

* refined(l): level-l positions whose sons exist on level l+1 as leaves or
  as refined positions (built from the finest level down);
* restriction pair of level l, layer 0: a refined position whose four sons
  are leaves and whose 8 in-plane neighbours include a leaf of level l;
  layer 1: not layer 0, four leaf sons, and a leaf of level l two steps away
  along x or y;
* prolongation pair of level l: a leaf of level l with a refined position
  among its 8 neighbours (sons: the four level-(l+1) positions below it);
* interface ghost cells of level l: the restriction positions of level l
  and the sons of the prolongation pairs of level l-1.

Pinned against the reference's own lists after regrids (tests/
test_oracle_interfaces.py runs the reference with regrids steered away from
the plain criterion and compares every pair list and ghost set).
"""
from __future__ import annotations

import numpy as np

AXIS2 = ((2, 0), (-2, 0), (0, 2), (0, -2))
NB8 = tuple((dx, dy) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if dx or dy)
SONS = ((0, 0), (0, 1), (1, 0), (1, 1))  # (x, y) offsets in the lists' son order


def interfaces(level, ix, iy, nlevels: int):
    """From the leaf cells (level, ix, iy): restriction pairs as rows (level,
    layer, cx, cy, 4 x (fx, fy)), prolongation pairs as rows (level, cx, cy,
    4 x (fx, fy)) and interface ghost cells (level, ix, iy), each sorted by
    (level, cy, cx) (int32 arrays)."""
    level, ix, iy = (np.asarray(a, np.int64) for a in (level, ix, iy))
    leaves = [set(zip(ix[level == l].tolist(), iy[level == l].tolist())) for l in range(nlevels)]
    refined = [set() for _ in range(nlevels)]
    for l in range(nlevels - 2, -1, -1):
        refined[l] = {(x >> 1, y >> 1) for (x, y) in leaves[l + 1] | refined[l + 1]}
    res, pro, ghost = [], [], []
    for l in range(nlevels - 1):
        for (cx, cy) in refined[l]:
            sons = [(2 * cx + a, 2 * cy + b) for a, b in SONS]
            if not all(s in leaves[l + 1] for s in sons):
                continue
            if any((cx + dx, cy + dy) in leaves[l] for dx, dy in NB8):
                layer = 0
            elif any((cx + dx, cy + dy) in leaves[l] for dx, dy in AXIS2):
                layer = 1
            else:
                continue
            res.append([l, layer, cx, cy] + [v for s in sons for v in s])
        for (cx, cy) in leaves[l]:
            if any((cx + dx, cy + dy) in refined[l] for dx, dy in NB8):
                pro.append([l, cx, cy] + [v for a, b in SONS for v in (2 * cx + a, 2 * cy + b)])
    for r in res:
        ghost.append([r[0], r[2], r[3]])
    for p in pro:
        for k in range(4):
            ghost.append([p[0] + 1, p[3 + 2 * k], p[4 + 2 * k]])

    def sort(rows, width, keys):
        a = np.array(rows, np.int32).reshape(-1, width)
        if len(a) == 0:
            return a
        return a[np.lexsort(tuple(a[:, k] for k in reversed(keys)))]

    ghost = np.unique(np.array(ghost, np.int32).reshape(-1, 3), axis=0)
    return (sort(res, 12, (0, 3, 2)), sort(pro, 11, (0, 2, 1)), sort(ghost, 3, (0, 2, 1)))


def reference_lists(d: dict):
    """The reference's own lists from a state dump (oracle/ref_driver.cpp):
    restriction rows (level, layer, cx, cy, sons), the set of prolongation
    rows (level, cx, cy, sons; the reference keeps f_pro_ghost and g_pro, the
    same pairs listed more than once) and the interface ghost cells (kind 3),
    sorted as ``interfaces`` sorts."""
    res = d["cf_res"].reshape(-1, 12)
    pro = d["cf_pro"].reshape(-1, 12)[:, [0, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11]]
    pro = np.unique(pro, axis=0)
    g = d["kind"] == 3
    ghost = np.stack([d["level"][g], d["ix"][g], d["iy"][g]], axis=1).astype(np.int32)

    def sort(a, keys):
        return a[np.lexsort(tuple(a[:, k] for k in reversed(keys)))] if len(a) else a

    return sort(res.astype(np.int32), (0, 3, 2)), sort(pro.astype(np.int32), (0, 2, 1)), \
        sort(np.unique(ghost, axis=0), (0, 2, 1))
