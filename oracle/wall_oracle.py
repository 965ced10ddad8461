"""CPU restatement of the reference's wall-distance passes for moved bodies
(test infrastructure only: nothing in the product imports this file).

Follows Body::RenewLevelDistance (Bodymove.cpp:127-300) for one level:

1. every box closer than 9.5 to a wall and not a block ghost walks from its
   current patch to the closest patch of its body (Body::FindClosePatchtoCell,
   Body.H:505-542, with PatchDistoBox, Body.H:563-580: a neighbour is taken
   when strictly closer; the walk ends at a patch none of whose neighbours
   is closer), its signed distance the patch normal dotted with
   centre - patch centre (PeriodicLength, mpiparams.cpp:294-310, on y);
2. boxes with an in-plane neighbour paired with another body (the
   neighbours' pairs after step 1, in Point_iterator_2d order) try that body
   from the neighbour's patch and switch by the reference's rule
   (Bodymove.cpp:158-228);
3. the signed distance is capped by the distance to the domain boundary,
   the solid flag follows its sign, and boxes that changed sides (domain
   ghosts excepted) go to the move lists in box order (Bodymove.cpp:231-255);

then Mesh::SynNormal_BlockDistance's block pairs (Mesh.cpp:2303-2374): each
block ghost takes its origin's body, patch, distance and signed distance,
with its solid flag and move-list entry.  Python floats are IEEE doubles
evaluated left to right, math.sqrt is correctly rounded: the results are
the reference's bit for bit.  Pinned against the reference itself through
the binding (tests/test_gpu_pitch.py compares the device passes with the
reference's own at every step of a pitching run); here the device passes are
checked against this restatement on seeded synthetic bodies and boxes.
"""
from __future__ import annotations

import math

import numpy as np

CRITIC = 9.5
FAR = 999.0
OTHER, DOMAIN_GHOST, BLOCK_GHOST = 0, 1, 2
INTO, OUT = 1, 2


def _dy(bodies, dy):
    c = bodies.get("critic_ylength", 1e300)
    if abs(dy) > c and bodies.get("periodic_y", 0):
        if dy > c:
            dy -= bodies["dm_length_y"]
        elif dy < -c:
            dy += bodies["dm_length_y"]
    return dy


def _dist(bodies, r, c):
    pc = bodies["pc"][r]
    dx = float(c[0]) - float(pc[0])
    dy = _dy(bodies, float(c[1]) - float(pc[1]))
    dz = float(c[2]) - float(pc[2])
    return math.sqrt(dx * dx + dy * dy + dz * dz)


def find_close(bodies, b, p, c):
    """(patch, distance, signed distance) of centre c walking body b from p."""
    base = int(bodies["patch_start"][b])
    best, bp = FAR, p
    d = _dist(bodies, base + p, c)
    if d < best:
        best = d
    old, ps0 = -1, bp
    while old != ps0:
        old = bp
        row = base + ps0
        for k in range(int(bodies["nb_count"][row])):
            q = int(bodies["nb"][row][k])
            d = _dist(bodies, base + q, c)
            if d < best:
                best, bp = d, q
        ps0 = bp
    r = base + bp
    pc, nv = bodies["pc"][r], bodies["nv"][r]
    dx = float(c[0]) - float(pc[0])
    dy = _dy(bodies, float(c[1]) - float(pc[1]))
    dz = float(c[2]) - float(pc[2])
    sd = float(nv[0]) * dx + float(nv[1]) * dy + float(nv[2]) * dz
    return bp, best, sd


def wall_distance(bodies, geom, pairs):
    """One level: geom (center, neib, kind, distance_to_dm, block_in,
    block_out), pairs (body, patch, distance, signdis, distance_to_body,
    solid); returns the new pairs with moved (per box) and block_moved."""
    n = len(geom["kind"])
    kind = np.asarray(geom["kind"])
    center = np.asarray(geom["center"], np.float64).reshape(-1, 3)
    neib = np.asarray(geom["neib"]).reshape(-1, 9)
    body = [int(v) for v in pairs["body"]]
    patch = [int(v) for v in pairs["patch"]]
    dist = [float(v) for v in pairs["distance"]]
    sd = [float(v) for v in pairs["signdis"]]
    dtb = [float(v) for v in pairs["distance_to_body"]]
    solid = [int(v) for v in pairs["solid"]]
    # 1. the walk
    for i in range(n):
        if sd[i] < CRITIC and kind[i] != BLOCK_GHOST:
            patch[i], dist[i], sd[i] = find_close(bodies, body[i], patch[i], center[i])
            dtb[i] = sd[i]
    # 2. junctions, from the walked pairs
    body1, patch1 = list(body), list(patch)
    for i in range(n):
        if not (sd[i] < CRITIC and kind[i] != BLOCK_GHOST):
            continue
        for k in range(9):
            an = int(neib[i][k])
            if an < 0 or body1[an] == body1[i]:
                continue
            cb, cp = body1[an], patch1[an]
            if body[i] == cb:
                continue
            np_, nd, nsd = find_close(bodies, cb, cp, center[i])
            change = False
            if nsd > 0.0 and sd[i] < 0.0:
                change = True
            elif nd < dist[i]:
                if sd[i] * nsd > 0.0 or nsd > 0.0:
                    change = True
            if change:
                body[i], patch[i], dist[i], sd[i], dtb[i] = cb, np_, nd, nsd, nsd
    # 3. caps, solid flags, move lists
    moved = [0] * n
    dm = np.asarray(geom["distance_to_dm"], np.float64)
    for i in range(n):
        if sd[i] < CRITIC and kind[i] != BLOCK_GHOST:
            sd[i] = float(dm[i]) if float(dm[i]) < sd[i] else sd[i]
            if sd[i] < 0.0:
                if not solid[i] and kind[i] != DOMAIN_GHOST:
                    moved[i] = INTO
                solid[i] = 1
            else:
                if solid[i] and kind[i] != DOMAIN_GHOST:
                    moved[i] = OUT
                solid[i] = 0
    # block ghosts
    bi = [int(v) for v in geom.get("block_in", [])]
    bo = [int(v) for v in geom.get("block_out", [])]
    block_moved = [0] * len(bi)
    for k, (a, o) in enumerate(zip(bi, bo)):
        body[o], patch[o], dist[o], sd[o] = body[a], patch[a], dist[a], sd[a]
        if sd[o] < 0.0:
            if not solid[o] and kind[o] != DOMAIN_GHOST:
                block_moved[k] = INTO
            solid[o] = 1
        else:
            if solid[o] and kind[o] != DOMAIN_GHOST:
                block_moved[k] = OUT
            solid[o] = 0
    return dict(body=np.array(body, np.int32), patch=np.array(patch, np.int32),
                distance=np.array(dist), signdis=np.array(sd), distance_to_body=np.array(dtb),
                solid=np.array(solid, np.uint8), moved=np.array(moved, np.uint8),
                block_moved=np.array(block_moved, np.uint8))


def synthetic_case(seed: int = 0, nx: int = 48, ny: int = 40, npts: int = 60, turn: float = 0.02):
    """Two bodies (upper and lower half of an ellipse, as the two surfaces of
    an airfoil), a grid of boxes around them with pairs found for the body
    before it turned by `turn` radians, a few domain ghosts along the
    border and block pairs along one side."""
    rng = np.random.default_rng(seed)

    def surface(angle):
        bodies = {"patch_start": [0], "pc": [], "nv": [], "nb_count": [], "nb": []}
        for b, (a0, a1) in enumerate(((0.0, math.pi), (math.pi, 2 * math.pi))):
            t = np.linspace(a0, a1, npts, endpoint=False) + (a1 - a0) / npts / 2
            x, y = 1.2 * np.cos(t), 0.35 * np.sin(t)
            nx_, ny_ = np.cos(t) / 1.2, np.sin(t) / 0.35
            ln = np.hypot(nx_, ny_)
            ca, sa = math.cos(angle), math.sin(angle)
            for j in range(npts):
                px, py = x[j] * ca - y[j] * sa + 2.5, x[j] * sa + y[j] * ca + 2.0
                vx, vy = (nx_[j] * ca - ny_[j] * sa) / ln[j], (nx_[j] * sa + ny_[j] * ca) / ln[j]
                bodies["pc"].append([px, py, 0.05])
                bodies["nv"].append([vx, vy, 0.0])
                nbs = [q for q in (j - 2, j - 1, j + 1, j + 2) if 0 <= q < npts]
                bodies["nb_count"].append(len(nbs))
                bodies["nb"].append(nbs + [-1] * (15 - len(nbs)))
            bodies["patch_start"].append(bodies["patch_start"][-1] + npts)
        for k in bodies:
            bodies[k] = np.array(bodies[k])
        return bodies

    old, new = surface(0.0), surface(turn)
    h = 5.0 / nx
    xs = (np.arange(nx) + 0.5) * h
    ys = (np.arange(ny) + 0.5) * h
    cx, cy = np.meshgrid(xs, ys)
    center = np.stack([cx.ravel(), cy.ravel(), np.full(cx.size, 0.05)], axis=1)
    n = len(center)
    neib = np.full((n, 9), -1, np.int32)
    for i in range(n):
        ix, iy = i % nx, i // nx
        for a in range(3):
            for b in range(3):
                jx, jy = ix + a - 1, iy + b - 1
                if 0 <= jx < nx and 0 <= jy < ny:
                    neib[i, 3 * a + b] = jy * nx + jx
    kind = np.zeros(n, np.uint8)
    border = (cx.ravel() < h) | (cy.ravel() < h) | (cy.ravel() > ys[-1] - h)
    kind[border] = DOMAIN_GHOST
    right = np.flatnonzero(cx.ravel() > xs[-1] - h)
    kind[right] = BLOCK_GHOST
    block_out = right.astype(np.int32)
    block_in = (right - nx // 2).astype(np.int32)  # boxes well inside
    dm = np.minimum.reduce([cx.ravel(), cy.ravel(), 5.0 - cx.ravel(), ys[-1] + h / 2 - cy.ravel()])
    # pairs for the old position: closest patch of the closer body, found by
    # a full scan (the state the reference's previous move left)
    body = np.zeros(n, np.int32)
    patch = np.zeros(n, np.int32)
    dist = np.zeros(n)
    sd = np.zeros(n)
    for i in range(n):
        d = np.hypot(*(old["pc"][:, :2] - center[i, :2]).T)
        r = int(np.argmin(d))
        b = 0 if r < npts else 1
        body[i], patch[i], dist[i] = b, r - old["patch_start"][b], d[r]
        sd[i] = float(np.dot(old["nv"][r], center[i] - old["pc"][r]))
    sd = np.minimum(sd, dm)
    far = rng.random(n) < 0.05  # a few boxes beyond the 9.5 band keep their pairs
    sd[far] = 20.0
    solid = (sd < 0.0).astype(np.uint8)
    geom = dict(center=center, neib=neib, kind=kind, distance_to_dm=dm, block_in=block_in,
                block_out=block_out)
    pairs = dict(body=body, patch=patch, distance=dist, signdis=sd, distance_to_body=sd.copy(),
                 solid=solid, nblock=len(block_in))
    return new, geom, pairs
