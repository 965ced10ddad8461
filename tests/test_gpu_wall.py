"""Wall distances of moved bodies on the device (ibgpu_wall_geometry /
ibgpu_wall_distance, csrc/wall.cu) against the CPU restatement of the
reference's passes (oracle/wall_oracle.py: Body::RenewLevelDistance,
Bodymove.cpp:127-300, with Mesh::SynNormal_BlockDistance's block pairs) on
seeded synthetic bodies and boxes, bit for bit: pairs, signed distances,
solid flags and the move lists' entries.  Against the reference itself the
same device passes are compared at every step of a pitching run through the
binding (tests/test_gpu_pitch.py)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import wall_oracle as wo  # noqa: E402
from conftest import load_pkg  # noqa: E402

pytestmark = pytest.mark.gpu
wl = load_pkg().workloads


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else a


@pytest.mark.parametrize("seed,turn", [(0, 0.02), (3, 0.25), (5, 0.6)])
def test_device_passes_equal_the_reference_restatement(cuda_lib, pkg, seed, turn):
    bodies, geom, pairs = wo.synthetic_case(seed=seed, turn=turn)
    ref = wo.wall_distance(bodies, geom, pairs)
    P, cells, prim = wl.vortex_case(32)
    sol = pkg.ibgpu.FlowSolver(P)
    # two levels: the same boxes twice, the second with no block pairs
    g2 = dict(geom, block_in=[], block_out=[])
    sol.wall_geometry([geom, g2])
    p1 = {k: np.array(v, copy=True) for k, v in pairs.items() if k != "nblock"}
    p1["nblock"] = pairs["nblock"]
    p2 = {k: np.array(v, copy=True) for k, v in pairs.items() if k != "nblock"}
    got = sol.wall_distance(bodies, [p1, p2])
    for k in ("body", "patch", "distance", "signdis", "distance_to_body", "solid", "moved",
              "block_moved"):
        assert np.array_equal(bits(got[0][k]), bits(ref[k])), k
    ref2 = wo.wall_distance(bodies, g2, pairs)
    for k in ("body", "patch", "distance", "signdis", "solid", "moved"):
        assert np.array_equal(bits(got[1][k]), bits(ref2[k])), k
    assert (got[0]["moved"] > 0).any()
    sol.close()


def test_resident_pairs_continue_from_the_previous_call(cuda_lib, pkg):
    """Two moves: the second starts from the pairs the device kept (its
    input arrays hold garbage) and equals the restatement applied twice."""
    bodies1, geom, pairs = wo.synthetic_case(seed=4, turn=0.05)
    bodies2, _, _ = wo.synthetic_case(seed=4, turn=0.15)
    ref1 = wo.wall_distance(bodies1, geom, pairs)
    ref2 = wo.wall_distance(bodies2, geom, dict(ref1, nblock=pairs["nblock"]))
    P, cells, prim = wl.vortex_case(32)
    ib = pkg.ibgpu
    sol = ib.FlowSolver(P)
    sol.wall_geometry([geom])
    p = {k: np.array(v, copy=True) for k, v in pairs.items() if k != "nblock"}
    p["nblock"] = pairs["nblock"]
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_distance(bodies1, [dict(p)], resident=True)  # nothing kept yet
    assert e.value.code == ib.E_STATE
    sol.wall_distance(bodies1, [p])
    for k in ("body", "patch", "distance", "signdis"):
        p[k] = np.full_like(p[k], -7)
    got = sol.wall_distance(bodies2, [p], resident=True)[0]
    for k in ("body", "patch", "distance", "signdis", "distance_to_body", "solid", "moved",
              "block_moved"):
        assert np.array_equal(bits(got[k]), bits(ref2[k])), k
    sol.close()


def test_invalid_pairs_and_geometry_are_reported(cuda_lib, pkg):
    ib = pkg.ibgpu
    bodies, geom, pairs = wo.synthetic_case(seed=1)
    P, cells, prim = wl.vortex_case(32)
    sol = ib.FlowSolver(P)
    p = {k: np.array(v, copy=True) for k, v in pairs.items() if k != "nblock"}
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_distance(bodies, [p])  # before the geometry
    assert e.value.code == ib.E_STATE
    bad = dict(geom, block_in=np.r_[geom["block_in"], geom["block_in"][:1]],
               block_out=np.r_[geom["block_out"], geom["block_out"][:1]])
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_geometry([bad])  # a block ghost targeted twice
    assert e.value.code == ib.E_ARG
    neib = np.array(geom["neib"], copy=True)
    neib.reshape(-1)[-1] = len(geom["kind"])  # one past the level's boxes
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_geometry([dict(geom, neib=neib)])
    assert e.value.code == ib.E_ARG
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_distance(bodies, [p])  # the bad geometry was dropped
    assert e.value.code == ib.E_STATE
    sol.wall_geometry([geom])
    p["body"][np.flatnonzero(p["signdis"] < 1.0)[0]] = 7  # no such body
    p["nblock"] = pairs["nblock"]
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_distance(bodies, [p])
    assert e.value.code == ib.E_ABORT
    sol.close()


def near_reference(prev, new, band):
    """The boxes ibgpu_wall_distance_near reports: |signdis| < band before or
    after the move, or a changed side; in box order."""
    keep = ((np.abs(np.asarray(prev["signdis"])) < band) | (np.abs(new["signdis"]) < band) |
            (new["moved"] != 0))
    return np.flatnonzero(keep)


def test_near_output_is_the_full_output_near_the_walls(cuda_lib, pkg):
    """From the pairs the device kept, the near-wall call reports exactly the
    boxes near a wall before or after the move or on the other side now,
    with the full call's pairs; the block pairs' flags in full; afterwards
    ibgpu_wall_fetch returns every box's pair as the full call does."""
    ib = pkg.ibgpu
    bodies1, geom, pairs = wo.synthetic_case(seed=2, turn=0.05)
    bodies2, _, _ = wo.synthetic_case(seed=2, turn=0.3)
    ref1 = wo.wall_distance(bodies1, geom, pairs)
    ref2 = wo.wall_distance(bodies2, geom, dict(ref1, nblock=pairs["nblock"]))
    P, cells, prim = wl.vortex_case(32)
    n, nblock = len(geom["kind"]), int(pairs["nblock"])
    for band in (0.0, 0.4, 1e9):
        sol = ib.FlowSolver(P)
        sol.wall_geometry([geom, geom])
        p = [{k: np.array(v, copy=True) for k, v in pairs.items() if k != "nblock"}
             for _ in range(2)]
        for q in p:
            q["nblock"] = pairs["nblock"]
        sol.wall_distance(bodies1, p)
        out = sol.wall_distance_near(bodies2, [band, band], [n, n], [nblock, nblock])
        want = near_reference(ref1, ref2, band)
        for ch, bm in out:
            assert np.array_equal(ch["box"], want)
            for k in ("body", "patch", "distance", "signdis", "distance_to_body", "solid",
                      "moved"):
                assert np.array_equal(bits(ch[k]), bits(np.asarray(ref2[k])[want])), (band, k)
            assert np.array_equal(bm, ref2["block_moved"])
        got = sol.wall_fetch([n, n])
        for g in got:
            for k in ("body", "patch", "distance", "signdis", "distance_to_body", "solid"):
                assert np.array_equal(bits(g[k]), bits(ref2[k])), k
        sol.close()


def test_near_output_needs_resident_pairs_and_room(cuda_lib, pkg):
    ib = pkg.ibgpu
    bodies1, geom, pairs = wo.synthetic_case(seed=6, turn=0.05)
    bodies2, _, _ = wo.synthetic_case(seed=6, turn=0.2)
    ref1 = wo.wall_distance(bodies1, geom, pairs)
    ref2 = wo.wall_distance(bodies2, geom, dict(ref1, nblock=pairs["nblock"]))
    P, cells, prim = wl.vortex_case(32)
    n, nblock = len(geom["kind"]), int(pairs["nblock"])
    sol = ib.FlowSolver(P)
    sol.wall_geometry([geom])
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_distance_near(bodies1, [1.0], [n], [nblock])  # no pairs on the device yet
    assert e.value.code == ib.E_STATE
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_fetch([n])
    assert e.value.code == ib.E_STATE
    p = {k: np.array(v, copy=True) for k, v in pairs.items() if k != "nblock"}
    p["nblock"] = pairs["nblock"]
    sol.wall_distance(bodies1, [p])
    with pytest.raises(ib.IbgpuError) as e:
        sol.wall_distance_near(bodies2, [1e9], [5], [nblock])  # room for 5 boxes only
    assert e.value.code == ib.E_ARG
    # the device moved on all the same: every pair is there
    got = sol.wall_fetch([n])[0]
    for k in ("body", "patch", "distance", "signdis", "distance_to_body", "solid"):
        assert np.array_equal(bits(got[k]), bits(ref2[k])), k
    sol.close()
