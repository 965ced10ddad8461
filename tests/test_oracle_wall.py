"""The CPU restatement of the reference's wall-distance passes for moved
bodies (oracle/wall_oracle.py) on seeded synthetic bodies and boxes: what
the reference's loops guarantee (Bodymove.cpp:127-255, Mesh.cpp:2303-2374)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import wall_oracle as wo  # noqa: E402


def test_walk_ends_where_no_neighbour_patch_is_closer():
    bodies, geom, pairs = wo.synthetic_case(seed=1)
    out = wo.wall_distance(bodies, geom, pairs)
    band = (np.asarray(pairs["signdis"]) < wo.CRITIC) & (geom["kind"] != wo.BLOCK_GHOST)
    assert band.sum() > 1000
    for i in np.flatnonzero(band)[::37]:
        b, p = int(out["body"][i]), int(out["patch"][i])
        base = int(bodies["patch_start"][b])
        d = wo._dist(bodies, base + p, geom["center"][i])
        assert d == out["distance"][i]
        for k in range(int(bodies["nb_count"][base + p])):
            q = int(bodies["nb"][base + p][k])
            assert wo._dist(bodies, base + q, geom["center"][i]) >= d


def test_sides_move_lists_and_block_ghosts():
    bodies, geom, pairs = wo.synthetic_case(seed=2, turn=0.2)
    out = wo.wall_distance(bodies, geom, pairs)
    kind = geom["kind"]
    moved = out["moved"]
    # the body turned: some boxes changed sides, never a domain ghost or a block ghost
    assert (moved == wo.INTO).any() and (moved == wo.OUT).any()
    assert not moved[kind != wo.OTHER].any()
    inside = out["signdis"] < 0
    band = (np.asarray(pairs["signdis"]) < wo.CRITIC) & (kind != wo.BLOCK_GHOST)
    assert np.array_equal(out["solid"][band].astype(bool), inside[band])
    # signed distance capped by the distance to the domain boundary
    assert np.all(out["signdis"][band] <= geom["distance_to_dm"][band])
    # block ghosts: their origin's pair
    bi, bo = geom["block_in"], geom["block_out"]
    for k in ("body", "patch", "distance", "signdis"):
        assert np.array_equal(out[k][bo], out[k][bi])
    # both bodies meet somewhere: junction boxes switched body
    assert (out["body"] != pairs["body"]).any()
