"""The coarse/fine interface lists as a function of the leaf cells
(oracle/interfaces_oracle.py) against the reference's own lists (no GPU):
after every one of 20 regrids of runs steered away from the plain criterion
(3 and 4 levels), the restriction pairs with their layers, the prolongation
pairs and the interface ghost cells equal the reference's, as keyed sets."""
import os
import sys

import numpy as np
import pytest

from conftest import ORACLE_DIR
from regrid_runs import BINARY, noisy_regrid_dumps

sys.path.insert(0, ORACLE_DIR)
import interfaces_oracle as io  # noqa: E402

pytestmark = pytest.mark.skipif(not os.path.exists(BINARY), reason="reference oracle not built")


@pytest.mark.parametrize("levels,seed", [(3, 7), (4, 11)])
def test_interface_lists_follow_from_the_leaves(levels, seed):
    dumps = noisy_regrid_dumps(levels, seed)
    assert len(dumps) == 20
    counts = set()
    for k, d in enumerate(dumps):
        leaf = d["kind"] == 0
        got = io.interfaces(d["level"][leaf], d["ix"][leaf], d["iy"][leaf], levels)
        want = io.reference_lists(d)
        for name, a, b in zip(("restriction", "prolongation", "ghost"), got, want):
            assert np.array_equal(a, b), f"regrid {k}: {name} pairs differ"
        counts.add(int(leaf.sum()))
        assert len(got[0]) and len(got[1])
    assert len(counts) > 5  # the regrids did change the mesh
