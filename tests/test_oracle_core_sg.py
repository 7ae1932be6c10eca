"""The oracle's Core-SG (core-sg.cu) on the reference's golden fixtures, bit
for bit against the reference's own core-SG: Union_kNNG_MST
(core-sg.cu:292-420) + update_core_sg_weights (core-sg.cu:432-471) run on the
fixture's kNN graph and its sorted MST (tests/golden/make_ref_golden.py
--add-core-sg): row offsets, rows (own kNN ids, non-mutual reverse sources,
MST neighbours in sorted-MST edge order) and the Euclidean weights."""
import glob
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
pytestmark = pytest.mark.skipif(not FILES, reason="no golden fixtures")


@pytest.fixture(params=FILES, ids=lambda p: os.path.basename(p)[4:-4])
def golden(request):
    with open(request.param[:-4] + ".json") as f:
        meta = json.load(f)
    return dict(np.load(request.param)), meta


def test_core_sg_equals_the_reference(oracle, golden):
    g, meta = golden
    nindex, nlist, ew = oracle.core_sg(g["ids"], g["dist"], g["X"], g["mst_32"])
    np.testing.assert_array_equal(nindex, g["coresg_nindex"])
    np.testing.assert_array_equal(nlist, g["coresg_nlist"])
    np.testing.assert_array_equal(ew.view(np.uint32), g["coresg_eweight"].view(np.uint32))
