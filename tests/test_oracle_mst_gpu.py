"""The oracle's mst_gpu = 1 MST (int-quantised weights, gpuMST, buildMST_gpu)
against the reference's own output on the golden fixtures (`mstgpu`, made by
tests/golden/make_ref_golden.py --add-mst-gpu): edges, order, dequantised
weights and the multiplier, bit for bit."""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
pytestmark = pytest.mark.skipif(not FILES, reason="no golden fixtures")


@pytest.mark.parametrize("path", FILES, ids=lambda p: os.path.basename(p)[4:-4])
def test_quantised_mst_matches_reference(oracle, path):
    g = dict(np.load(path))
    mst, mult = oracle.mst_quantised(g["nindex"], g["nlist"], g["eweight"], g["dist"][:, 0])
    assert mult == int(g["mstgpu_mult"][0])
    np.testing.assert_array_equal(mst.view(np.int32), g["mstgpu"].view(np.int32))


def test_quantised_weight_overflow_takes_int_min(oracle):
    """A scaled weight beyond the int range becomes INT_MIN (the value x86's
    truncating conversion gives): its key sorts last in the Boruvka (the
    unsigned compare of the sign-extended key), and its dequantised weight
    is negative, so the final stable sort puts the edge first."""
    # path 0 - 1 - 2 with a tiny first distance and one heavy edge
    nindex = np.array([0, 1, 3, 4], np.int64)
    nlist = np.array([1, 0, 2, 1], np.int32)
    w = np.array([0.5, 0.5, 100.0, 100.0], np.float32)
    first = np.full(3, 1e-6, np.float32)
    mst, mult = oracle.mst_quantised(nindex, nlist, w, first)
    # float32(1e-6) lies just below 1e-6: ceil(-log10) = 7, so the multiplier is 9
    assert mult == int(np.ceil(-np.log10(np.float64(first[0])))) + 2 == 9
    assert mst["weight"][0] < 0 and (mst["from_node"][0], mst["to_node"][0]) == (1, 2)
    assert mst["weight"][1] == np.float32(0.5)
