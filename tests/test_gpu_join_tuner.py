"""FP32 local-join forms (one or two 4 x 4 distance tiles per lane) and the
per-shape tuner that picks between them: every form reaches the reference
algorithm's recall with exact distances, and the run statistics name the
form that ran."""
import numpy as np
import pytest

from conftest import blobs

pytestmark = pytest.mark.gpu


@pytest.fixture
def join_tiles(ctx):
    yield ctx.set_join_tiles
    ctx.set_join_tiles(0)


@pytest.mark.parametrize("n,d,k,S", [(20000, 12, 32, 16), (6000, 128, 32, 16), (12000, 24, 16, 8)])
def test_join_forms_reach_the_reference_recall(ctx, oracle, join_tiles, n, d, k, S):
    """Both forms compute the same exact FP32 pair distances; the graphs of
    two runs differ only where the order of the reverse-sample atomics does
    (as two runs of one form do), so each form is held to the recall of the
    oracle's NN-Descent and to exact distances."""
    X = blobs(n, d, seed=n + d + k, blobs=20)
    q = np.arange(0, n, 7)
    gt, _ = oracle.bruteforce_knn(X, k, q)
    oids, _ = oracle.nndescent(X, k, S, 6)
    r_orc = oracle.recall(oids[q], gt, k)
    rng = np.random.default_rng(1)
    for tiles in (1, 2):
        join_tiles(tiles)
        ids, dist = (a.cpu().numpy() for a in ctx.knn_split(
            ctx.NNDescent(X, k=k, sample_num=S, iterations=6)))
        assert oracle.validate_knn(ids)
        assert oracle.recall(ids[q], gt, k) >= r_orc - 0.005, tiles
        for i in rng.choice(n, 50, replace=False):
            for j in range(k):
                ref = np.float32(oracle.diffsum(X[i], X[ids[i, j]]))
                assert ref.view(np.uint32) == dist[i, j].view(np.uint32)


def test_run_statistics_name_the_join_form(ctx, join_tiles):
    X = blobs(8000, 16, seed=3)
    join_tiles(1)
    _, st1 = ctx.hdbscan(X, k=32, mpts=32)
    assert st1["join_config"] == 1
    join_tiles(2)
    _, st2 = ctx.hdbscan(X, k=32, mpts=32)
    assert st2["join_config"] == 2
    join_tiles(0)
    _, st0 = ctx.hdbscan(X, k=32, mpts=32)
    assert st0["join_config"] in (1, 2)
    # a second run of the shape reuses the tuned form
    _, st0b = ctx.hdbscan(X, k=32, mpts=32)
    assert st0b["join_config"] == st0["join_config"]
    _, stb = ctx.hdbscan(X, k=32, mpts=32, precision=1)
    assert stb["join_config"] == 0


def test_join_tiles_argument_is_checked(ctx):
    from gpu_hdbscan_b200._lib import HdbError

    with pytest.raises(HdbError):
        ctx.set_join_tiles(3)
