"""The autotuner of the size-bucketed schedule: it times both GEMM tile
shapes over the edges 128..2048 and one batched eigensolve under several
cluster limits, sets the device's table to its choices, and the solver stays
correct under any limit it can choose (blocks above the limit take the
cooperative panel path for their leading columns)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    return (A + A.T) / 2


def test_autotune_sets_the_schedule_it_reports():
    import nrgb
    ctx = nrgb.Context(0)
    try:
        saved = ctx.get_schedule()
        rep = ctx.autotune()
        print("autotune report:", rep)
        sch = ctx.get_schedule()
        assert sch["cluster_limit"] == rep["cluster_limit"]
        assert sch["gemm_large_from"] == rep["gemm_large_from"]
        assert [g["edge"] for g in rep["gemm"]] == [128, 192, 256, 384, 512, 768, 1024, 1536, 2048]
        assert all(g["small_tf"] > 0 and g["large_tf"] > 0 for g in rep["gemm"])
        assert rep["cluster"][0]["limit"] == sch["cluster_capacity"]
        ctx.set_schedule(saved["cluster_limit"], saved["gemm_large_from"])
    finally:
        ctx.close()


@pytest.mark.parametrize("limit", [237, 400])
def test_solver_is_correct_under_a_lower_cluster_limit(limit):
    import nrgb
    ctx = nrgb.Context(0)
    saved = ctx.get_schedule()
    try:
        ctx.set_schedule(limit, saved["gemm_large_from"])
        mats = [_sym(n, n) for n in (100, limit, limit + 1, 500, 700)]
        w, Z = ctx.syev_batched(mats)
        for A, wi, Zi in zip(mats, w, Z):
            n = A.shape[0]
            ref = np.linalg.eigvalsh(A)
            nrm = np.abs(ref).max()
            assert np.max(np.abs(wi - ref)) <= 1e-13 * nrm * max(10, n)
            assert np.abs(A @ Zi - Zi * wi).max() <= 1e-13 * nrm * max(10, n)
            assert np.abs(Zi.T @ Zi - np.eye(n)).max() <= 1e-13 * max(10, n)
    finally:
        ctx.set_schedule(saved["cluster_limit"], saved["gemm_large_from"])
        ctx.close()
