"""Failure detection of a device wait, without a GPU fault: every
grid-barrier wait of the cooperative tridiagonalisation is bounded.  The
fault is injected on the host: the panel launches' barriers are told to
expect one CTA more than is launched (a CTA that never arrives), with the
wait bound set short (2^14 polls, a few milliseconds).  Each wait must run
out, the launch must end early, the error must come back through
nrgb_syev_batched as a status with "grid barrier timed out", and the same
context must then solve the same block correctly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    return (A + A.T) / 2


def test_barrier_wait_runs_out_and_the_context_stays_usable():
    import nrgb
    ctx = nrgb.Context(0)
    try:
        # 800 > the largest cluster-sized block: the panel path with its grid
        # barriers runs for the leading columns; small blocks ride along
        mats = [_sym(800, 1), _sym(20, 2), _sym(200, 3)]
        ctx.set_wait_limit(14)
        ctx.inject_barrier_shortfall(True)
        with pytest.raises(RuntimeError, match="grid barrier timed out"):
            ctx.syev_batched(mats)
        ctx.inject_barrier_shortfall(False)
        ctx.set_wait_limit(23)
        w, Z = ctx.syev_batched(mats)
        for A, wi, Zi in zip(mats, w, Z):
            n = A.shape[0]
            ref = np.linalg.eigvalsh(A)
            nrm = np.abs(ref).max()
            assert np.max(np.abs(wi - ref)) <= 1e-13 * nrm * max(10, n)
            assert np.abs(A @ Zi - Zi * wi).max() <= 1e-13 * nrm * max(10, n)
    finally:
        ctx.close()
