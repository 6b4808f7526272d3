"""Numerics of the CUDA kernels through the C ABI, against FP64 references:
torch float64 matmul for the grouped GEMM, LAPACK (numpy eigh) for the
batched eigensolver (eigenvalues, residual, orthogonality)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    import nrgb
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    c = nrgb.Context(0)
    yield c
    c.close()


def _col(t):
    """column-major view: a torch tensor T (m x n) stored as T.t().contiguous()"""
    return t.t().contiguous()


def test_gemm_grouped_segments_and_transposes(ctx):
    import nrgb
    rng = np.random.default_rng(1)
    dev = "cuda:0"
    outs, terms, refs, keep = [], [], [], []
    cases = [(1, 1, 1), (7, 5, 3), (64, 64, 16), (65, 130, 33), (200, 17, 301), (128, 128, 1000)]
    for (m, n, k) in cases:
        for ta in (0, 1):
            for tb in (0, 1):
                nseg = 2
                C0 = torch.tensor(rng.standard_normal((m, n)), device=dev)
                Cc = _col(C0)
                ref = 0.5 * C0.clone()
                t0 = len(terms)
                for s in range(nseg):
                    kk = k + s
                    A = torch.tensor(rng.standard_normal((m, kk)), device=dev)
                    B = torch.tensor(rng.standard_normal((kk, n)), device=dev)
                    alpha = 0.7 - s
                    As = _col(A.t()) if ta else _col(A)   # storage of A or A^T, column-major
                    Bs = _col(B.t()) if tb else _col(B)
                    keep += [As, Bs]
                    terms.append(nrgb.GemmTerm(As.data_ptr(), Bs.data_ptr(),
                                               (kk if ta else m), (n if tb else kk), kk, ta, tb, alpha))
                    ref += alpha * (A @ B)
                outs.append(nrgb.GemmOut(Cc.data_ptr(), m, m, n, 0.5, t0, nseg))
                refs.append((Cc, ref))
    ctx.gemm_grouped_dev(outs, terms)
    torch.cuda.synchronize()
    for Cc, ref in refs:
        got = Cc.t()
        err = (got - ref).abs().max().item()
        scale = ref.abs().max().item() + 1.0
        assert err <= 1e-13 * scale * 50


def test_gemm_grouped_unaligned_views(ctx):
    """Operands at odd element offsets (base addresses not 16-byte aligned),
    even leading dimensions above odd row counts (element pairs that cross
    the matrix edge) and odd K, in all four transpose combinations."""
    import nrgb
    rng = np.random.default_rng(11)
    dev = "cuda:0"
    outs, terms, refs, keep = [], [], [], []
    for (m, n, k, off) in [(65, 67, 33, 1), (130, 129, 63, 0), (257, 96, 100, 3), (64, 64, 17, 1)]:
        for ta in (0, 1):
            for tb in (0, 1):
                ra, ca = (k, m) if ta else (m, k)
                rb, cb = (n, k) if tb else (k, n)
                lda, ldb = ra + 2 - (ra & 1), rb + 2 - (rb & 1)      # even, above the row count
                bufA = torch.tensor(rng.standard_normal(off + lda * ca), device=dev)
                bufB = torch.tensor(rng.standard_normal(off + ldb * cb), device=dev)
                Asto = bufA[off:].view(ca, lda).t()[:ra]              # column-major ra x ca
                Bsto = bufB[off:].view(cb, ldb).t()[:rb]
                A = Asto.t() if ta else Asto
                B = Bsto.t() if tb else Bsto
                C0 = torch.tensor(rng.standard_normal((m, n)), device=dev)
                Cc = _col(C0)
                keep += [bufA, bufB]
                t0 = len(terms)
                terms.append(nrgb.GemmTerm(bufA.data_ptr() + 8 * off, bufB.data_ptr() + 8 * off,
                                           lda, ldb, k, ta, tb, -0.5))
                outs.append(nrgb.GemmOut(Cc.data_ptr(), m, m, n, 1.0, t0, 1))
                refs.append((Cc, C0 - 0.5 * (A @ B)))
    ctx.gemm_grouped_dev(outs, terms)
    torch.cuda.synchronize()
    for Cc, ref in refs:
        err = (Cc.t() - ref).abs().max().item()
        assert err <= 1e-13 * (ref.abs().max().item() + 1.0) * 50


@pytest.mark.parametrize("stages", ["0", "3", "4", "232", "332"])
def test_gemm_pipelined_variants(stages):
    """The grouped GEMM's register-staged kernel (NRGB_GEMM_PIPE=0) and its
    cp.async-pipelined forms: K step 16 with 3 or 4 stages, K step 32 with 2
    or 3 stages (232, 332).  The switch is read once per process, so each
    form runs the GEMM tests in a child process."""
    import subprocess
    import sys
    env = dict(os.environ, NRGB_GEMM_PIPE=stages)
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider",
                        os.path.join(here, "test_kernels_gpu.py"), "-k",
                        "gemm_grouped_segments or gemm_grouped_unaligned"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]


def _random_sym(n, rng, kind):
    if kind == "gauss":
        A = rng.standard_normal((n, n))
        return (A + A.T) / 2
    Q, R = np.linalg.qr(rng.standard_normal((n, n)))
    Q = Q * np.sign(np.diag(R))
    if kind == "logspaced":  # the 40-block benchmark spectrum
        lam = np.logspace(-12, 1, n) * rng.choice([-1.0, 1.0], n)
    elif kind == "degenerate":  # NRG-like multiplets: many exactly repeated levels
        lam = np.repeat(rng.standard_normal((n + 3) // 4), 4)[:n]
    else:
        lam = rng.standard_normal(n)
    A = (Q * lam) @ Q.T
    return (A + A.T) / 2


# covers the warp path (n <= 32), the cluster path (one cluster of 1..16 CTAs
# per block, the smallest that holds it: the size changes after 167, 235,
# 287, 329, 367, 402, 433, 461, 486, 511, 539, 559, 583, 602, 619; single-CTA
# launches split at 64, 96, 128; blocks above 640 take the cooperative panel
# path; 168, 237, 333, 469 and 656 are the two-barrier kernel's limits) and
# the panel path
SIZES = [1, 2, 3, 5, 16, 31, 32, 33, 40, 64, 65, 96, 97, 100, 128, 129, 167, 168, 169, 235, 236, 237, 238, 257,
         287, 288, 329, 330, 333, 334, 367, 368, 402, 403, 433, 434, 461, 462, 469, 470, 486, 487, 511, 512, 539,
         540, 559, 560, 583, 584, 600, 602, 603, 619, 620, 640, 641, 656, 657, 1100]


@pytest.mark.parametrize("kind", ["gauss", "logspaced", "degenerate"])
def test_syev_batched_host_api(ctx, kind):
    rng = np.random.default_rng(7)
    mats = [_random_sym(n, rng, kind) for n in SIZES]
    w, Z = ctx.syev_batched(mats)
    for A, wi, Zi in zip(mats, w, Z):
        n = A.shape[0]
        ref = np.linalg.eigvalsh(A)
        nrm = max(np.abs(ref).max(), 1e-300)
        assert np.all(np.diff(wi) >= 0)
        assert np.max(np.abs(wi - ref)) <= 1e-13 * nrm * max(10, n)
        res = np.abs(A @ Zi - Zi * wi).max()
        assert res <= 1e-13 * nrm * max(10, n)
        orth = np.abs(Zi.T @ Zi - np.eye(n)).max()
        assert orth <= 1e-13 * max(10, n)


@pytest.mark.parametrize("env", [{"NRGB_TRDC_BARRIERS": "2"}, {"NRGB_TRDC_FUSED": "1"}, {"NRGB_TRDC_POW2": "1"}])
def test_syev_cluster_kernel_variants(env):
    """The other forms of the cluster tridiagonalisation (two cluster
    barriers per column; one barrier with the update and the next products
    fused; clusters of 1, 2, 4, 8, 16 CTAs only), selected when a context is
    created, solve the cluster-sized blocks to the same bounds."""
    import nrgb
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        c = nrgb.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    try:
        rng = np.random.default_rng(5)
        mats = [_random_sym(n, rng, kind) for n in (33, 100, 167, 200, 300, 461, 600, 640, 700)
                for kind in ("gauss", "degenerate")]
        w, Z = c.syev_batched(mats)
    finally:
        c.close()
    for A, wi, Zi in zip(mats, w, Z):
        n = A.shape[0]
        ref = np.linalg.eigvalsh(A)
        nrm = max(np.abs(ref).max(), 1e-300)
        assert np.max(np.abs(wi - ref)) <= 1e-13 * nrm * max(10, n)
        assert np.abs(A @ Zi - Zi * wi).max() <= 1e-13 * nrm * max(10, n)
        assert np.abs(Zi.T @ Zi - np.eye(n)).max() <= 1e-13 * max(10, n)


def test_syev_per_block_mode_matches_batched(ctx):
    """One solver call per block gives the same decomposition as one batched
    call for all blocks (the eigenvector signs may differ)."""
    rng = np.random.default_rng(11)
    mats = [_random_sym(n, rng, "degenerate") for n in (40, 170, 300, 500, 700)]
    w0, Z0 = ctx.syev_batched(mats)
    ctx.set_eig_mode(1)
    try:
        w1, Z1 = ctx.syev_batched(mats)
    finally:
        ctx.set_eig_mode(0)
    for A, a, b, Za, Zb in zip(mats, w0, w1, Z0, Z1):
        nrm = np.abs(a).max()
        assert np.max(np.abs(a - b)) <= 1e-13 * nrm * A.shape[0]
        assert np.abs(A @ Zb - Zb * b).max() <= 1e-13 * nrm * A.shape[0]


def test_profile_only_times_one_kernel(ctx):
    """With timing restricted to one kernel, every launch is still counted but
    only that kernel's launches carry CUDA-event time."""
    rng = np.random.default_rng(12)
    mats = [_random_sym(n, rng, "degenerate") for n in (100, 200)]
    ctx.profile(True, only="trd_cluster")
    try:
        ctx.syev_batched(mats)
        n_cl, ms_cl = ctx.kernel_stats("trd_cluster")
        n_dc, ms_dc = ctx.kernel_stats("dc_*")
        n_all, _ = ctx.kernel_stats("*")
    finally:
        ctx.profile(False)
    assert n_cl >= 1 and ms_cl > 0
    assert n_dc >= 1 and ms_dc == 0
    assert n_all > n_cl + n_dc - 1
    ctx.profile(True)
    try:
        ctx.syev_batched(mats)
        n_dc2, ms_dc2 = ctx.kernel_stats("dc_*")
    finally:
        ctx.profile(False)
    assert n_dc2 == n_dc and ms_dc2 > 0


def test_gemm_grouped_large_tiles(ctx):
    """Problems large enough for the 128x128-tile kernel, with the schedule
    forcing it (gemm_large_from = 1) so that this kernel is the one that runs."""
    import nrgb
    saved = ctx.get_schedule()
    ctx.set_schedule(saved["cluster_limit"], 1)
    try:
        _large_tiles_case(ctx, nrgb)
    finally:
        ctx.set_schedule(saved["cluster_limit"], saved["gemm_large_from"])


def _large_tiles_case(ctx, nrgb):
    rng = np.random.default_rng(5)
    dev = "cuda:0"
    outs, terms, refs, keep = [], [], [], []
    for idx in range(8):
        m, n, k = 600 + 7 * idx, 590 - 5 * idx, 300 + 11 * idx
        ta, tb = idx & 1, (idx >> 1) & 1
        C0 = torch.tensor(rng.standard_normal((m, n)), device=dev)
        Cc = _col(C0)
        ref = -1.0 * C0.clone()
        t0 = len(terms)
        for s in range(3):
            kk = k + 17 * s
            A = torch.tensor(rng.standard_normal((m, kk)), device=dev)
            B = torch.tensor(rng.standard_normal((kk, n)), device=dev)
            alpha = 1.5 - 0.75 * s
            As = _col(A.t()) if ta else _col(A)
            Bs = _col(B.t()) if tb else _col(B)
            keep += [As, Bs]
            terms.append(nrgb.GemmTerm(As.data_ptr(), Bs.data_ptr(), (kk if ta else m), (n if tb else kk), kk,
                                       ta, tb, alpha))
            ref += alpha * (A @ B)
        outs.append(nrgb.GemmOut(Cc.data_ptr(), m, m, n, -1.0, t0, 3))
        refs.append((Cc, ref))
    ctx.gemm_grouped_dev(outs, terms)
    torch.cuda.synchronize()
    for Cc, ref in refs:
        err = (Cc.t() - ref).abs().max().item()
        assert err <= 1e-13 * (ref.abs().max().item() + 1.0) * 50


def _sym_torch(n, seed, kind, dev):
    """Q diag(lam) Q^T in float64 on the device (Q from the QR of a Gaussian
    matrix, column signs fixed by diag R), as the 40-block benchmark builds
    its blocks; lam as in _random_sym."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    G = torch.randn(n, n, generator=g, dtype=torch.float64).to(dev)
    Q, R = torch.linalg.qr(G)
    Q = Q * torch.sign(torch.diagonal(R))
    rng = np.random.default_rng(seed)
    if kind == "logspaced":
        lam = np.logspace(-12, 1, n) * rng.choice([-1.0, 1.0], n)
    else:
        lam = np.repeat(rng.standard_normal((n + 3) // 4), 4)[:n]
    lam_t = torch.tensor(lam, device=dev)
    A = (Q * lam_t) @ Q.T
    return (A + A.T) / 2, np.sort(lam)


# the block sizes of the workloads: up to 4096 in the 40-block benchmark,
# about 8000 in the two-channel Kondo run at keep 3000
@pytest.mark.parametrize("n", [2048, 4096, 8000])
@pytest.mark.parametrize("kind", ["logspaced", "degenerate"])
def test_syev_large_blocks(ctx, n, kind):
    """Eigenvalues against the spectrum the block was built from (whose
    construction error is ~1e-15 n |lam|max), residual |A Z - Z diag(w)| and
    orthogonality |Z^T Z - 1| in FP64 on the device, at the same n-scaled
    1e-13 bounds as the smaller sizes; the batch mixes the large block with
    small and medium ones so the panel, cluster and warp paths run together."""
    dev = "cuda:0"
    A, lam = _sym_torch(n, 100 + n, kind, dev)
    small = [torch.tensor(_random_sym(m, np.random.default_rng(m), kind), device=dev) for m in (24, 300, 700)]
    mats = [A] + small
    ns = [m.shape[0] for m in mats]
    a_in = [m.t().contiguous() for m in mats]          # column-major copies, overwritten by the solver
    ws = [torch.empty(k, dtype=torch.float64, device=dev) for k in ns]
    zs = [torch.empty(k, k, dtype=torch.float64, device=dev) for k in ns]
    ctx.syev_batched_dev(ns, [x.data_ptr() for x in a_in], [x.data_ptr() for x in ws], [x.data_ptr() for x in zs])
    torch.cuda.synchronize()
    for k, (M, w, Zc) in enumerate(zip(mats, ws, zs)):
        m = M.shape[0]
        Z = Zc.t()                                       # column r of Z = eigenvector r
        nrm = max(w.abs().max().item(), 1e-300)
        assert bool(torch.all(w[1:] >= w[:-1]))
        ref = lam if k == 0 else np.linalg.eigvalsh(M.cpu().numpy())
        assert np.max(np.abs(w.cpu().numpy() - ref)) <= 1e-13 * nrm * max(10, m)
        res = (M @ Z - Z * w).abs().max().item()
        assert res <= 1e-13 * nrm * max(10, m)
        orth = (Z.T @ Z - torch.eye(m, dtype=torch.float64, device=dev)).abs().max().item()
        assert orth <= 1e-13 * max(10, m)
