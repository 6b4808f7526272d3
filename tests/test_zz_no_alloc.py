"""nrgb_basis_change_noalloc: the allocation-free basis change for callers
that must not see the library allocate device memory (hosts that own the
device-memory budget, loops that cannot take cudaMalloc's synchronisation).

Its results are compared with those of the regular entry point
(nrgb_eig_recalc_step_dev, which allocates its intermediates in the context),
within the GEMM tolerance of the other kernel tests, on two calls in a row
that share the library's static scratch array.  This file is collected last
so that a run stopping at the first failure has already run everything else.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _call(lib, nb, nk, zb, zk, op, out, stream):
    n = len(nb)
    P = lambda xs: (ctypes.c_void_p * n)(*xs)
    return lib.nrgb_basis_change_noalloc(n, (ctypes.c_int * n)(*nb), (ctypes.c_int * n)(*nk), P(zb), P(zk),
                                         P(op), P(out), ctypes.c_void_p(stream))


def test_noalloc_basis_change_matches_regular_entry_point():
    import nrgb
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    lib = nrgb.load()
    ctx = nrgb.Context(0)
    dev = "cuda:0"
    st = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device=dev)
    # the third call comes close to the 32 MiB limit: two intermediates of
    # 1400 x 1440 doubles (2 x 15.4 MiB) plus the descriptors
    for call, ns in enumerate(([5, 40, 33, 100, 64], [17, 129, 2, 70, 45, 8], [1400, 1440])):
        g.manual_seed(100 + call)
        nblk = len(ns)
        bra = [k for k in range(nblk) for _ in range(2)]
        ket = [(k + 1) % nblk for k in range(nblk) for _ in range(2)]
        H = []
        for n in ns:
            X = torch.randn(n, n, generator=g, device=dev, dtype=torch.float64)
            H.append(((X + X.T) / 2).contiguous())
        A = [h.clone() for h in H]
        W = [torch.empty(n, device=dev, dtype=torch.float64) for n in ns]
        Z = [torch.empty(n, n, device=dev, dtype=torch.float64) for n in ns]
        # op[o] is n_bra x n_ket column-major = a torch (n_ket x n_bra) row-major tensor
        O = [torch.randn(ns[k], ns[b], generator=g, device=dev, dtype=torch.float64) for b, k in zip(bra, ket)]
        ref = [torch.empty(ns[k], ns[b], device=dev, dtype=torch.float64) for b, k in zip(bra, ket)]
        ctx.eig_recalc_step_dev(ns, [a.data_ptr() for a in A], [w.data_ptr() for w in W],
                                [z.data_ptr() for z in Z], bra, ket, [o.data_ptr() for o in O],
                                [r.data_ptr() for r in ref], stream=st)
        if nblk == 2:
            bra, ket, O, ref = bra[::2], ket[::2], O[::2], ref[::2]
        new = [torch.full((ns[k], ns[b]), float("nan"), device=dev, dtype=torch.float64) for b, k in zip(bra, ket)]
        nb_, nk_ = [ns[b] for b in bra], [ns[k] for k in ket]
        zb_, zk_ = [Z[b].data_ptr() for b in bra], [Z[k].data_ptr() for k in ket]
        op_, out_ = [o.data_ptr() for o in O], [x.data_ptr() for x in new]
        if call == 1:
            # empty operators (no bra or no ket states) take no GEMM work but
            # still advance the scratch layout: the operators after them must
            # come out unchanged
            spare = torch.zeros(8, device=dev, dtype=torch.float64)
            for pos, (b0, k0) in ((0, (0, 7)), (3, (6, 0))):
                nb_.insert(pos, b0)
                nk_.insert(pos, k0)
                zb_.insert(pos, spare.data_ptr())
                zk_.insert(pos, spare.data_ptr())
                op_.insert(pos, spare.data_ptr())
                out_.insert(pos, spare.data_ptr())
        rc = _call(lib, nb_, nk_, zb_, zk_, op_, out_, st)
        assert rc == 0
        torch.cuda.synchronize()
        for r, x in zip(ref, new):
            scale = r.abs().max().item() + 1.0
            assert torch.isfinite(x).all()
            assert (x - r).abs().max().item() <= 1e-13 * scale * 50
    ctx.close()


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    import nrgb
    lib = nrgb.load()
    # more than 32 MiB of intermediates: refused before any GPU work
    assert _call(lib, [3000], [3000], [0], [0], [0], [0], 0) == 5
    # more operators than the descriptor capacity
    n = 1025
    assert lib.nrgb_basis_change_noalloc(n, (ctypes.c_int * n)(*([1] * n)), (ctypes.c_int * n)(*([1] * n)),
                                         (ctypes.c_void_p * n)(), (ctypes.c_void_p * n)(),
                                         (ctypes.c_void_p * n)(), (ctypes.c_void_p * n)(), None) == 5


def test_noalloc_refuses_a_capturing_stream():
    """A call on a stream that is capturing returns 7 before enqueueing
    anything, and the caller's capture stays valid (the graph still
    instantiates and replays)."""
    import nrgb
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    lib = nrgb.load()
    dev = "cuda:0"
    Z = torch.eye(4, device=dev, dtype=torch.float64)
    O = torch.ones(4, 4, device=dev, dtype=torch.float64)
    out = torch.zeros(4, 4, device=dev, dtype=torch.float64)
    x = torch.ones(16, device=dev)
    # first call outside any capture: the per-device set-up
    assert _call(lib, [4], [4], [Z.data_ptr()], [Z.data_ptr()], [O.data_ptr()], [out.data_ptr()],
                 torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        y = x * 2
        st = torch.cuda.current_stream().cuda_stream
        rc = _call(lib, [4], [4], [Z.data_ptr()], [Z.data_ptr()], [O.data_ptr()], [out.data_ptr()], st)
    assert rc == 7
    graph.replay()
    torch.cuda.synchronize()
    assert torch.all(y == 2)
