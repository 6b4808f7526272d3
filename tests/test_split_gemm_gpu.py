"""The split-precision grouped GEMM (nrgb_gemm_grouped_split_dev: INT8
slices on the tcgen05 tensor cores, INT32 accumulators in tensor memory,
FP64 recombination) against torch FP64.

* Integer operands whose rows/columns reach 127 are cut exactly into their
  first slice, so every product is an exact integer: the result must equal
  the FP64 product bit for bit (this pins the shared-memory layout, the
  matrix and instruction descriptors and the tensor-memory read-back).
* Gaussian operands, all transposes, several segments per output, beta,
  ragged sizes: the error must stay within the slicing bound
  k * 2^-7S * (S + 3) * max|row of op(A)| * max|column of op(B)|.
"""
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
    return t.t().contiguous()


def _run(ctx, slices, cases, gen, seed):
    """cases: list of (m, n, [(k, ta, tb, alpha), ...], beta). Returns
    [(got, ref, bound)]."""
    import nrgb
    g = torch.Generator(device="cpu").manual_seed(seed)
    dev = "cuda:0"
    outs, terms, keep, res = [], [], [], []
    for m, n, segs, beta in cases:
        C0 = gen(g, (m, n)).to(dev)
        Cc = _col(C0)
        ref = beta * C0.clone()
        bound = torch.zeros(m, n, dtype=torch.float64, device=dev)
        t0 = len(terms)
        for k, ta, tb, alpha in segs:
            A = gen(g, (m, k)).to(dev)
            B = gen(g, (k, n)).to(dev)
            As = _col(A.t()) if ta else _col(A)
            Bs = _col(B.t()) if tb else _col(B)
            keep += [As, Bs]
            terms.append(nrgb.GemmTerm(As.data_ptr(), Bs.data_ptr(), (k if ta else m), (n if tb else k), k,
                                       ta, tb, alpha))
            ref += alpha * (A @ B)
            ra = A.abs().amax(dim=1, keepdim=True)
            cb = B.abs().amax(dim=0, keepdim=True)
            bound += abs(alpha) * k * 2.0 ** (-7 * slices) * (slices + 3) * 4.0 * (ra @ cb)
        outs.append(nrgb.GemmOut(Cc.data_ptr(), m, m, n, beta, t0, len(segs)))
        res.append((Cc, ref, bound))
    ctx.gemm_grouped_split_dev(slices, outs, terms)
    torch.cuda.synchronize()
    return [(Cc.t(), ref, bound) for Cc, ref, bound in res]


def _ints(g, shape):
    x = torch.randint(-127, 128, shape, generator=g, dtype=torch.int64).to(torch.float64)
    x[..., 0] = 127.0  # every row reaches 127 ...
    x[0, ...] = 127.0  # ... and every column: one exact slice
    return x


def _gauss(g, shape):
    return torch.randn(shape, generator=g, dtype=torch.float64)


@pytest.mark.parametrize("slices", [2, 8])
def test_split_gemm_integer_operands_are_exact(ctx, slices):
    cases = [(128, 64, [(64, 0, 0, 1.0)], 0.0),
             (200, 100, [(300, 0, 1, 1.0), (40, 1, 0, 1.0)], 0.0)]
    for got, ref, _ in _run(ctx, slices, cases, _ints, 1):
        assert torch.equal(got, ref), (got - ref).abs().max().item()


@pytest.mark.parametrize("slices", [4, 8])
def test_split_gemm_gaussian_within_the_slicing_bound(ctx, slices):
    cases = []
    for i, (m, n, k) in enumerate([(1, 1, 1), (7, 5, 3), (128, 64, 64), (129, 65, 65), (300, 17, 1000),
                                   (64, 300, 777)]):
        segs = [(k + s, (i + s) & 1, (i >> 1 + s) & 1, 0.5 - s) for s in range(1 + i % 3)]
        cases.append((m, n, segs, 0.25 if i % 2 else 0.0))
    for got, ref, bound in _run(ctx, slices, cases, _gauss, 2):
        err = (got - ref).abs()
        assert bool(torch.all(err <= bound + 1e-15 * ref.abs())), (err / (bound + 1e-300)).max().item()
    if slices == 8:
        # FP64 level: within the rounding bound of an FP64 product
        for got, ref, _ in _run(ctx, slices, cases, _gauss, 2):
            scale = ref.abs().max().item() + 1.0
            assert (got - ref).abs().max().item() <= 1e-13 * scale


def test_split_gemm_long_inner_dimension_is_cut(ctx):
    """k beyond the INT32 accumulator limit (16000) is cut into pieces."""
    for got, ref, bound in _run(ctx, 8, [(33, 20, [(16100, 1, 0, 1.0)], 0.0)], _gauss, 3):
        assert bool(torch.all((got - ref).abs() <= bound + 1e-15 * ref.abs()))
