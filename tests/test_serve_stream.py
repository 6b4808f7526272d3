"""The served workload's definition (host only): the seeded request stream,
the Poisson arrivals and the bench's helpers that weight per-Nkeep timings
by the stream's Nkeep mix."""
import numpy as np
import pytest

import bench
import serve


def test_stream_is_seeded_z_by_eps_grid():
    a, b = serve.stream(), serve.stream()
    assert len(a) == 256
    assert [(r.z, r.eps_d, r.keep) for r in a] == [(r.z, r.eps_d, r.keep) for r in b]
    # eps_d runs fastest: 8 z values, each crossed with the same 32 eps_d
    assert [r.z for r in a[::32]] == [(k + 1) / 8 for k in range(8)]
    eps = [r.eps_d for r in a[:32]]
    assert len(set(eps)) == 32 and all(-0.2 <= e <= 0.0 for e in eps)
    for k in range(8):
        assert [r.eps_d for r in a[32 * k:32 * k + 32]] == eps
    assert {r.keep for r in a} <= set(serve.KEEPS)
    assert len({r.keep for r in a}) == len(serve.KEEPS)
    c = serve.stream(seed=serve.SEED + 1)
    assert [(r.eps_d, r.keep) for r in c] != [(r.eps_d, r.keep) for r in a]


def test_arrivals_are_poisson_at_the_stated_rate():
    assert np.all(serve.arrivals(5, 0.0) == 0.0)
    t = serve.arrivals(20000, 4.0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert np.all(gaps > 0)
    assert np.mean(gaps) == pytest.approx(0.25, rel=0.03)
    # exponential gaps: standard deviation equal to the mean
    assert np.std(gaps) == pytest.approx(np.mean(gaps), rel=0.05)
    assert np.array_equal(serve.arrivals(100, 4.0), serve.arrivals(100, 4.0))


def test_bench_waves_extend_the_stream():
    base = serve.stream()
    w4 = bench.stream_waves(4)
    assert len(w4) == 4 * bench.WAVE
    assert [(r.z, r.eps_d, r.keep) for r in w4] == [(r.z, r.eps_d, r.keep) for r in base[:4 * bench.WAVE]]
    w9 = bench.stream_waves(9)
    assert [(r.eps_d, r.keep) for r in w9[:256]] == [(r.eps_d, r.keep) for r in base]
    nxt = serve.stream(seed=serve.SEED + 1000)
    assert [(r.eps_d, r.keep) for r in w9[256:]] == [(r.eps_d, r.keep) for r in nxt[:32]]


def test_mix_weighting():
    reqs = bench.stream_waves(4)
    mix = bench.keep_mix(reqs)
    assert sum(mix.values()) == pytest.approx(1.0)
    one = bench.one_per_keep(reqs)
    assert [r.keep for r in one] == sorted(mix)
    # one run at a time: the mean time per run is the mix-weighted time
    per = {200: 1.0, 500: 2.0, 1000: 4.0, 2000: 8.0}
    rate = bench.mix_rate(per, mix)
    assert rate == pytest.approx(3600.0 / sum(f * per[k] for k, f in mix.items()))
    assert bench.mix_rate(per, {200: 0.5, 500: 0.5}) == pytest.approx(2400.0)
