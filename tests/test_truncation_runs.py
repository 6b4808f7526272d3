"""The device truncation replays the reference's cluster scan
(src/splitting.cc:45-77) in parallel: values at least fixeps above their
predecessor always start a new cluster, so the sorted list splits into
independent runs and one thread scans each run; new keys come out in key
order with adjacent duplicates dropped, and keys already mapped keep their
value.  This CPU test restates that decomposition (as the kernels in
csrc/truncate.cu do it) and checks it against the oracle's sequential scan,
pass for pass, on lists made of tight groups whose spacings straddle fixeps,
with a map carried over several steps."""
import numpy as np
import pytest

import nrg_oracle as O


def runs_scan(es, eps):
    """The kernels' candidate list: (key, value) in key order."""
    n = len(es)
    cand = {}
    for i0 in range(n):
        if i0 > 0 and not (es[i0] - es[i0 - 1] >= eps):
            continue
        i1 = i0 + 1
        while i1 < n and not (es[i1] - es[i1 - 1] >= eps):
            i1 += 1
        c0, e0 = i0, es[i0]
        for i in range(i0 + 1, i1 + 1):
            if i < i1 and es[i] - e0 < eps:
                continue
            if i < n:
                if any(es[k] != es[c0] for k in range(c0 + 1, i)):
                    for k in range(c0 + 1, i):
                        if es[k] != es[c0] and es[k] != es[k - 1]:
                            cand[k] = (float(es[k]), float(es[c0]))
            if i < i1:
                c0, e0 = i, es[i]
    return [cand[k] for k in sorted(cand)]


def merge(mapping, cands):
    for k, v in cands:
        if k not in mapping:
            mapping[k] = v


def groups(rng, eps, n):
    base = np.sort(rng.uniform(0.0, 5.0, n // 4))
    vals = []
    for b in base:
        m = rng.integers(1, 7)
        steps = rng.choice([0.0, 0.3, 0.7, 1.0, 1.5], m) * eps
        vals.extend(b + np.cumsum(steps))
    return np.array(vals)


@pytest.mark.parametrize("seed", range(6))
def test_parallel_runs_match_the_sequential_scan(seed):
    rng = np.random.default_rng(seed)
    eps = 1e-15 * 4  # spacings of a few ulp around 1..5
    o = O.Oracle.__new__(O.Oracle)
    o.P = {"fixeps": eps}
    o.cluster_map = {}
    mine = {}
    for step in range(4):
        vals = groups(rng, eps, 400)
        for _ in range(2):  # find_clusters, fix_splittings, find_clusters
            es = np.sort(vals)
            o.find_clusters(es)
            merge(mine, runs_scan(es, eps))
            assert mine == o.cluster_map
            vals = np.array([mine.get(float(v), float(v)) for v in vals])
    assert len(mine) > 0
