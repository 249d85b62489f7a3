"""Host side of the serving stream (CPU): the seeded request mix the serving
bench draws, and its arrival process.

Each request is a function of its index alone, so a stream of N requests is
the first N of every longer stream and the batched and one-after-another arms
see the same solves; the mix spans the sizes, methods and precisions it
states; Poisson arrivals are increasing with the requested mean rate.
"""
import numpy as np

from kamayan_b200 import serving


def test_requests_depend_on_index_only():
    a = [serving.make_request(i) for i in range(40)]
    b = [serving.make_request(i) for i in range(40)]
    for x, y in zip(a, b):
        assert x.deck.text() == y.deck.text()
        assert (x.problem, x.cells, x.label) == (y.problem, y.cells, y.label)
    assert len({r.deck.text() for r in a}) == len(a)


def test_request_mix_covers_the_stated_space():
    reqs = [serving.make_request(i) for i in range(400)]
    sizes = {(n, d) for n, d in serving.SIZES}
    seen = set()
    for r in reqs:
        n = round(r.cells ** (1 / 3)) if "^3" in r.label else round(r.cells ** 0.5)
        d = 3 if "^3" in r.label else 2
        assert n ** d == r.cells
        seen.add((n, d))
        assert r.problem in ("isentropic_vortex", "blast")
        assert r.label.split()[-1] in ("fp32", "fp64")
        assert r.deck.get("parthenon/time", "integrator") == "rk2"
    assert seen == sizes
    methods = {tuple(r.label.split()[2].split("/")) for r in reqs}
    assert methods == {(m[0], m[1]) for m in serving.METHODS}


def test_poisson_arrivals():
    t = serving.poisson_arrivals(20000, 50.0, seed=3)
    assert np.all(np.diff(t) > 0)
    assert abs(t[-1] / len(t) - 1 / 50.0) < 0.05 / 50.0
    assert np.array_equal(t, serving.poisson_arrivals(20000, 50.0, seed=3))


def test_percentile():
    assert serving.percentile([], 50) is None
    assert serving.percentile([1.0, 2.0, 3.0], 50) == 2.0
