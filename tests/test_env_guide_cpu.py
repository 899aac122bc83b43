"""The guide tables of the environment light's CDF searches, restated on the
CPU: a search that starts from the guide's bucket range ends at the index the
full upper_bound search (CUDA-RayTracer/Helpers.cu:16-31) ends at, for every
float draw, on sorted lists with plateaus, and every list that is not sorted
(a NaN, an entry one ulp below its predecessor) falls back to the full range.

Follows the device code: k_env_guide (firefly_b200/csrc/ff_envmap.cu) builds
entry k of G buckets as the full search's end index for the float k / G, or
kGuideFull for a list that is not sorted; upper_bound_ref<G>
(firefly_b200/csrc/ff_shade.cuh) takes k = min(int(v * G), G - 1) for a draw v
in [0, 1] and searches [guide[k], guide[k + 1]).  The on-device check of the
same claim against the device's own tables is
tests/test_env_gpu.py::test_env_pick_matches_full_search.
"""
from __future__ import annotations

import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

GUIDE_FULL = 0x80000000


def search(lst, val, left=0, right=None):
    """The loop of upper_bound: (double)val >= list[middle] moves right."""
    right = len(lst) if right is None else right
    v = float(np.float32(val))
    while left < right:
        mid = (right - left) // 2 + left
        if v >= lst[mid]:
            left = mid + 1
        else:
            right = mid
    return left


def build_guide(lst, G):
    lst = np.asarray(lst, np.float64)
    n = len(lst)
    bad = any(not (lst[i] <= lst[i + 1]) for i in range(n - 1)) or (n > 0 and not (lst[-1] == lst[-1]))
    if bad:
        return [GUIDE_FULL] * (G + 1)
    return [search(lst, np.float32(k) / np.float32(G)) for k in range(G + 1)]


def guided(lst, val, guide, G):
    v = np.float32(val)
    left, right = 0, len(lst)
    if v >= 0 and v <= 1:
        k = min(int(v * np.float32(G)), G - 1)
        a, b = guide[k], guide[k + 1]
        if not a & GUIDE_FULL:
            left, right = a, b
    return search(lst, v, left, right)


def draws(lst, rng, n_random=300):
    edges = [np.float32(k) / np.float32(64) for k in range(65)]
    vals = [np.float32(x) for x in lst if np.isfinite(x) and 0 <= x <= 1]
    base = np.array(edges + vals + [0.0, 1.0], np.float32)
    near = np.concatenate([base, np.nextafter(base, np.float32(0)), np.nextafter(base, np.float32(1))])
    extra = np.array([-0.0, 1.5, -0.25, np.nan, np.inf], np.float32)
    return np.concatenate([rng.random(n_random, dtype=np.float32), near, extra])


def cdf_with_plateaus(rng, n, zero_frac):
    p = rng.random(n)
    p[rng.random(n) < zero_frac] = 0.0
    c = np.cumsum(p)
    return c / c[-1] if c[-1] > 0 else c


def check(lst, G, rng):
    g = build_guide(lst, G)
    for v in draws(lst, rng):
        assert guided(lst, v, g, G) == search(lst, v), (len(lst), G, float(v))
    return g


def test_sorted_lists_take_the_guided_path():
    rng = np.random.default_rng(0)
    for n in (1, 2, 3, 7, 64, 257):
        for G in (1, 4, 64, 512):
            for zero_frac in (0.0, 0.5, 0.95):
                g = check(cdf_with_plateaus(rng, n, zero_frac), G, rng)
                assert not g[0] & GUIDE_FULL


def test_lists_that_are_not_sorted_search_everything():
    rng = np.random.default_rng(1)
    c = cdf_with_plateaus(rng, 100, 0.2)
    nan_row = np.full(50, np.nan)
    inverted = c.copy()
    inverted[40] = np.nextafter(inverted[39], -np.inf)   # one ulp below its predecessor
    holed = c.copy()
    holed[70] = np.nan
    for lst in (nan_row, inverted, holed):
        g = check(lst, 64, rng)
        assert all(x == GUIDE_FULL for x in g)


def test_environment_like_cdf_with_a_sun():
    """A sky row: smooth mass everywhere and one texel holding most of it."""
    rng = np.random.default_rng(2)
    p = rng.lognormal(0.0, 0.5, 2048)
    p[1300:1303] = 5e4
    c = np.cumsum(p) / p.sum()
    check(c, 512, rng)


@settings(max_examples=60, deadline=None)
@given(st.lists(st.floats(min_value=0.0, max_value=1.0, allow_nan=False, width=32), min_size=1, max_size=40),
       st.sampled_from([1, 2, 8, 64, 512]), st.integers(0, 2**31 - 1))
def test_hypothesis_sorted_lists(values, G, seed):
    lst = np.sort(np.asarray(values, np.float64))
    check(lst, G, np.random.default_rng(seed))
