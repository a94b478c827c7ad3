"""Oracle pins: Morton codes, radix tree, escapes, refit and traversals.

Restates test/neighbor_search_tests.jl of the reference: prime-hash
coordinates (:45-54), Karras split/child rules re-derived per node for
n = 1..20 and 5 offsets (:177-232), identical codes (:236-247), AABB
containment (:251-287), node scale = recursive max (:291-305), radius queries
vs brute force on the 4-point square (:309-333) and line traversals vs brute
force (:415-457).  The Karras helpers below are an independent Python
restatement of BinaryRadixTree/toolbox.jl:14-76.
"""
import numpy as np
import pytest

import oracle as O

PRIMES = (37, 61, 97, 131, 197, 263)


def build_coords(dim, n, offset):
    mod = 1021
    out = []
    for d in range(dim):
        p, s = PRIMES[d], PRIMES[d + dim]
        out.append(np.array([float((p * i + s * offset) % mod) / mod for i in range(1, n + 1)]))
    return out


def clz64(v):
    v = int(v)
    return 64 - v.bit_length()


def delta(c, i, j):
    a, b = int(c[i - 1]), int(c[j - 1])
    return clz64(i ^ j) if a == b else clz64(a ^ b)


def find_range(c, i):
    n = len(c)
    dL = delta(c, i, i - 1) if i > 1 else -1
    dR = delta(c, i, i + 1) if i < n else -1
    d = 1 if dR - dL >= 0 else -1
    dmin = delta(c, i, i - d) if 1 <= i - d <= n else -1
    lmax = 2
    while True:
        j = i + lmax * d
        if j < 1 or j > n or delta(c, i, j) <= dmin:
            break
        lmax *= 2
    l, t = 0, lmax >> 1
    while t > 0:
        j = i + (l + t) * d
        if 1 <= j <= n and delta(c, i, j) > dmin:
            l += t
        t >>= 1
    j = i + l * d
    return min(i, j), max(i, j)


def split_position(c, first, last):
    if c[first - 1] == c[last - 1]:
        return min(max((first + last) >> 1, first), last - 1)
    p = delta(c, first, last)
    split, step = first, last - first
    while step > 1:
        step = (step + 1) >> 1
        ns = split + step
        if ns < last and delta(c, first, ns) > p:
            split = ns
    return split


def make(coords, h=None):
    n = len(coords[0])
    x, y, z = coords
    h = np.full(n, 0.1) if h is None else h
    return O.Oracle(x, y, z, np.ones(n), h, np.ones(n), [np.ones(n)])


@pytest.mark.parametrize("offset", range(5))
def test_karras_structure(offset):
    for n in range(1, 21):
        orc = make(build_coords(3, n, offset))
        t = orc.tree()
        codes = orc.codes
        tot = 2 * n - 1
        assert len(t["left"]) == tot
        assert t["root"] == (1 if n >= 2 else 0)
        if n >= 2:
            assert t["parent"][0] == 0
        assert np.all((t["parent"] >= 0) & (t["parent"] < tot + 1))
        assert np.all(codes[1:] > codes[:-1])  # strictly increasing after dedup
        for i in range(1, n):
            lo, hi = find_range(codes, i)
            s = split_position(codes, lo, hi)
            l, r = t["left"][i - 1], t["right"][i - 1]
            assert l == (n - 1 + lo if s == lo else s)
            assert r == (n - 1 + hi if s + 1 == hi else s + 1)
        assert np.all((t["escape"] >= 0) & (t["escape"] <= tot))


def test_escape_walk_visits_every_leaf_in_order():
    # with nothing pruned, left/escape DFS visits leaves 1..n in order
    for n in (2, 3, 7, 33, 200):
        orc = make(build_coords(3, n, 2))
        t = orc.tree()
        node, seen = t["root"], []
        for _ in range(4 * n):
            if node == 0:
                break
            if node >= n:
                seen.append(node - n + 1)
                node = t["escape"][node - 1]
            else:
                node = t["left"][node - 1]
        assert seen == list(range(1, n + 1))


@pytest.mark.parametrize("n", [1, 2, 8, 16])
def test_identical_codes(n):
    orc = make([np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.5)])
    t = orc.tree()
    assert t["root"] == (1 if n >= 2 else 0)
    assert int(np.sum(t["parent"] == 0)) == 1
    assert np.all(orc.codes[1:] > orc.codes[:-1])


def _child_bounds(t, orc_leaf, n, child, d, which):
    if child >= n:
        return orc_leaf[d][child - n]
    return t["node_min" if which == "min" else "node_max"][d][child - 1]


@pytest.mark.parametrize("n", [2, 8, 32])
def test_aabb_containment(n):
    c = np.linspace(0.0, 1.0, n)
    orc = make([c, c.copy(), c.copy()])
    t = orc.tree()
    leaf = [c[orc.perm], c[orc.perm], c[orc.perm]]
    for i in range(1, n):
        l, r = t["left"][i - 1], t["right"][i - 1]
        for d in range(3):
            lmin = _child_bounds(t, leaf, n, l, d, "min")
            rmin = _child_bounds(t, leaf, n, r, d, "min")
            lmax = _child_bounds(t, leaf, n, l, d, "max")
            rmax = _child_bounds(t, leaf, n, r, d, "max")
            assert t["node_min"][d][i - 1] == min(lmin, rmin)
            assert t["node_max"][d][i - 1] == max(lmax, rmax)


def test_node_scale_is_subtree_max():
    rng = np.random.default_rng(0xBEEF)
    n = 64
    h = rng.random(n)
    orc = make([rng.random(n), rng.random(n), rng.random(n)], h=h)
    t = orc.tree()
    hs = h[orc.perm]

    def smax(node):
        if node >= n:
            return hs[node - n]
        return max(smax(t["left"][node - 1]), smax(t["right"][node - 1]))

    for i in range(1, n):
        assert t["node_scale"][i - 1] == smax(i)


def test_radius_queries_match_brute_force():
    # 4-point square, test/neighbor_search_tests.jl:309-333
    x = np.array([0.0, 1.0, 0.0, 1.0])
    y = np.array([0.0, 0.0, 1.0, 1.0])
    z = np.zeros(4)
    orc = make([x, y, z])
    pts = np.array([[0.1, 0.1, 0.0], [0.9, 0.9, 0.0], [0.5, 0.5, 0.0]])
    radii = np.array([0.25, 0.25, 0.75])
    # gather with ha = r / 2 (support 2 ha = r)
    cnt, hsh, _ = orc.digest(tuple(pts.T), strategy=O.GATHER, hmode=O.H_PER_SAMPLE, hs=radii / 2)
    bc, bh = orc.brute_digest(tuple(pts.T), radii / 2, strategy=O.GATHER)
    assert np.array_equal(cnt, bc) and np.array_equal(hsh, bh)
    assert list(cnt) == [1, 1, 4]


@pytest.mark.parametrize("strategy", [O.GATHER, O.SCATTER, O.SYMMETRIC])
def test_traversals_match_brute_force_random(strategy):
    rng = np.random.default_rng(0xCAFE)
    n = 2000
    h = rng.uniform(0.01, 0.08, n)
    orc = make([rng.random(n), rng.random(n), rng.random(n)], h=h)
    s = tuple(rng.uniform(-0.1, 1.1, 500) for _ in range(3))
    ha = rng.uniform(0.01, 0.05, 500)
    cnt, hsh, _ = orc.digest(s, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=ha)
    bc, bh = orc.brute_digest(s, ha, strategy=strategy)
    assert np.array_equal(cnt, bc) and np.array_equal(hsh, bh)
    # nearest-h traversal equals the brute-force argmin (smallest index on ties)
    _, _, hn = orc.digest(s, strategy=O.GATHER, hmode=O.H_NEAREST)
    idx = orc.brute_nearest(*s)
    assert np.array_equal(hn, h[orc.perm][idx])


@pytest.mark.parametrize("strategy", [O.GATHER, O.SCATTER, O.SYMMETRIC])
def test_line_traversals_match_brute_force(strategy):
    # 5-point set in a plane, line along +x through the origin, r^2 = 0.04
    # (test/neighbor_search_tests.jl:415-457), then random lines
    x = np.array([0.0, 0.1, 0.3, 0.5, 0.2])
    y = np.array([0.0, 0.15, 0.25, 0.05, -0.1])
    z = np.zeros(5)
    orc = make([x, y, z], h=np.full(5, 0.1))
    o = (np.array([0.0]), np.array([0.0]), np.array([0.0]))
    d = (np.array([1.0]), np.array([0.0]), np.array([0.0]))
    cnt, hsh, _ = orc.digest(o, d, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=np.array([0.1]))
    bc, bh = orc.brute_digest(o, np.array([0.1]), d=d, strategy=strategy)
    assert np.array_equal(cnt, bc) and np.array_equal(hsh, bh)
    rng = np.random.default_rng(7)
    n = 3000
    orc = make([rng.random(n), rng.random(n), rng.random(n)], h=rng.uniform(0.005, 0.03, n))
    nl = 300
    o = tuple(rng.uniform(-0.5, 1.5, nl) for _ in range(3))
    dd = rng.standard_normal((3, nl))
    dd /= np.linalg.norm(dd, axis=0)
    ha = rng.uniform(0.005, 0.02, nl)
    cnt, hsh, _ = orc.digest(o, tuple(dd), strategy=strategy, hmode=O.H_PER_SAMPLE, hs=ha)
    bc, bh = orc.brute_digest(o, ha, d=tuple(dd), strategy=strategy)
    assert np.array_equal(cnt, bc) and np.array_equal(hsh, bh)


def test_morton_quantisation_known_answers():
    # corners of the bounding box map to 0 and 2^63 - 1; a flat axis maps to 0.5
    x = np.array([0.0, 1.0, 0.5])
    y = np.array([2.0, 3.0, 2.5])
    z = np.array([-1.0, 1.0, 0.0])
    c = O.morton_codes(x, y, z)
    assert c[0] == 0
    assert c[1] == (1 << 63) - 1
    flat = O.morton_codes(x, np.full(3, 7.0), z)
    # iy = floor(2097151 * 0.5) = 1048575 for every particle
    iy = 1048575
    spread = sum(((iy >> b) & 1) << (3 * b + 1) for b in range(21))
    assert all((int(v) & int(0x2492492492492492)) == spread for v in flat)
