"""Pin the CPU oracle to the reference.

Two kinds of evidence: the known answers of the reference's own test-suite
(transcribed expectations, each cited), and fixtures produced by running the
reference's CUDA sources (tests/golden/*.npz, see make_golden.py).  Integer
outputs must match bit-exactly; floating-point outputs to 1e-12 relative
(the oracle follows the reference's operation order, so in practice they are
bit-identical as well).
"""
import math

import numpy as np
import pytest

from conftest import golden

FLOAT_RTOL = 1e-12


# ------------------------------------------------------------------ bbox ---

def test_bbox_known_answers(oracle):
    # tests/unit/cuda/globalbounding_test.cu:60-72
    b = oracle.bbox([-2.0, 4.0, 1.0], [10.0, 14.0, -2.0], [-1.0, 0.0, 5.0])
    assert b.tolist() == pytest.approx([1.0, 6.0, 2.0, 17.6], rel=1e-15)
    # :74-89
    b = oracle.bbox([-2.0, 4.0], [10.0, 14.0], [-1.0, 5.0])
    assert b.tolist() == pytest.approx([1.0, 12.0, 2.0, 6.6], rel=1e-15)
    # :91-102 coincident particles get side 1
    assert oracle.bbox([3.5, 3.5], [-4.0, -4.0], [8.25, 8.25]).tolist() == [3.5, -4.0, 8.25, 1.0]
    # :104-120
    b = oracle.bbox([10.0, 14.0], [20.0, 22.0], [30.0, 31.0])
    assert b.tolist() == pytest.approx([12.0, 21.0, 30.5, 4.4], rel=1e-15)


@pytest.mark.parametrize("bad", [math.nan, math.inf, -math.inf])
def test_bbox_rejects_non_finite(oracle, bad):
    # globalbounding_test.cu:122-160 (std::domain_error)
    with pytest.raises(oracle.OracleError) as e:
        oracle.bbox([0.0, bad], [0.0, 1.0], [0.0, 1.0])
    assert e.value.code == -2
    with pytest.raises(oracle.OracleError):
        oracle.bbox([], [], [])


# ---------------------------------------------------------------- morton ---

def _reference_morton(x, y, z):
    """morton_test.cu:114-219 restated in numpy."""
    x, y, z = (np.asarray(a, float) for a in (x, y, z))
    c = [(a.min() + a.max()) * 0.5 for a in (x, y, z)]
    side = 1.1 * max(a.max() - a.min() for a in (x, y, z))
    side = 1.0 if side == 0.0 else side

    def q(a, cc):
        nrm = (a - (cc - side * 0.5)) / side
        return np.clip(nrm * 1024.0, 0.0, 1023.0).astype(np.uint32)

    def expand(v):
        v = v.astype(np.uint64) & 0x3FF
        v = (v | (v << 16)) & 0x030000FF
        v = (v | (v << 8)) & 0x0300F00F
        v = (v | (v << 4)) & 0x030C30C3
        v = (v | (v << 2)) & 0x09249249
        return v.astype(np.uint32)

    keys = (expand(q(x, c[0])) << 2) | (expand(q(y, c[1])) << 1) | expand(q(z, c[2]))
    order = np.argsort(keys, kind="stable")
    return keys[order], order.astype(np.uint32)


def test_morton_matches_reference_restatement(oracle):
    # morton_test.cu:223-246
    x, y, z = [0.8, -1.0, 0.1, 1.0, -0.4], [-0.2, 0.9, 0.0, -1.0, 0.3], [1.0, -0.7, 0.2, 0.4, -1.0]
    keys, idx = oracle.morton(x, y, z)
    ek, ei = _reference_morton(x, y, z)
    assert np.array_equal(keys, ek) and np.array_equal(idx, ei)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)


def test_morton_stability_and_corners(oracle):
    # morton_test.cu:248-262: equal keys keep input order
    keys, idx = oracle.morton([1.0, 1.0, 0.0], [1.0, 1.0, 0.0], [1.0, 1.0, 0.0])
    assert idx.tolist() == [2, 0, 1] and keys[1] == keys[2]
    # :264-290 opposite corners
    keys, idx = oracle.morton([0.0, 1.0], [0.0, 1.0], [0.0, 1.0])
    assert idx.tolist() == [0, 1] and keys[0] < keys[1]
    # :353-384 coincident particles
    keys, idx = oracle.morton([3.5] * 4, [-4.0] * 4, [8.25] * 4)
    assert len(set(keys.tolist())) == 1 and idx.tolist() == [0, 1, 2, 3]


def test_morton_random_against_restatement(oracle):
    rng = np.random.Generator(np.random.Philox(11))
    for n in (1, 2, 17, 1000, 20000):
        x, y, z = rng.standard_normal((3, n))
        keys, idx = oracle.morton(x, y, z)
        ek, ei = _reference_morton(x, y, z)
        assert np.array_equal(keys, ek) and np.array_equal(idx, ei)


# ----------------------------------------------------------- leaf groups ---

@pytest.mark.parametrize("keys,uniq,first,count", [
    # morton_leaf_groups_test.cu:277-320
    ([42], [42], [0], [1]),
    ([2, 5, 8, 10], [2, 5, 8, 10], [0, 1, 2, 3], [1, 1, 1, 1]),
    ([7, 7, 7, 7], [7], [0], [4]),
    ([1, 1, 2, 4, 4, 4, 9], [1, 2, 4, 9], [0, 2, 3, 6], [2, 1, 3, 1]),
    ([0, 0, 1, 0xFFFFFFFF, 0xFFFFFFFF], [0, 1, 0xFFFFFFFF], [0, 2, 3], [2, 1, 2]),
])
def test_leaf_groups_known_answers(oracle, keys, uniq, first, count):
    u, f, c = oracle.leaf_groups(np.array(keys, np.uint32))
    assert u.tolist() == uniq and f.tolist() == first and c.tolist() == count


# ------------------------------------------------------------ radix tree ---

def test_radix_tree_exact_topologies(oracle):
    # tree_builder_test.cu:550-577
    t = oracle.radix_tree([0x00000000, 0x80000000])
    assert t["left"].tolist() == [0] and t["right"].tolist() == [1]
    assert t["parent"].tolist() == [2, 2, -1]
    assert t["rangeFirst"].tolist() == [0] and t["rangeLast"].tolist() == [1]
    assert t["prefixLength"].tolist() == [0]
    t = oracle.radix_tree([0x00000000, 0x40000000, 0x80000000, 0xC0000000])
    assert t["left"].tolist() == [5, 0, 2] and t["right"].tolist() == [6, 1, 3]
    assert t["parent"].tolist() == [5, 5, 6, 6, -1, 4, 4]
    assert t["rangeFirst"].tolist() == [0, 0, 2] and t["rangeLast"].tolist() == [3, 1, 3]
    assert t["prefixLength"].tolist() == [0, 1, 1]


def _validate_radix(keys, t):
    """Structural validation in the spirit of tree_builder_test.cu:243-386:
    every node reached once from the root, leaf ranges contiguous, prefix
    lengths equal the longest common prefix of the range ends."""
    n = len(keys)

    def lcp(i, j):
        if keys[i] != keys[j]:
            return 32 - int(keys[i] ^ keys[j]).bit_length()
        return 32 + 32 - int(i ^ j).bit_length()

    seen = np.zeros(2 * n - 1, int)
    stack = [n if n > 1 else 0]
    while stack:
        v = stack.pop()
        seen[v] += 1
        if v >= n:
            i = v - n
            a, b = t["rangeFirst"][i], t["rangeLast"][i]
            assert 0 <= a < b < n
            assert t["prefixLength"][i] == lcp(a, b)
            for c in (t["left"][i], t["right"][i]):
                assert t["parent"][c] == v
                stack.append(c)
    assert np.all(seen == 1)


def test_radix_tree_random_with_duplicates(oracle):
    # tree_builder_test.cu:602-642 sizes, duplicates every 11 keys
    for n in (3, 5, 7, 16, 31, 64, 257, 5000):
        bg = np.random.MT19937()
        bg._legacy_seeding(0xC0FFEE + n)
        keys = np.sort(bg.random_raw(n).astype(np.uint32))
        for i in range(5, n, 11):
            keys[i] = keys[i - 1]
        _validate_radix(keys, oracle.radix_tree(keys))


def test_radix_tree_duplicates_only(oracle):
    # tree_builder_test.cu:579-589 (six equal keys)
    keys = np.full(6, 7, np.uint32)
    _validate_radix(keys, oracle.radix_tree(keys))


# ------------------------------------------------------------------ plan ---

@pytest.mark.parametrize("keys,levels,counts,offsets,m", [
    # radix_to_octree_test.cu:310-352
    ([0], [1], [1], [0], 2),
    ([0, 1 << 29], [1, 1, 0], [1, 1, 0], [0, 1, 2], 3),
    ([0, 1 << 26], [2, 2, 1], [1, 1, 1], [0, 1, 2], 4),
    ([7, 7, 7, 7], [1], [1], [0], 2),
])
def test_plan_known_answers(oracle, keys, levels, counts, offsets, m):
    r = oracle.octree_from_keys(np.array(keys, np.uint32))
    assert r["plan"]["radixLevel"].tolist() == levels
    assert r["plan"]["edgeNodeCount"].tolist() == counts
    assert r["plan"]["edgeNodeOffset"].tolist() == offsets
    assert r["plan"]["nOctreeNodes"] == m


def test_plan_rejects_keys_outside_30_bits(oracle):
    # radix_to_octree_test.cu (RejectsKeysOutsideThirtyBitLayout): code 1
    with pytest.raises(oracle.OracleError) as e:
        oracle.octree_from_keys(np.array([0, 0x40000000], np.uint32))
    assert e.value.code == 1


# ---------------------------------------------------------- sparse octree ---

def _validate_octree(keys, r):
    """sparse_octree_test.cu:100-325 in spirit: every child one level below
    its parent, prefixes consistent, each group one leaf holding its range."""
    o = r["octree"]
    uniq, first, count = r["groups"]
    m = o["nNodes"]
    ch = o["children"].reshape(m, 8)
    assert o["parent"][0] == -1 and o["level"][0] == 0
    leaves = 0
    for v in range(m):
        kids = ch[v][ch[v] >= 0]
        for oc in range(8):
            c = ch[v][oc]
            if c < 0:
                continue
            assert o["parent"][c] == v and o["level"][c] == o["level"][v] + 1
            shift = 30 - 3 * o["level"][c]
            assert (o["prefix"][c] >> shift) & 7 == oc
        if o["particleCount"][v] > 0:
            leaves += 1
            assert kids.size == 0
        else:
            assert kids.size > 0
    assert leaves == uniq.size
    assert o["particleCount"].sum() == len(keys)


@pytest.mark.parametrize("keys", [
    # sparse_octree_test.cu:564-601
    [0], [7, 7, 7, 7], [0, 1 << 29], [0, 1 << 26],
    [0, 1 << 23, 1 << 26, 1 << 29, (1 << 29) | (1 << 26)],
])
def test_sparse_octree_cases(oracle, keys):
    k = np.array(keys, np.uint32)
    _validate_octree(k, oracle.octree_from_keys(k))


def test_sparse_octree_random(oracle):
    # sparse_octree_test.cu:523-556: N=257, 30-bit keys, duplicates every 17
    bg = np.random.MT19937()
    bg._legacy_seeding(0xC0FFEE)
    keys = np.sort(bg.random_raw(257).astype(np.uint32) & 0x3FFFFFFF)
    for i in range(7, 257, 17):
        keys[i] = keys[i - 1]
    _validate_octree(keys, oracle.octree_from_keys(keys))


# -------------------------------------------------------------- geometry ---

def test_geometry_known_answers(oracle):
    box = oracle.bbox([-10.0, 10.0], [-10.0, 10.0], [-10.0, 10.0])
    # octree_geometry_test.cu:120-160 root
    cx, cy, cz, h = oracle.octree_geometry([0], [0], box)
    assert (cx[0], cy[0], cz[0], h[0]) == (0.0, 0.0, 0.0, 11.0)
    # :162-229 opposite level-one octants
    cx, cy, cz, h = oracle.octree_geometry([0, 1, 1], [0, 0, 7 << 27], box)
    assert (cx[1], cy[1], cz[1], h[1]) == (-5.5, -5.5, -5.5, 5.5)
    assert (cx[2], cy[2], cz[2], h[2]) == (5.5, 5.5, 5.5, 5.5)
    # :243-311 deep prefix path 5, 2, 7
    prefix = (5 << 27) | (2 << 24) | (7 << 21)
    cx, cy, cz, h = oracle.octree_geometry([0, 3], [0, prefix], box)
    assert (cx[1], cy[1], cz[1], h[1]) == (4.125, -1.375, 4.125, 1.375)


def test_geometry_rejects_invalid(oracle):
    box = oracle.bbox([-1.0, 1.0], [-1.0, 1.0], [-1.0, 1.0])
    with pytest.raises(oracle.OracleError) as e:
        oracle.octree_geometry([0, 11], [0, 0], box)
    assert e.value.code == 1
    with pytest.raises(oracle.OracleError) as e:
        oracle.octree_geometry([0, 1], [0, 1], box)
    assert e.value.code == 2


# ------------------------------------------------- hand-built BH octrees ---

def five_node_tree():
    """barnes_hut_test.cu:294-400: root -> {node1 (p0), node2 -> {node3 (p1),
    node4 (p2)}}, particles at x = -10, 10, 12 with masses 1, 2, 3."""
    ch = np.full(5 * 8, -1, np.int32)
    ch[0 * 8 + 0], ch[0 * 8 + 7], ch[2 * 8 + 0], ch[2 * 8 + 7] = 1, 2, 3, 4
    return dict(
        children=ch, parent=np.array([-1, 0, 0, 2, 2], np.int32),
        firstParticle=np.array([-1, 0, -1, 1, 2], np.int32),
        particleCount=np.array([0, 1, 0, 1, 1], np.int32),
        mass=np.array([6.0, 1.0, 5.0, 2.0, 3.0]),
        comX=np.array([46.0 / 6.0, -10.0, 11.2, 10.0, 12.0]), comY=np.zeros(5), comZ=np.zeros(5),
        centerX=np.array([0.0, -8.0, 8.0, 10.0, 12.0]), centerY=np.zeros(5), centerZ=np.zeros(5),
        halfSize=np.array([16.0, 8.0, 8.0, 1.0, 1.0]), nParticles=3)


def direct_reference(m, x, y, z, g, soft):
    """barnes_hut_test.cu:73-137 restated."""
    n = len(m)
    a = np.zeros((3, n))
    for t in range(n):
        for s in range(n):
            if s == t:
                continue
            d = np.array([x[s] - x[t], y[s] - y[t], z[s] - z[t]])
            r2 = d @ d + soft * soft
            inv = 1.0 / math.sqrt(r2)
            a[:, t] += g * m[s] * inv ** 3 * d
    return a


def test_bh_theta_zero_matches_direct(oracle):
    t = five_node_tree()
    m, x = np.array([1.0, 2.0, 3.0]), np.array([-10.0, 10.0, 12.0])
    ax, ay, az = oracle.bh_accel(t, np.arange(3, dtype=np.uint32), m, x, np.zeros(3), np.zeros(3),
                                 0.0, 0.1, 1.0)
    e = direct_reference(m, x, np.zeros(3), np.zeros(3), 1.0, 0.1)
    assert np.allclose(np.stack([ax, ay, az]), e, rtol=0, atol=1e-12)


def test_bh_accepts_far_cluster(oracle):
    # barnes_hut_test.cu:568-781
    t = five_node_tree()
    ax, _, _ = oracle.bh_accel(t, np.arange(3, dtype=np.uint32), [1.0, 2.0, 3.0], [-10.0, 10.0, 12.0],
                               np.zeros(3), np.zeros(3), 1.0, 0.0, 1.0)
    assert abs(ax[0] - 5.0 / (21.2 * 21.2)) < 1e-12
    assert abs(ax[0] - (2.0 / 400.0 + 3.0 / 484.0)) > 1e-6


def test_bh_opens_off_centre_cluster(oracle):
    # barnes_hut_test.cu:784-1025 (theta 0.85: d > s/theta + delta rejects)
    t = five_node_tree()
    ax, _, _ = oracle.bh_accel(t, np.arange(3, dtype=np.uint32), [1.0, 2.0, 3.0], [-10.0, 10.0, 12.0],
                               np.zeros(3), np.zeros(3), 0.85, 0.0, 1.0)
    assert abs(ax[0] - (2.0 / 400.0 + 3.0 / 484.0)) < 1e-12


def test_bh_single_particle(oracle):
    # barnes_hut_test.cu:161-292
    t = dict(children=np.full(8, -1, np.int32), parent=np.array([-1], np.int32),
             firstParticle=np.array([0], np.int32), particleCount=np.array([1], np.int32),
             mass=np.array([2.0]), comX=np.array([3.0]), comY=np.array([4.0]), comZ=np.array([5.0]),
             centerX=np.array([3.0]), centerY=np.array([4.0]), centerZ=np.array([5.0]),
             halfSize=np.array([1.0]))
    ax, ay, az = oracle.bh_accel(t, np.zeros(1, np.uint32), [2.0], [3.0], [4.0], [5.0], 0.5, 1e-3, 1.0)
    assert (ax[0], ay[0], az[0]) == (0.0, 0.0, 0.0)


# ------------------------------------------------------------ integrator ---

def test_leapfrog_constant_acceleration(oracle):
    # integrator_test.cu:181-305
    dt = 0.25
    x, y, z, vx, vy, vz = oracle.kick_drift([1.0], [-2.0], [3.0], [4.0], [5.0], [-6.0], [2.0], [-4.0],
                                            [1.0], dt)
    vx, vy, vz = oracle.kick(vx, vy, vz, [2.0], [-4.0], [1.0], dt)
    assert abs(x[0] - (1.0 + 4.0 * dt + 0.5 * 2.0 * dt * dt)) < 1e-14
    assert abs(y[0] - (-2.0 + 5.0 * dt - 0.5 * 4.0 * dt * dt)) < 1e-14
    assert abs(z[0] - (3.0 - 6.0 * dt + 0.5 * dt * dt)) < 1e-14
    assert abs(vx[0] - (4.0 + 2.0 * dt)) < 1e-14
    assert abs(vy[0] - (5.0 - 4.0 * dt)) < 1e-14
    assert abs(vz[0] - (-6.0 + dt)) < 1e-14


# ------------------------------------------------------------ simulation ---

def test_free_particle_constant_velocity(oracle):
    # simulation_test.cu:162-190
    from nbb.ics import ParticleData

    p = ParticleData(np.array([1.0]), np.array([0.5]), np.array([-1.0]), np.array([2.0]),
                     np.array([0.1]), np.array([0.2]), np.array([-0.3]))
    x, y, z, vx, vy, vz, *_ = oracle.simulate(p, 4, 0.25, 0.6, 0.03, g=6.67430e-11)
    assert abs(x[0] - (0.5 + 0.1)) < 1e-12 and abs(y[0] - (-1.0 + 0.2)) < 1e-12
    assert abs(z[0] - (2.0 - 0.3)) < 1e-12
    assert (vx[0], vy[0], vz[0]) == (0.1, 0.2, -0.3)


def test_circular_two_body_orbit(oracle):
    # simulation_test.cu:195-283 with the SI constant
    from nbb.ics import ParticleData

    g, mass, sep, steps = 6.67430e-11, 1.0e10, 1.0, 128
    v = math.sqrt(g * mass / (2.0 * sep))
    period = 2.0 * math.pi / (2.0 * v / sep)
    dt = period / steps
    p = ParticleData(np.array([mass, mass]), np.array([-0.5, 0.5]), np.zeros(2), np.zeros(2),
                     np.zeros(2), np.array([-v, v]), np.zeros(2))
    e0 = mass * v * v - g * mass * mass / sep
    emax = drift = 0.0
    state = p.copy()
    for _ in range(steps):
        x, y, z, vx, vy, vz, *_ = oracle.simulate(state, 1, dt, 0.5, 0.0, g=g)
        state = ParticleData(state.mass, x, y, z, vx, vy, vz)
        d = math.dist((x[0], y[0], z[0]), (x[1], y[1], z[1]))
        ke = 0.5 * mass * float((vx ** 2 + vy ** 2 + vz ** 2).sum())
        emax = max(emax, abs((ke - g * mass * mass / d - e0) / e0))
        drift = max(drift, math.hypot(0.5 * (x[0] + x[1]), 0.5 * (y[0] + y[1]), 0.5 * (z[0] + z[1])))
    assert emax < 5e-6 and drift < 1e-12
    assert abs(state.x[0] - p.x[0]) < 3e-3 and abs(state.y[0] - p.y[0]) < 3e-3


# -------------------------------------------------- accuracy vs theta ---

@pytest.mark.parametrize("dataset", ["uniform", "clusters"])
def test_accuracy_bounds_by_theta(oracle, dataset):
    # barnes_hut_accuracy_test.cu:662-697 bounds on relative L2 error, N=256,
    # softening 0.02, G=1 (datasets regenerated with this project's seeds)
    rng = np.random.Generator(np.random.Philox(0xBADC0FFEE))
    n = 256
    if dataset == "uniform":
        pos = rng.uniform(-1.0, 1.0, (n, 3))
    else:
        centres = np.array([[-5, -5, -5], [5, -5, 5], [-5, 5, 5], [5, 5, -5]], float)
        pos = centres[np.arange(n) % 4] + 0.5 * rng.standard_normal((n, 3))
    m = rng.uniform(0.5, 1.5, n)
    x, y, z = pos.T.copy()
    e = np.stack(oracle.direct_accel(m, x, y, z, 1.0, 0.02))
    bounds = {0.0: 1e-11, 0.3: 2e-3, 0.5: 1e-2, 0.7: 2e-2, 1.0: 4e-2}
    for theta, bound in bounds.items():
        r = oracle.pipeline(m, x, y, z, theta=theta, soft=0.02, g=1.0)
        a = np.stack([r["ax"], r["ay"], r["az"]])
        rel_l2 = math.sqrt(((a - e) ** 2).sum() / (e ** 2).sum())
        assert rel_l2 < bound, (theta, rel_l2)


# ----------------------------------------- fixtures made by the reference ---

INT_FIELDS = ["keys", "idx", "uniq", "gfirst", "gcount", "left", "right", "rfirst", "rlast", "plen",
              "rparent", "plan_level", "plan_count", "plan_offset", "children", "oparent", "olevel",
              "oprefix", "ofirst", "ocount", "child_count"]
FLOAT_FIELDS = ["cx", "cy", "cz", "half", "mass", "comx", "comy", "comz", "ax", "ay", "az"]


def rel_err(a, b):
    """max |a-b| / max(|b|, rms(b)): per-element relative error with the
    reference accuracy test's floor against near-zero values."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    if b.size == 0:
        return 0.0
    floor = max(np.sqrt(np.mean(b * b)), 1e-300)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


@pytest.mark.parametrize("name", ["plummer4096", "blobs4096", "dupes1024"])
def test_oracle_matches_reference_fixture(oracle, name):
    f = golden(name)
    r = oracle.pipeline(f["in_mass"], f["in_x"], f["in_y"], f["in_z"], theta=float(f["theta"]),
                        soft=float(f["soft"]), g=float(f["g"]))
    assert r["n_groups"] == int(f["n_groups"]) and r["n_octree"] == int(f["n_octree"])
    assert np.array_equal(r["box"], f["box"])
    for k in INT_FIELDS:
        assert np.array_equal(r[k], f[k]), k
    for k in FLOAT_FIELDS:
        assert rel_err(r[k], f[k]) <= FLOAT_RTOL, (k, rel_err(r[k], f[k]))


def test_oracle_trajectory_matches_reference_fixture(oracle):
    from nbb.ics import ParticleData

    f = golden("plummer4096")
    p = ParticleData(*(f["in_" + k] for k in ("mass", "x", "y", "z", "vx", "vy", "vz")))
    out = oracle.simulate(p, int(f["traj_steps"]), float(f["traj_dt"]), float(f["theta"]),
                          float(f["soft"]), float(f["g"]))
    for k, v in zip(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"), out):
        assert rel_err(v, f["traj_" + k]) <= FLOAT_RTOL, k


def test_oracle_radix_matches_reference_fixture(oracle):
    f = golden("radix_random")
    sizes = sorted({int(k.split("_")[1]) for k in f if k.startswith("keys_")})
    assert sizes
    for n in sizes:
        t = oracle.radix_tree(f[f"keys_{n}"])
        for k in ("left", "right", "rangeFirst", "rangeLast", "prefixLength", "parent"):
            assert np.array_equal(t[k], f[f"{k}_{n}"]), (n, k)
