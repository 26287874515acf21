"""The simulation's octree build (level order, straight from the sorted unique
keys: no radix tree, plan or per-level preorder passes) against the one-shot
evaluation, which builds the reference-numbered octree of the reference's
pipeline (Karras tree, radix_to_octree plan, materialisation) and lays out
the same traversal records from it.

Both builds must give the same octree (node count, walk counts) and the same
traversal records, which the walks turn into bit-identical accelerations:
FP64 plain form per target, mixed form per target group (the same target
groups on both trees).  The tree export of a simulation (rebuilt in the
reference numbering from the step's leaf groups) must equal the one-shot
export.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _particles(m, x, y, z):
    from nbb.ics import ParticleData

    n = len(m)
    return ParticleData(np.asarray(m, float), np.asarray(x, float), np.asarray(y, float),
                        np.asarray(z, float), np.zeros(n), np.zeros(n), np.zeros(n))


def _case(name):
    from nbb import ics

    rng = np.random.Generator(np.random.Philox(11))
    if name == "single":
        return _particles([2.0], [3.0], [4.0], [5.0])
    if name == "pair":
        return _particles([1.0, 2.0], [0.0, 1.0], [0.0, 0.5], [0.0, -0.25])
    if name == "coincident":
        return _particles(np.ones(37), np.full(37, 3.5), np.full(37, -4.0), np.full(37, 8.25))
    if name == "duplicates":
        pts = rng.uniform(-1, 1, (41, 3))
        pick = rng.integers(0, 41, 5000)
        return _particles(rng.uniform(0.5, 1.5, 5000), *pts[pick].T)
    if name == "two_clusters":
        a = 1e-4 * rng.standard_normal((3, 2000))
        a[:, 1000:] += 100.0
        return _particles(np.ones(2000), *a)
    if name == "deep_pairs":
        # pairs about one quantisation cell apart: leaves at the deepest levels
        base = rng.uniform(-1, 1, (3, 500))
        x = np.concatenate([base[0], base[0] + 2.2 / 1024])
        return _particles(np.ones(1000), x, np.tile(base[1], 2), np.tile(base[2], 2))
    if name == "plummer":
        return ics.plummer(100_000, seed=3)
    if name == "disk":
        return ics.disk_bulge(65_536, seed=1)
    if name == "blobs":
        return ics.blobs(50_000, seed=2)
    raise KeyError(name)


CASES = ["single", "pair", "coincident", "duplicates", "two_clusters", "deep_pairs", "plummer", "disk",
         "blobs"]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision", [0, 1])
def test_level_order_build_equals_reference_numbered_build(nbb_mod, case, precision):
    p = _case(case)
    theta, soft = 0.5, 0.05
    ax, ay, az, st = nbb_mod.compute_accelerations(p, theta, soft, 1.0, precision=precision, stats=True)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, theta, soft, 1.0, precision=precision,
                                                         group_size=32 if precision else 0))
    sim.initialize()
    ss = sim.stats()
    assert ss.n_octree_nodes == st.n_octree_nodes
    assert ss.n_groups == st.n_groups
    assert ss.interactions == st.interactions
    if precision:
        assert ss.mac_tests == st.mac_tests
    for a, b in zip(sim.accelerations(), (ax, ay, az)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case", ["duplicates", "plummer"])
def test_simulation_tree_export_after_steps(nbb_mod, case):
    p = _case(case)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.05, 1.0))
    sim.initialize()
    sim.run(2)
    got = sim.export_tree()
    # the state after the steps, evaluated in one shot, builds the same tree
    # (the last step's tree was built after its drift; the closing kick moves
    # no particle)
    x, y, z, _, _, _ = sim.download()
    q = _particles(p.mass, x, y, z)
    _, _, _, ref = nbb_mod.compute_accelerations(q, 0.5, 0.05, 1.0, export=True)
    assert got["n_octree"] == ref["n_octree"] and got["n_groups"] == ref["n_groups"]
    for k, v in ref.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(got[k], v), k


def test_level_order_build_on_an_ensemble(nbb_mod):
    """Systems above the 30 Morton bits: levels above the system roots."""
    from nbb import ics

    ens = ics.plummer_ensemble(n_systems=9, seed=5, n_min=200, n_max=3000)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.02, 1.0)
    sim = nbb_mod.EnsembleSimulation(ens, cfg)
    sim.initialize()
    acc = np.stack(sim.accelerations())
    off = ens.offsets
    for k in range(len(off) - 1):
        sl = slice(int(off[k]), int(off[k + 1]))
        part = _particles(ens.particles.mass[sl], ens.particles.x[sl], ens.particles.y[sl], ens.particles.z[sl])
        soft = 0.02 if ens.softening is None else float(ens.softening[k])
        ref = np.stack(nbb_mod.compute_accelerations(part, 0.5, soft, 1.0))
        assert np.array_equal(acc[:, sl], ref), k


@pytest.mark.parametrize("case,group_size", [("plummer", 64), ("disk", 32), ("blobs", 128)])
def test_node_cache_depth_changes_no_result(nbb_mod, case, group_size):
    """The mixed walk's shared-memory node cache (the top 0, 1 or 2 levels
    below the root, loaded per block from the step's table) relocates records
    only: accelerations and walk counts equal the uncached walk's."""
    p = _case(case)
    outs = []
    for depth in (0, 1, 2):
        sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=nbb_mod.PRECISION_MIXED,
                                                             group_size=group_size, cache_depth=depth))
        sim.initialize()
        sim.run(2)
        st = sim.stats()
        assert st.cache_depth == depth and st.stack_overflow == 0
        outs.append((sim.download() + sim.accelerations(), st.interactions, st.mac_tests))
    for got, inter, tests in outs[1:]:
        assert inter == outs[0][1] and tests == outs[0][2]
        for a, b in zip(got, outs[0][0]):
            assert np.array_equal(a, b)


def test_node_cache_depth_tuned_and_validated(nbb_mod):
    p = _case("plummer")
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=nbb_mod.PRECISION_MIXED))
    sim.initialize()
    assert sim.stats().cache_depth in (0, 1, 2)
    for bad in (-2, 3):
        with pytest.raises(nbb_mod.InvalidArgument):
            nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=nbb_mod.PRECISION_MIXED,
                                                           cache_depth=bad))
