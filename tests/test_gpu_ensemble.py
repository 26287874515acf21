"""Ensembles of independent systems stepped together (one launch per stage).

Every system keeps its own box, keys, octree and softening, so in the FP64
plain form each system's result must equal running it alone, bit for bit;
the mixed form must stay within the Barnes-Hut error of each system's FP64
direct sum.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_ensemble(sizes, seed=3, eps_ref=0.01):
    from nbb import ics

    parts = [ics.plummer(int(k), seed=seed * 1000 + s) for s, k in enumerate(sizes)]
    offsets = np.zeros(len(sizes) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    cat = ics.ParticleData(*(np.concatenate([getattr(p, f) for p in parts])
                             for f in ("mass", "x", "y", "z", "vx", "vy", "vz")))
    eps = eps_ref * (4096.0 / np.asarray(sizes, float)) ** (1.0 / 3.0)
    return ics.Ensemble(cat, offsets, eps), parts


@pytest.mark.parametrize("sizes", [[1500, 4000, 777, 2048, 3333], list(range(40, 40 + 9 * 70, 9)),
                                   [5, 17, 64, 65, 200]])
def test_ensemble_fp64_equals_standalone_systems(nbb_mod, sizes):
    ens, parts = _small_ensemble(sizes)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.0, 1.0)
    sim = nbb_mod.EnsembleSimulation(ens, cfg)
    sim.initialize()
    a0 = sim.accelerations()
    sim.run(3)
    state = sim.download()
    for k, p in enumerate(parts):
        lo, hi = ens.offsets[k], ens.offsets[k + 1]
        single = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, float(ens.softening[k]), 1.0))
        single.initialize()
        b0 = single.accelerations()
        for a, b in zip(a0, b0):
            assert np.array_equal(a[lo:hi], b), k
        single.run(3)
        for a, b in zip(state, single.download()):
            assert np.array_equal(a[lo:hi], b), k


def test_ensemble_mixed_error_per_system(nbb_mod):
    ens, parts = _small_ensemble([3000, 8000, 1200, 20000])
    sim = nbb_mod.EnsembleSimulation(ens, nbb_mod.SimulationConfig(
        1e-3, 0.5, 0.0, 1.0, precision=nbb_mod.PRECISION_MIXED))
    sim.initialize()
    a = np.stack(sim.accelerations())
    for k, p in enumerate(parts):
        lo, hi = ens.offsets[k], ens.offsets[k + 1]
        exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0,
                                                              float(ens.softening[k])))
        plain = np.stack(nbb_mod.compute_accelerations(p, 0.5, float(ens.softening[k]), 1.0))
        rel = np.linalg.norm(a[:, lo:hi] - exact, axis=0) / np.linalg.norm(exact, axis=0)
        relp = np.linalg.norm(plain - exact, axis=0) / np.linalg.norm(exact, axis=0)
        assert np.sqrt(np.mean(rel ** 2)) <= np.sqrt(np.mean(relp ** 2)) * 1.05, k


def test_ensemble_512_systems_graph_steps(nbb_mod):
    from nbb import ics

    ens = ics.plummer_ensemble(512, seed=4, n_min=64, n_max=2048)
    for prec in (nbb_mod.PRECISION_FP64, nbb_mod.PRECISION_MIXED):
        sim = nbb_mod.EnsembleSimulation(ens, nbb_mod.SimulationConfig(1e-3, 0.5, 0.0, 1.0, precision=prec))
        sim.initialize()
        sim.run(2)
        x = sim.download()[0]
        assert np.all(np.isfinite(x))
        st = sim.stats()
        assert st.interactions > 0


def test_ensemble_rejects_bad_layouts(nbb_mod):
    ens, _ = _small_ensemble([100, 200])
    bad = ens.__class__(ens.particles, np.array([0, 150, 299], dtype=np.int64), ens.softening)
    with pytest.raises(nbb_mod.InvalidArgument):
        nbb_mod.EnsembleSimulation(bad, nbb_mod.SimulationConfig(1e-3, 0.5, 0.0, 1.0))
    bad = ens.__class__(ens.particles, np.array([0, 300, 300], dtype=np.int64), ens.softening)
    with pytest.raises(nbb_mod.InvalidArgument):
        nbb_mod.EnsembleSimulation(bad, nbb_mod.SimulationConfig(1e-3, 0.5, 0.0, 1.0))
