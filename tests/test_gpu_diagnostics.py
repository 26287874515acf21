"""Conserved-quantity monitor (nbb_sim_diagnostics) against plain numpy sums
and an all-pairs potential computed here, plus the physics it must show:
virial equilibrium of a Plummer sphere and conservation in a two-body orbit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _direct_potential(p, g, eps):
    x = np.stack([p.x, p.y, p.z], axis=1)
    w = 0.0
    for i in range(len(p)):
        r = np.sqrt(np.sum((x - x[i]) ** 2, axis=1) + eps * eps)
        r[i] = np.inf
        w += p.mass[i] * np.sum(p.mass / r)
    return -0.5 * g * w


def test_moments_match_numpy(nbb_mod):
    from nbb import ics

    p = ics.plummer(20000, seed=41)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0))
    d = sim.diagnostics(nbb_mod.POTENTIAL_NONE)
    x = np.stack([p.x, p.y, p.z]); v = np.stack([p.vx, p.vy, p.vz])
    assert np.isclose(d["mass"], p.mass.sum(), rtol=1e-14)
    assert np.allclose(d["center_of_mass"], (p.mass * x).sum(1) / p.mass.sum(), rtol=0, atol=1e-14)
    assert np.allclose(d["momentum"], (p.mass * v).sum(1), rtol=0, atol=1e-14)
    assert np.allclose(d["angular_momentum"], (p.mass * np.cross(x.T, v.T).T).sum(1), rtol=0, atol=1e-13)
    assert np.isclose(d["kinetic_energy"], 0.5 * np.sum(p.mass * (v ** 2).sum(0)), rtol=1e-13)
    assert d["potential_energy"] == 0.0


def test_potential_direct_and_tree(nbb_mod):
    from nbb import ics

    p = ics.plummer(3000, seed=42)
    w = _direct_potential(p, 1.0, 0.01)
    for theta in (0.0, 0.5):
        sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, theta, 0.01, 1.0))
        sim.initialize()
        dd = sim.diagnostics(nbb_mod.POTENTIAL_DIRECT)
        dt = sim.diagnostics(nbb_mod.POTENTIAL_TREE)
        assert np.isclose(dd["potential_energy"], w, rtol=1e-12)
        assert np.isclose(dt["potential_energy"], w, rtol=1e-12 if theta == 0.0 else 1e-3)
        assert dt["total_energy"] == dt["kinetic_energy"] + dt["potential_energy"]
        again = sim.diagnostics(nbb_mod.POTENTIAL_TREE)
        assert again["potential_energy"] == dt["potential_energy"]  # fixed summation order


def test_plummer_sphere_is_in_virial_equilibrium(nbb_mod):
    from nbb import ics

    p = ics.plummer(65536, seed=43)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0))
    d = sim.diagnostics(nbb_mod.POTENTIAL_TREE)
    assert abs(2.0 * d["kinetic_energy"] / abs(d["potential_energy"]) - 1.0) < 0.05
    # Plummer: W = -3 pi / 32 G M^2 / a (the r < 10a truncation and softening shift it slightly)
    assert abs(d["potential_energy"] / (-3.0 * np.pi / 32.0) - 1.0) < 0.03


def test_two_body_orbit_conserves_energy_and_momentum(nbb_mod):
    from nbb import ics

    # equal masses 0.5 on a circular orbit of separation 1 (G = 1): angular
    # speed 1, each body at radius 0.5 moves at 0.5
    p = ics.ParticleData(np.array([0.5, 0.5]), np.array([-0.5, 0.5]), np.zeros(2), np.zeros(2),
                         np.zeros(2), np.array([-0.5, 0.5]), np.zeros(2))
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.0, 1.0))
    sim.initialize()
    mon = nbb_mod.ConservationMonitor(sim, nbb_mod.POTENTIAL_DIRECT)
    mon.record()
    for _ in range(20):
        sim.run(100)
        mon.record()
    dr = mon.drift()
    assert dr["steps"] == 2000
    assert dr["energy"] < 1e-5
    assert np.linalg.norm(mon.records[-1]["momentum"]) < 1e-14
    assert dr["angular_momentum"] < 1e-12


def test_ensemble_diagnostics(nbb_mod):
    from nbb import ics

    ens = ics.plummer_ensemble(6, seed=44, n_min=500, n_max=3000)
    sim = nbb_mod.EnsembleSimulation(ens, nbb_mod.SimulationConfig(1e-3, 0.5, 0.0, 1.0))
    d = sim.diagnostics(nbb_mod.POTENTIAL_TREE)
    assert np.isclose(d["mass"], ens.particles.mass.sum(), rtol=1e-14)
    assert d["potential_energy"] < 0.0
    with pytest.raises(nbb_mod.InvalidArgument):
        sim.diagnostics(nbb_mod.POTENTIAL_DIRECT)


@pytest.mark.parametrize("group_size", [32, 64, 128])
def test_tree_potential_of_a_mixed_simulation(nbb_mod, group_size):
    from nbb import ics

    p = ics.plummer(3000, seed=45)
    w = _direct_potential(p, 1.0, 0.01)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.0, 0.01, 1.0, precision=nbb_mod.PRECISION_MIXED,
                                                         group_size=group_size))
    sim.initialize()
    assert np.isclose(sim.diagnostics(nbb_mod.POTENTIAL_TREE)["potential_energy"], w, rtol=1e-12)
