"""Frame capture on the GPU (nbb_sim_capture_frame) against the oracle's
restatement byte for byte, and against the reference's own capture code
(oracle/_ref, compiled from src/streaming/device_capture.cu) where it was
built."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(nbb_mod, n=5000, seed=31, types=True):
    from nbb import ics

    p = ics.plummer(n, seed=seed)
    t = np.random.default_rng(seed).integers(0, 5, n).astype(np.uint8) if types else None
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0), types=t)
    return sim, p, t


@pytest.mark.parametrize("max_particles", [0, 1000, 4999, 7, 100000])
def test_frame_equals_oracle_bytes(nbb_mod, oracle, max_particles):
    sim, p, t = _sim(nbb_mod)
    sim.initialize()
    sim.run(3)
    x, y, z = sim.download()[:3]
    frame = sim.capture_frame(max_particles, sequence=11)
    ref = oracle.frame_capture(x, y, z, t, max_particles=max_particles, sequence=11, step=3, time=sim.time())
    assert frame == ref


def test_frame_without_types_writes_unknown(nbb_mod, oracle):
    from nbb import frames

    sim, p, _ = _sim(nbb_mod, types=False)
    frame = sim.capture_frame(0)
    assert frames.read_types(frame).max() == 0
    assert frame == oracle.frame_capture(p.x, p.y, p.z, np.zeros(len(p), np.uint8))


def test_frame_equals_reference_capture(nbb_mod, oracle, tmp_path):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    sim, p, t = _sim(nbb_mod, n=3000)
    for max_particles in (0, 1000):
        frame = sim.capture_frame(max_particles, sequence=5)
        ref = oracle.ref_capture_frame(p.x, p.y, p.z, t, max_particles, 5, 0, 0.0, str(tmp_path / str(max_particles)))
        assert frame == ref


def test_frame_errors(nbb_mod):
    from nbb import ics

    p = ics.plummer(100, seed=1)
    p.x[7] = np.inf
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0))
    with pytest.raises(nbb_mod.DomainError):
        sim.capture_frame(0)
    q = ics.plummer(100, seed=2)
    bad = np.zeros(100, np.uint8)
    bad[50] = 9
    sim = nbb_mod.Simulation(q, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0), types=bad)
    with pytest.raises(nbb_mod.InvalidArgument):
        sim.capture_frame(0)
