"""Adjoint at the differentiable-rollout configuration's size and loss.

Plummer sphere N = 65536 (seed 0), theta = 0.5, eps = 0.01, dt = 1e-3,
checkpoints every 32 steps, loss = mean over particles of |x_T - x_T*|^2
where x_T* is the final state of a rollout from the same initial state with
velocities perturbed by N(0, 0.01^2) (Philox 4321).  The rollout is cut
from 1000 steps to 64 (two checkpoint segments) to keep the test within a
minute; the full 1000-step run is `bench.py --workload adjoint`.

FP64 rollout: its adjoint must match central differences of the
frozen-structure FP64 rollout (nbb_frozen_rollout, the function the adjoint
differentiates) on 64 seeded coordinates -- positions, velocities, masses --
to 1e-5 relative.  The differences use h = 1e-4 for positions and
velocities and 0.1 m for masses with a Richardson pair (h, 2h), which
removes the O(h^2) truncation term.  Steps 100x smaller leave rounding noise
in the differenced final states: with h = 1e-6 (1e-3 m) the smallest
components (a mass gradient 100x below the median) come out 2e-3 off, while
every component agrees to 5e-6 with the steps used here.

Mixed rollout: its gradient is the vector-Jacobian product of the mixed
force itself (group-box acceptance, the mixed walk's interaction lists, FP32
arithmetic) along the mixed trajectory.  Its position and velocity components
are held to the FP64 finite differences within MIXED_L2_BAR relative L2.
Its mass components are not: a mass derivative through a cell's monopole
misses the cell's dipole-order term, so the mass gradients of two tree
forces with different acceptance sets (the mixed form opens more cells)
differ by a few percent.  Both tree gradients are instead held to the
all-pairs FP64 adjoint (the exact gradient of the Newtonian rollout) under a
linear loss: the mixed one within MIXED_DIRECT_BAR per kind and no farther
than the plain tree gradient (with a 1.5x margin).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 65536
STEPS = 64
EVERY = 32
COORDS = 64
FD_RTOL = 1e-5
MIXED_L2_BAR = 1e-2
MIXED_DIRECT_BAR = 5e-2


def _perturbed(p, which, k, h):
    from nbb import ics

    arrs = {f: np.array(getattr(p, f), dtype=np.float64) for f in ("mass", "x", "y", "z", "vx", "vy", "vz")}
    arrs[which][k] += h
    return ics.ParticleData(*(arrs[f] for f in ("mass", "x", "y", "z", "vx", "vy", "vz")))


def _coords(n, count, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    kinds = ["x", "y", "z", "vx", "vy", "vz", "mass"]
    return [(kinds[i % len(kinds)], int(rng.integers(n))) for i in range(count)]


def _pick(grads, coords):
    gm, gx, gv = grads
    axis = {"x": 0, "y": 1, "z": 2}
    out = []
    for which, k in coords:
        if which == "mass":
            out.append(gm[k])
        elif which in axis:
            out.append(gx[axis[which], k])
        else:
            out.append(gv[axis[which[1]], k])
    return np.array(out)


@pytest.fixture(scope="module")
def config4(nbb_mod):
    from nbb import ics

    p = ics.plummer(N, seed=0)
    rng = np.random.Generator(np.random.Philox(4321))
    pt = ics.ParticleData(p.mass, p.x, p.y, p.z, p.vx + 0.01 * rng.standard_normal(N),
                          p.vy + 0.01 * rng.standard_normal(N), p.vz + 0.01 * rng.standard_normal(N))
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    tsim = nbb_mod.Simulation(pt, cfg)
    tsim.initialize()
    tsim.run(STEPS)
    target = np.stack(tsim.download()[:3])
    tsim.close()
    coords = _coords(N, COORDS, 777)
    # frozen-structure central differences with a Richardson pair: each loss
    # difference is formed from the difference of the two final states
    hs = np.array([0.1 * float(p.mass[k]) if w == "mass" else 1e-4 for w, k in coords])
    copies = []
    for (w, k), h in zip(coords, hs):
        for s in (h, -h, 2 * h, -2 * h):
            copies.append(_perturbed(p, w, k, s))
    fin = nbb_mod.frozen_rollout(p, cfg, copies, STEPS)[:, :3]

    def dloss(a, b):
        return np.sum((a - b) * (a + b - 2.0 * target)) / N

    d1 = np.array([dloss(fin[4 * i], fin[4 * i + 1]) / (2 * hs[i]) for i in range(COORDS)])
    d2 = np.array([dloss(fin[4 * i + 2], fin[4 * i + 3]) / (4 * hs[i]) for i in range(COORDS)])
    fd = (4.0 * d1 - d2) / 3.0
    return p, target, coords, fd


def _gradient(nbb_mod, p, target, precision):
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=precision))
    sim.initialize()
    sim.rollout(STEPS, EVERY)
    xf = np.stack(sim.download()[:3])
    grads = sim.backward(2.0 * (xf - target) / N)
    sim.close()
    return grads


def test_fp64_rollout_adjoint_matches_finite_differences(nbb_mod, config4):
    p, target, coords, fd = config4
    ad = _pick(_gradient(nbb_mod, p, target, nbb_mod.PRECISION_FP64), coords)
    rel = np.abs(ad - fd) / np.abs(fd)
    assert np.all(np.isfinite(ad)) and np.all(np.abs(fd) > 0)
    assert np.max(rel) <= FD_RTOL, list(zip(coords, rel))


def test_mixed_rollout_gradient_within_bar_of_finite_differences(nbb_mod, config4):
    p, target, coords, fd = config4
    ad = _pick(_gradient(nbb_mod, p, target, nbb_mod.PRECISION_MIXED), coords)
    assert np.all(np.isfinite(ad))
    phase = np.array([w != "mass" for w, _ in coords])
    assert np.linalg.norm(ad[phase] - fd[phase]) <= MIXED_L2_BAR * np.linalg.norm(fd[phase])


def test_tree_gradients_against_all_pairs_adjoint(nbb_mod, config4):
    p = config4[0]
    rng = np.random.Generator(np.random.Philox(99))
    wx = rng.standard_normal((3, N)) / N
    wv = rng.standard_normal((3, N)) / N
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    _, dm, dx, dv = nbb_mod.direct_rollout_adjoint(p, cfg, STEPS, wx, wv)
    err = {}
    for prec in (nbb_mod.PRECISION_FP64, nbb_mod.PRECISION_MIXED):
        sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=prec))
        sim.initialize()
        sim.rollout(STEPS, EVERY)
        gm, gx, gv = sim.backward(wx, wv)
        sim.close()
        err[prec] = [np.linalg.norm(a - b) / np.linalg.norm(b) for a, b in ((gm, dm), (gx, dx), (gv, dv))]
    for kind, (e_plain, e_mixed) in enumerate(zip(err[nbb_mod.PRECISION_FP64], err[nbb_mod.PRECISION_MIXED])):
        assert e_mixed <= MIXED_DIRECT_BAR, (kind, err)
        assert e_mixed <= 1.5 * e_plain, (kind, err)
