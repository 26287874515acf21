"""Hand-written adjoint of the Barnes-Hut rollout.

The differentiated function is the FP64 leapfrog rollout whose force keeps,
at every step, the tree and each target's accepted-node and opened-leaf sets
of the unperturbed trajectory.  Central finite differences of exactly that
function come from nbb_frozen_rollout; the adjoint must match them to 1e-5
relative.  With theta = 0 the tree force is the direct sum, so the tree
adjoint must equal the independent direct-sum adjoint.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plummer(nbb_mod, n, seed):
    from nbb import ics

    return ics.plummer(n, seed=seed)


def _linear_loss_weights(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((3, n)), rng.standard_normal((3, n))


def _perturbed(p, which, k, h):
    from nbb import ics

    arrs = {f: np.array(getattr(p, f), dtype=np.float64) for f in ("mass", "x", "y", "z", "vx", "vy", "vz")}
    arrs[which][k] += h
    return ics.ParticleData(arrs["mass"], arrs["x"], arrs["y"], arrs["z"], arrs["vx"], arrs["vy"], arrs["vz"])


def _frozen_fd(nbb_mod, p, cfg, steps, coords, wx, wv):
    """Central differences of L = <wx, x_T> + <wv, v_T> under the frozen
    structure, one pair of perturbed copies per coordinate."""
    copies, hs = [], []
    for which, k in coords:
        h = 1e-6 if which != "mass" else 1e-3 * float(p.mass[k])
        hs.append(h)
        copies.append(_perturbed(p, which, k, h))
        copies.append(_perturbed(p, which, k, -h))
    final = nbb_mod.frozen_rollout(p, cfg, copies, steps)
    # difference the final states before the weighted sum: the loss itself is
    # O(100) and would cancel to its rounding level
    d = final[0::2] - final[1::2]
    dl = np.einsum("qan,an->q", d[:, :3], wx) + np.einsum("qan,an->q", d[:, 3:], wv)
    return dl / (2.0 * np.array(hs))


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


def _coords(n, seed, count=12):
    rng = np.random.default_rng(seed)
    kinds = ["x", "y", "z", "vx", "vy", "vz", "mass"]
    return [(kinds[i % len(kinds)], int(rng.integers(n))) for i in range(count)]


def test_frozen_replay_without_perturbation_follows_the_plain_trajectory(nbb_mod):
    p = _plummer(nbb_mod, 3000, 11)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    final = nbb_mod.frozen_rollout(p, cfg, [p], 8)[0]
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.run(8)
    ref = np.stack(sim.download())
    # node centres of mass come from a different summation order than the
    # build's octant-ordered combination: rounding-level differences only
    assert np.max(np.abs(final - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("theta,steps,every", [(0.5, 20, 6), (0.5, 9, 32), (0.8, 16, 4)])
def test_tree_adjoint_matches_frozen_finite_differences(nbb_mod, theta, steps, every):
    n = 2048
    p = _plummer(nbb_mod, n, 5)
    cfg = nbb_mod.SimulationConfig(1e-3, theta, 0.01, 1.0)
    wx, wv = _linear_loss_weights(n, 6)
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.rollout(steps, every)
    grads = sim.backward(wx, wv)
    coords = _coords(n, 7)
    fd = _frozen_fd(nbb_mod, p, cfg, steps, coords, wx, wv)
    ad = _pick(grads, coords)
    rel = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-12)
    assert np.max(rel) <= 1e-5, (coords, ad, fd)


def test_theta_zero_tree_adjoint_equals_direct_sum_adjoint(nbb_mod):
    n = 1024
    p = _plummer(nbb_mod, n, 9)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.0, 0.01, 1.0)
    wx, wv = _linear_loss_weights(n, 10)
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.rollout(12, 5)
    gm, gx, gv = sim.backward(wx, wv)
    final, dm, dx, dv = nbb_mod.direct_rollout_adjoint(p, cfg, 12, wx, wv)
    assert np.allclose(np.stack(sim.download()), final, rtol=0, atol=1e-12)
    for a, b in ((gm, dm), (gx, dx), (gv, dv)):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))


def test_direct_adjoint_matches_finite_differences(nbb_mod):
    n = 512
    p = _plummer(nbb_mod, n, 12)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    wx, wv = _linear_loss_weights(n, 13)
    _, gm, gx, gv = nbb_mod.direct_rollout_adjoint(p, cfg, 15, wx, wv)
    coords = _coords(n, 14, count=10)
    fd = []
    for which, k in coords:
        h = 1e-6 if which != "mass" else 1e-3 * float(p.mass[k])
        lp = nbb_mod.direct_rollout_adjoint(_perturbed(p, which, k, h), cfg, 15, wx, wv)[0]
        lm = nbb_mod.direct_rollout_adjoint(_perturbed(p, which, k, -h), cfg, 15, wx, wv)[0]
        d = lp - lm
        fd.append((np.sum(d[:3] * wx) + np.sum(d[3:] * wv)) / (2 * h))
    ad = _pick((gm, gx, gv), coords)
    assert np.max(np.abs(ad - np.array(fd)) / np.abs(np.array(fd))) <= 1e-5


def test_tree_adjoint_close_to_direct_adjoint_at_theta_half(nbb_mod):
    n = 4096
    p = _plummer(nbb_mod, n, 15)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    wx, wv = _linear_loss_weights(n, 16)
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.rollout(10, 4)
    gm, gx, gv = sim.backward(wx, wv)
    _, dm, dx, dv = nbb_mod.direct_rollout_adjoint(p, cfg, 10, wx, wv)
    for a, b in ((gx, dx), (gv, dv)):
        assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b)
    assert np.linalg.norm(gm - dm) <= 1e-2 * np.linalg.norm(dm)


@pytest.mark.parametrize("precision", [0, 1])
def test_backward_restores_state_and_is_repeatable(nbb_mod, precision):
    n = 5000
    p = _plummer(nbb_mod, n, 17)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=precision)
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.rollout(10, 3)
    after = np.stack(sim.download())
    ref = nbb_mod.Simulation(p, cfg)
    ref.initialize()
    ref.run(10)
    assert np.array_equal(after, np.stack(ref.download()))
    wx, wv = _linear_loss_weights(n, 18)
    g1 = sim.backward(wx, wv)
    assert np.array_equal(np.stack(sim.download()), after)
    g2 = sim.backward(wx, wv)
    for a, b in zip(g1, g2):
        # cotangents of shared nodes are added atomically: rounding-level order effects
        assert np.allclose(a, b, rtol=1e-12, atol=1e-15 * np.max(np.abs(b)))
    sim.step()  # the handle keeps stepping from the rollout's final state
    ref.step()
    assert np.array_equal(np.stack(sim.download()), np.stack(ref.download()))


def test_mixed_theta_zero_adjoint_equals_direct_sum_adjoint(nbb_mod):
    """The mixed form's VJP (FP32, on the mixed walk's lists) at theta = 0,
    where the walk opens every cell: the exact all-pairs adjoint up to FP32
    rounding."""
    n = 1024
    p = _plummer(nbb_mod, n, 9)
    wx, wv = _linear_loss_weights(n, 10)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.0, 0.01, 1.0, precision=nbb_mod.PRECISION_MIXED))
    sim.initialize()
    sim.rollout(12, 5)
    gm, gx, gv = sim.backward(wx, wv)
    _, dm, dx, dv = nbb_mod.direct_rollout_adjoint(p, nbb_mod.SimulationConfig(1e-3, 0.0, 0.01, 1.0), 12, wx, wv)
    for a, b in ((gm, dm), (gx, dx), (gv, dv)):
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b)


@pytest.mark.parametrize("group_size", [0, 32, 64, 128])
def test_mixed_rollout_gradient_close_to_fp64_gradient(nbb_mod, group_size):
    # the mixed rollout is differentiated with the mixed force's own VJP
    # (group-box acceptance, FP32): its gradient differs from the plain
    # form's at the level of the mixed form's force error; the backward pass
    # rebuilds one-warp target groups whatever group size the walk uses
    n = 4096
    p = _plummer(nbb_mod, n, 19)
    wx, wv = _linear_loss_weights(n, 20)
    out = []
    for prec in (0, 1):
        sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=prec,
                                                             group_size=group_size if prec else 0))
        sim.initialize()
        sim.rollout(12, 4)
        out.append(sim.backward(wx, wv))
    for a, b in zip(out[0], out[1]):
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(a)


def test_zero_step_rollout_gradient_is_the_cotangent(nbb_mod):
    p = _plummer(nbb_mod, 300, 21)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0))
    sim.initialize()
    sim.rollout(0, 4)
    wx, wv = _linear_loss_weights(300, 22)
    gm, gx, gv = sim.backward(wx, wv)
    assert np.array_equal(gx, wx) and np.array_equal(gv, wv) and not np.any(gm)


def test_adjoint_errors(nbb_mod):
    p = _plummer(nbb_mod, 200, 23)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0))
    with pytest.raises(nbb_mod.LogicError):
        sim.rollout(3, 2)
    sim.initialize()
    with pytest.raises(nbb_mod.LogicError):
        sim.backward(np.zeros((3, 200)))
    with pytest.raises(nbb_mod.InvalidArgument):
        sim.rollout(3, 0)


def test_torch_wrapper_mse_loss(nbb_mod):
    torch = pytest.importorskip("torch")
    from nbb.autograd import rollout

    n = 2048
    p = _plummer(nbb_mod, n, 24)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    target = np.stack([p.x, p.y, p.z]) + 0.01
    m = torch.tensor(p.mass, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(np.stack([p.x, p.y, p.z]), requires_grad=True)
    v = torch.tensor(np.stack([p.vx, p.vy, p.vz]), requires_grad=True)
    xf, vf = rollout(m, x, v, cfg, 10, 4)
    loss = ((xf - torch.from_numpy(target)) ** 2).sum(dim=0).mean()
    loss.backward()
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.rollout(10, 4)
    xf2 = np.stack(sim.download()[:3])
    gm, gx, gv = sim.backward(2.0 * (xf2 - target) / n)
    assert np.allclose(m.grad.numpy(), gm, rtol=1e-11, atol=1e-14 * np.max(np.abs(gm)))
    assert np.allclose(x.grad.numpy(), gx, rtol=1e-11, atol=1e-14 * np.max(np.abs(gx)))
    assert np.allclose(v.grad.numpy(), gv, rtol=1e-11, atol=1e-14 * np.max(np.abs(gv)))
