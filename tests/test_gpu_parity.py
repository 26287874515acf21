"""Parity of the CUDA library (through its C ABI) with the oracle and with
fixtures produced by the reference itself.

Bar: integer outputs (Morton keys, permutation, leaf groups, Karras tree,
plan, octree topology) bit-exact; plain-FP64 floating-point outputs within
1e-12 relative (FLOAT_RTOL; per element |a-b| / max(|b|, rms(b))).  The mixed
form is held to RMS relative force error <= 1e-3 against FP64 direct
summation.
"""
import math

import numpy as np
import pytest

from conftest import golden
from test_oracle_golden import FLOAT_FIELDS, INT_FIELDS, five_node_tree, rel_err

pytestmark = pytest.mark.gpu

FLOAT_RTOL = 1e-12
MIXED_RMS_BOUND = 1e-3


def _compare(out, ref, ints=INT_FIELDS, floats=FLOAT_FIELDS, rtol=FLOAT_RTOL, bitwise=True):
    """Integers bit-exact; floats within rtol (the bar), and -- because the
    plain path performs the reference's operations in the reference's order
    with the same roundings -- also bit-identical when `bitwise`."""
    assert out["n_groups"] == int(ref["n_groups"])
    assert out["n_octree"] == int(ref["n_octree"])
    assert np.array_equal(out["box"], np.asarray(ref["box"]))
    for k in ints:
        assert np.array_equal(out[k], np.asarray(ref[k])), k
    worst = {}
    for k in floats:
        worst[k] = rel_err(out[k], ref[k])
        assert worst[k] <= rtol, (k, worst[k])
        if bitwise:
            assert np.array_equal(out[k], np.asarray(ref[k])), (k, "not bit-identical", worst[k])
    return worst


def _gpu_pipeline(nbb, p, theta, soft, g, precision=0):
    ax, ay, az, ex, st = nbb.compute_accelerations(p, theta, soft, g, precision=precision,
                                                   export=True, stats=True)
    ex.update(ax=ax, ay=ay, az=az)
    return ex, st


# ------------------------------------------------ bit-exact vs oracle ---

@pytest.mark.parametrize("recipe,n,theta,soft", [
    ("plummer", 4096, 0.5, 0.01),
    ("plummer", 4096, 0.0, 0.01),
    ("plummer", 50000, 0.5, 0.01),
    ("disk", 20000, 0.5, 0.005),
    ("blobs", 20000, 0.3, 1e-3),
    ("blobs", 20000, 0.7, 1e-3),
])
def test_pipeline_matches_oracle(nbb_mod, oracle, recipe, n, theta, soft):
    from nbb import ics

    p = {"plummer": lambda: ics.plummer(n, seed=0), "disk": lambda: ics.disk_bulge(n, seed=1),
         "blobs": lambda: ics.blobs(n, seed=2)}[recipe]()
    out, st = _gpu_pipeline(nbb_mod, p, theta, soft, 1.0)
    ref = oracle.pipeline(p.mass, p.x, p.y, p.z, theta=theta, soft=soft, g=1.0)
    _compare(out, ref)
    assert st.interactions == ref["interactions"]


@pytest.mark.parametrize("name", ["plummer4096", "blobs4096", "dupes1024"])
def test_pipeline_matches_reference_fixture(nbb_mod, name):
    from nbb.ics import ParticleData

    f = golden(name)
    p = ParticleData(*(f["in_" + k] for k in ("mass", "x", "y", "z", "vx", "vy", "vz")))
    out, _ = _gpu_pipeline(nbb_mod, p, float(f["theta"]), float(f["soft"]), float(f["g"]))
    _compare(out, f)


def test_radix_tree_matches_reference_fixture(nbb_mod):
    f = golden("radix_random")
    sizes = sorted({int(k.split("_")[1]) for k in f if k.startswith("keys_")})
    for n in sizes:
        t = nbb_mod.radix_tree(f[f"keys_{n}"])
        for k in ("left", "right", "rangeFirst", "rangeLast", "prefixLength", "parent"):
            assert np.array_equal(t[k], f[f"{k}_{n}"]), (n, k)


# -------------------------------------------------------- edge cases ---

def _particles(m, x, y, z):
    from nbb.ics import ParticleData

    n = len(m)
    return ParticleData(np.asarray(m, float), np.asarray(x, float), np.asarray(y, float),
                        np.asarray(z, float), np.zeros(n), np.zeros(n), np.zeros(n))


@pytest.mark.parametrize("case", ["single", "pair", "coincident", "zero_mass", "duplicates",
                                  "line", "two_clusters", "odd_sizes"])
def test_edge_cases_match_oracle(nbb_mod, oracle, case):
    rng = np.random.Generator(np.random.Philox(5))
    if case == "single":
        p = _particles([2.0], [3.0], [4.0], [5.0])
    elif case == "pair":
        p = _particles([1.0, 2.0], [0.0, 1.0], [0.0, 0.5], [0.0, -0.25])
    elif case == "coincident":
        p = _particles(np.ones(37), np.full(37, 3.5), np.full(37, -4.0), np.full(37, 8.25))
    elif case == "zero_mass":
        m = rng.uniform(0, 1, 3000)
        m[::3] = 0.0
        p = _particles(m, *rng.standard_normal((3, 3000)))
    elif case == "duplicates":
        pts = rng.uniform(-1, 1, (41, 3))
        pick = rng.integers(0, 41, 5000)
        p = _particles(rng.uniform(0.5, 1.5, 5000), *pts[pick].T)
    elif case == "line":
        p = _particles(np.ones(777), np.linspace(-3, 3, 777), np.zeros(777), np.zeros(777))
    elif case == "two_clusters":
        a = 1e-4 * rng.standard_normal((3, 2000))
        a[:, 1000:] += 100.0
        p = _particles(np.ones(2000), *a)
    else:
        p = _particles(np.ones(4097), *rng.standard_normal((3, 4097)))
    soft = 0.05
    out, _ = _gpu_pipeline(nbb_mod, p, 0.5, soft, 1.0)
    ref = oracle.pipeline(p.mass, p.x, p.y, p.z, theta=0.5, soft=soft, g=1.0)
    _compare(out, ref)


def test_non_finite_positions_raise_domain_error(nbb_mod):
    p = _particles([1.0, 1.0], [0.0, math.nan], [0.0, 1.0], [0.0, 1.0])
    with pytest.raises(nbb_mod.DomainError):
        nbb_mod.compute_accelerations(p, 0.5, 0.01, 1.0)


def test_singular_interaction_reports_error(nbb_mod):
    # barnes_hut.cu:67-69: coincident distinct particles with zero softening
    p = _particles([1.0, 1.0, 1.0], [0.0, 0.0, 1.0], [0.0, 0.0, 1.0], [0.0, 0.0, 1.0])
    with pytest.raises(nbb_mod.DeviceError) as e:
        nbb_mod.compute_accelerations(p, 0.5, 0.0, 1.0)
    assert e.value.code == 806
    with pytest.raises(nbb_mod.DeviceError):
        nbb_mod.compute_accelerations(p, 0.5, 0.0, 1.0, precision=nbb_mod.PRECISION_MIXED)


@pytest.mark.parametrize("bad", [dict(theta=-0.1), dict(theta=math.nan), dict(softening=-1.0),
                                 dict(g=0.0)])
def test_invalid_parameters_rejected(nbb_mod, bad):
    p = _particles([1.0, 1.0], [0.0, 1.0], [0.0, 1.0], [0.0, 1.0])
    args = dict(theta=0.5, softening=0.01, g=1.0)
    args.update(bad)
    with pytest.raises(nbb_mod.InvalidArgument):
        nbb_mod.compute_accelerations(p, args["theta"], args["softening"], args["g"])


# ------------------------------------------------ function-level API ---

def test_function_level_known_answers(nbb_mod):
    t = nbb_mod.radix_tree([0x00000000, 0x40000000, 0x80000000, 0xC0000000])
    assert t["left"].tolist() == [5, 0, 2] and t["right"].tolist() == [6, 1, 3]
    assert t["parent"].tolist() == [5, 5, 6, 6, -1, 4, 4]
    assert t["prefixLength"].tolist() == [0, 1, 1]
    for keys, levels, counts, offsets, m in [([0], [1], [1], [0], 2),
                                             ([0, 1 << 29], [1, 1, 0], [1, 1, 0], [0, 1, 2], 3),
                                             ([0, 1 << 26], [2, 2, 1], [1, 1, 1], [0, 1, 2], 4),
                                             ([7, 7, 7, 7], [1], [1], [0], 2)]:
        r = nbb_mod.octree_from_keys(keys)
        assert r["plan_level"].tolist() == levels and r["plan_count"].tolist() == counts
        assert r["plan_offset"].tolist() == offsets and r["n_octree"] == m
    with pytest.raises(nbb_mod.DeviceError):
        nbb_mod.octree_from_keys([0, 0x40000000])


def test_octree_from_keys_matches_oracle(nbb_mod, oracle):
    bg = np.random.MT19937()
    bg._legacy_seeding(0xC0FFEE)
    keys = np.sort(bg.random_raw(257).astype(np.uint32) & 0x3FFFFFFF)
    for i in range(7, 257, 17):
        keys[i] = keys[i - 1]
    r = nbb_mod.octree_from_keys(keys)
    o = oracle.octree_from_keys(keys)
    assert np.array_equal(r["uniq"], o["groups"][0])
    assert np.array_equal(r["plan_offset"], o["plan"]["edgeNodeOffset"])
    assert np.array_equal(r["children"], o["octree"]["children"])
    assert np.array_equal(r["oprefix"], o["octree"]["prefix"])
    assert np.array_equal(r["ocount"], o["octree"]["particleCount"])


def test_hand_built_octrees(nbb_mod):
    t = five_node_tree()
    P = nbb_mod.BarnesHutParameters
    m, x, zero = np.array([1.0, 2.0, 3.0]), np.array([-10.0, 10.0, 12.0]), np.zeros(3)
    idx = np.arange(3, dtype=np.uint32)
    ax, _, _ = nbb_mod.computeBarnesHutAcceleration(t, idx, m, x, zero, zero, 3, P(1.0, 0.0, 1.0))
    assert abs(ax[0] - 5.0 / (21.2 * 21.2)) < 1e-12
    ax, _, _ = nbb_mod.computeBarnesHutAcceleration(t, idx, m, x, zero, zero, 3, P(0.85, 0.0, 1.0))
    assert abs(ax[0] - (2.0 / 400.0 + 3.0 / 484.0)) < 1e-12
    ax, ay, az = nbb_mod.computeBarnesHutAcceleration(t, idx, m, x, zero, zero, 3, P(0.0, 0.1, 1.0),
                                                      particle_order="morton")
    from test_oracle_golden import direct_reference

    e = direct_reference(m, x, zero, zero, 1.0, 0.1)
    assert np.allclose(np.stack([ax, ay, az]), e, rtol=0, atol=1e-12)


def test_leapfrog_analytic(nbb_mod):
    import torch

    dev = torch.device("cuda:0")
    T = lambda v: torch.tensor([v], dtype=torch.float64, device=dev)  # noqa: E731
    x, y, z, vx, vy, vz = T(1.0), T(-2.0), T(3.0), T(4.0), T(5.0), T(-6.0)
    ax, ay, az = T(2.0), T(-4.0), T(1.0)
    dt = 0.25
    nbb_mod.leapfrog_kick_drift(x, y, z, vx, vy, vz, ax, ay, az, dt)
    nbb_mod.leapfrog_kick(vx, vy, vz, ax, ay, az, dt)
    assert abs(x.item() - (1.0 + 4.0 * dt + dt * dt)) < 1e-14
    assert abs(y.item() - (-2.0 + 5.0 * dt - 2.0 * dt * dt)) < 1e-14
    assert abs(z.item() - (3.0 - 6.0 * dt + 0.5 * dt * dt)) < 1e-14
    assert abs(vx.item() - 4.5) < 1e-14 and abs(vy.item() - 4.0) < 1e-14
    assert abs(vz.item() + 5.75) < 1e-14
    with pytest.raises(nbb_mod.InvalidArgument):
        nbb_mod.leapfrog_kick(vx, vy, vz, ax, ay, az, 0.0)


def test_direct_sum_matches_oracle(nbb_mod, oracle):
    from nbb import ics

    p = ics.plummer(3000, seed=4)
    tg = np.arange(0, 3000, 7, dtype=np.int32)
    a = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    e = np.stack(oracle.direct_accel(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    assert np.array_equal(a, e)


def test_direct_sum_over_source_chunks_matches_oracle(nbb_mod, oracle):
    # few targets over many sources: partial sums of consecutive source
    # ranges, added in range order -- the sequential sum up to rounding
    from nbb import ics

    p = ics.plummer(200_000, seed=14)
    tg = np.sort(np.random.default_rng(3).choice(200_000, 1000, replace=False)).astype(np.int32)
    a = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    e = np.stack(oracle.direct_accel(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    assert rel_err(a, e) <= 1e-13


# --------------------------------------------------- simulation API ---

def test_simulation_trajectory_matches_oracle(nbb_mod, oracle):
    from nbb import ics

    p = ics.plummer(4096, seed=0)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    sim = nbb_mod.Simulation(p, cfg)
    sim.initialize()
    sim.run(10)
    assert sim.step_number() == 10 and abs(sim.time() - 0.01) < 1e-15
    got = sim.download() + sim.accelerations()
    ref = oracle.simulate(p, 10, 1e-3, 0.5, 0.01, 1.0)
    for name, a, b in zip(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"), got, ref):
        assert rel_err(a, b) <= FLOAT_RTOL, name


def test_simulation_matches_reference_trajectory(nbb_mod):
    from nbb.ics import ParticleData

    f = golden("plummer4096")
    p = ParticleData(*(f["in_" + k] for k in ("mass", "x", "y", "z", "vx", "vy", "vz")))
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(float(f["traj_dt"]), float(f["theta"]),
                                                         float(f["soft"]), float(f["g"])))
    sim.initialize()
    sim.run(int(f["traj_steps"]))
    got = sim.download() + sim.accelerations()
    for name, a in zip(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"), got):
        assert rel_err(a, f["traj_" + name]) <= FLOAT_RTOL, name


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replay_equals_eager(nbb_mod, precision):
    from nbb import ics

    p = ics.plummer(20000, seed=3)
    outs = []
    for graph in (True, False):
        sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=precision,
                                                             use_graph=graph))
        sim.initialize()
        sim.run(3)
        outs.append(sim.download())
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision,graph", [(0, True), (1, True), (1, False)])
def test_host_step_equals_upload_step_download(nbb_mod, precision, graph):
    import torch
    from nbb import ics

    p = ics.plummer(30000, seed=5)
    cfg = nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=precision, use_graph=graph)
    a = nbb_mod.Simulation(p, cfg)
    b = nbb_mod.Simulation(p, cfg)
    with pytest.raises(nbb_mod.LogicError):
        b.step_host(p)
    a.initialize()
    b.initialize()
    state = [np.array(v) for v in p.arrays()[1:]]
    pinned = [torch.from_numpy(v.copy()).pin_memory() for v in state]
    for k in range(3):
        # mass goes up on the first step only; the pinned copy on the last
        mass = p.mass if k == 0 else None
        a.upload(mass=mass, x=state[0], y=state[1], z=state[2], vx=state[3], vy=state[4], vz=state[5])
        a.step()
        want = a.download()
        if k < 2:
            got = b.step_host(mass=mass, x=state[0], y=state[1], z=state[2], vx=state[3], vy=state[4],
                              vz=state[5])
        else:
            for t, v in zip(pinned, state):
                t.copy_(torch.from_numpy(v))
            b.step_host(x=pinned[0], y=pinned[1], z=pinned[2], vx=pinned[3], vy=pinned[4], vz=pinned[5],
                        out=pinned)
            got = [t.numpy() for t in pinned]
        for w, g in zip(want, got):
            assert np.array_equal(w, g)
        state = [np.array(w) for w in want]
    assert b.step_number() == a.step_number() == 3
    assert b.time() == a.time()
    # outputs may be left out; the device state still advances
    b.step_host(x=state[0], y=state[1], z=state[2], vx=state[3], vy=state[4], vz=state[5],
                out=[None] * 6)
    a.upload(x=state[0], y=state[1], z=state[2], vx=state[3], vy=state[4], vz=state[5])
    a.step()
    for w, g in zip(a.download(), b.download()):
        assert np.array_equal(w, g)


def test_simulation_state_machine(nbb_mod):
    p = _particles([1.0, 1.0], [0.0, 1.0], [0.0, 0.0], [0.0, 0.0])
    cfg = nbb_mod.SimulationConfig(0.25, 0.5, 0.01, 1.0)
    sim = nbb_mod.Simulation(p, cfg)
    with pytest.raises(nbb_mod.LogicError):
        sim.step()
    with pytest.raises(nbb_mod.LogicError):
        sim.run(1)
    sim.initialize()
    assert sim.time() == 0.0 and sim.step_number() == 0
    with pytest.raises(nbb_mod.LogicError):
        sim.initialize()
    for bad in (dict(time_step=0.0), dict(time_step=-1.0), dict(time_step=math.nan), dict(theta=-0.1),
                dict(theta=math.nan), dict(softening=-0.01), dict(softening=math.nan)):
        c = dict(time_step=1.0, theta=0.5, softening=0.01)
        c.update(bad)
        with pytest.raises(nbb_mod.InvalidArgument):
            nbb_mod.Simulation(p, nbb_mod.SimulationConfig(c["time_step"], c["theta"], c["softening"]))


def test_free_particle(nbb_mod):
    # simulation_test.cu:162-190
    p = _particles([1.0], [0.5], [-1.0], [2.0])
    p.vx[:], p.vy[:], p.vz[:] = 0.1, 0.2, -0.3
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(0.25, 0.6, 0.03))
    sim.initialize()
    sim.run(4)
    x, y, z, vx, vy, vz = sim.download()
    assert abs(x[0] - 0.6) < 1e-12 and abs(y[0] + 0.8) < 1e-12 and abs(z[0] - 1.7) < 1e-12
    assert (vx[0], vy[0], vz[0]) == (0.1, 0.2, -0.3)


def test_two_body_orbit(nbb_mod):
    # simulation_test.cu:195-283 (SI G, the Simulation default)
    g, mass, sep, steps = nbb_mod.G_SI, 1.0e10, 1.0, 128
    v = math.sqrt(g * mass / (2.0 * sep))
    period = 2.0 * math.pi / (2.0 * v / sep)
    p = _particles([mass, mass], [-0.5, 0.5], [0.0, 0.0], [0.0, 0.0])
    p.vy[:] = [-v, v]
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(period / steps, 0.5, 0.0))
    sim.initialize()
    e0 = mass * v * v - g * mass * mass / sep
    emax = drift = 0.0
    for _ in range(steps):
        sim.step()
        x, y, z, vx, vy, vz = sim.download()
        d = math.dist((x[0], y[0], z[0]), (x[1], y[1], z[1]))
        ke = 0.5 * mass * float((vx ** 2 + vy ** 2 + vz ** 2).sum())
        emax = max(emax, abs((ke - g * mass * mass / d - e0) / e0))
        drift = max(drift, math.hypot(0.5 * (x[0] + x[1]), 0.5 * (y[0] + y[1]), 0.5 * (z[0] + z[1])))
    assert abs(sim.time() - period) < period * 1e-13
    assert emax < 5e-6 and drift < 1e-12


def test_failed_step_poisons_simulation(nbb_mod):
    p = _particles([1.0, 1.0, 1.0], [0.0, 0.0, 1.0], [0.0, 0.0, 1.0], [0.0, 0.0, 1.0])
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(0.1, 0.5, 0.0, 1.0))
    with pytest.raises(nbb_mod.DeviceError):
        sim.initialize()
    with pytest.raises(nbb_mod.LogicError):
        sim.step()


# ------------------------------------------------------ mixed form ---

def _rms_rel(approx, exact):
    rel = np.linalg.norm(approx - exact, axis=0) / np.linalg.norm(exact, axis=0)
    return float(np.sqrt(np.mean(rel ** 2)))


@pytest.mark.parametrize("recipe,n,theta,soft", [("plummer", 65536, 0.5, 0.01),
                                                 ("plummer", 262144, 0.5, 0.01),
                                                 ("disk", 65536, 0.5, 0.005),
                                                 ("blobs", 65536, 0.3, 1e-3),
                                                 ("blobs", 65536, 0.5, 1e-3),
                                                 ("blobs", 65536, 0.7, 1e-3)])
def test_mixed_force_error(nbb_mod, recipe, n, theta, soft):
    """Mixed-form force error against FP64 direct summation: never worse
    than the reference's own per-target acceptance test in FP64 (the group
    test is stricter, FP32 rounding is far below the Barnes-Hut error), and
    within the headline's RMS bound of 1e-3 on the Plummer sphere."""
    from nbb import ics

    p = {"plummer": lambda: ics.plummer(n, seed=0), "disk": lambda: ics.disk_bulge(n, seed=1),
         "blobs": lambda: ics.blobs(n, seed=2)}[recipe]()
    rng = np.random.Generator(np.random.Philox(99))
    tg = np.sort(rng.choice(n, 2048, replace=False)).astype(np.int32)
    exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, soft, targets=tg))
    mixed = np.stack(nbb_mod.compute_accelerations(p, theta, soft, 1.0, precision=nbb_mod.PRECISION_MIXED))
    plain = np.stack(nbb_mod.compute_accelerations(p, theta, soft, 1.0))
    rms_mixed = _rms_rel(mixed[:, tg], exact)
    rms_plain = _rms_rel(plain[:, tg], exact)
    assert rms_mixed <= rms_plain * 1.05, (rms_mixed, rms_plain)
    if recipe == "plummer":
        assert rms_mixed <= MIXED_RMS_BOUND, rms_mixed


@pytest.mark.parametrize("group_size", [32, 64, 128])
def test_mixed_group_sizes(nbb_mod, group_size):
    """Every warp group size (one, two or four targets per lane) stays within the
    headline bound and match each other to the Barnes-Hut error level."""
    from nbb import ics

    n = 65536
    p = ics.plummer(n, seed=0)
    rng = np.random.Generator(np.random.Philox(99))
    tg = np.sort(rng.choice(n, 2048, replace=False)).astype(np.int32)
    exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0,
                                                         precision=nbb_mod.PRECISION_MIXED,
                                                         group_size=group_size))
    sim.initialize()
    assert sim.stats().group_size == group_size
    a = np.stack(sim.accelerations())[:, tg]
    assert _rms_rel(a, exact) <= MIXED_RMS_BOUND


@pytest.mark.parametrize("group_size", [32, 64, 128])
def test_mixed_group_sizes_on_a_disk(nbb_mod, group_size):
    """A thin disk with a sparse halo, every group size pinned: target groups
    stay compact (sparse outer cells split instead of forming one wide group),
    and the mixed error stays at the plain form's Barnes-Hut level."""
    from nbb import ics

    n = 65536
    p = ics.disk_bulge(n, seed=1)
    rng = np.random.Generator(np.random.Philox(98))
    tg = np.sort(rng.choice(n, 2048, replace=False)).astype(np.int32)
    exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.005, targets=tg))
    plain = np.stack(nbb_mod.compute_accelerations(p, 0.5, 0.005, 1.0))[:, tg]
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.005, 1.0,
                                                         precision=nbb_mod.PRECISION_MIXED,
                                                         group_size=group_size))
    sim.initialize()
    st = sim.stats()
    assert st.group_size == group_size and st.stack_overflow == 0
    a = np.stack(sim.accelerations())[:, tg]
    assert _rms_rel(a, exact) <= _rms_rel(plain, exact) * 1.05


def test_mixed_autotuned_group_size(nbb_mod):
    from nbb import ics

    p = ics.plummer(32768, seed=1)
    sizes = []
    for _ in range(2):
        sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0,
                                                             precision=nbb_mod.PRECISION_MIXED))
        sim.initialize()
        sizes.append(sim.stats().group_size)
    assert sizes[0] in (32, 64, 128) and sizes[0] == sizes[1]  # cached per process and size
    with pytest.raises(nbb_mod.InvalidArgument):
        nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, 0.5, 0.01, 1.0, group_size=48))


@pytest.mark.parametrize("theta", [0.2, 0.5])
@pytest.mark.parametrize("group_size", [32, 64, 128])
def test_mixed_walk_tests_every_node(nbb_mod, theta, group_size):
    """Plummer N=2^20: the mixed walk never accepts a node for lack of stack
    space (the shared-memory stack spills to its global extension instead),
    also at theta = 0.2, whose deep, wide walks fill the shared part."""
    from nbb import ics

    n = 1 << 20
    p = ics.plummer(n, seed=0)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(1e-3, theta, 0.01, 1.0,
                                                         precision=nbb_mod.PRECISION_MIXED,
                                                         group_size=group_size))
    sim.initialize()
    st = sim.stats()
    assert st.stack_overflow == 0
    rng = np.random.Generator(np.random.Philox(7))
    tg = np.sort(rng.choice(n, 1024, replace=False)).astype(np.int32)
    exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    a = np.stack(sim.accelerations())[:, tg]
    assert _rms_rel(a, exact) <= (2e-4 if theta < 0.3 else MIXED_RMS_BOUND)


def test_mixed_theta_zero_is_direct(nbb_mod):
    from nbb import ics

    p = ics.plummer(8192, seed=6)
    exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.01))
    ax, ay, az = nbb_mod.compute_accelerations(p, 0.0, 0.01, 1.0, precision=nbb_mod.PRECISION_MIXED)
    rel = np.linalg.norm(np.stack([ax, ay, az]) - exact, axis=0) / np.linalg.norm(exact, axis=0)
    assert float(np.sqrt(np.mean(rel ** 2))) < 1e-5


# ----------------------------------------- full size: size-free checks ---

def test_full_size_invariants(nbb_mod):
    """Plummer N=2^20: keys sorted, permutation complete, groups and leaves
    partition the particles, octree parent/level/prefix consistent, and the
    plain accelerations on a sample agree with direct summation to the
    Barnes-Hut error level."""
    from nbb import ics

    n = 1 << 20
    p = ics.plummer(n, seed=0)
    out, st = _gpu_pipeline(nbb_mod, p, 0.5, 0.01, 1.0)
    keys, idx = out["keys"], out["idx"]
    assert np.all(keys[1:] >= keys[:-1])
    assert np.array_equal(np.sort(idx), np.arange(n, dtype=np.uint32))
    eq = keys[1:] == keys[:-1]
    assert np.all(idx[1:][eq] > idx[:-1][eq])  # stable
    g = out["n_groups"]
    assert out["gcount"].sum() == n and out["gfirst"][0] == 0
    assert np.array_equal(out["gfirst"][1:], np.cumsum(out["gcount"])[:-1])
    m = out["n_octree"]
    ch = out["children"].reshape(m, 8)
    par, lev = out["oparent"], out["olevel"]
    kids = np.nonzero(ch >= 0)
    c = ch[kids]
    assert np.all(par[c] == kids[0]) and np.all(lev[c] == lev[kids[0]] + 1)
    leaf = out["ocount"] > 0
    assert leaf.sum() == g and out["ocount"].sum() == n
    assert np.all((ch[leaf] < 0).all(axis=1))
    assert np.isclose(out["mass"][0], p.mass.sum(), rtol=1e-12)
    rng = np.random.Generator(np.random.Philox(1))
    tg = np.sort(rng.choice(n, 1024, replace=False)).astype(np.int32)
    exact = np.stack(nbb_mod.compute_direct_accelerations(p.mass, p.x, p.y, p.z, 1.0, 0.01, targets=tg))
    a = np.stack([out["ax"], out["ay"], out["az"]])[:, tg]
    rel = np.linalg.norm(a - exact, axis=0) / np.linalg.norm(exact, axis=0)
    assert float(np.sqrt(np.mean(rel ** 2))) < 1e-2


def test_bounded_wait_reports_timeout_and_context_survives(nbb_mod):
    """A look-back whose predecessor never publishes ends with
    NBB_ERR_TIMEOUT instead of hanging, and the GPU stays usable."""
    import time

    lib = nbb_mod.load()
    t0 = time.time()
    st = lib.nbb_selftest_bounded_wait()
    assert st == 6, lib.nbb_last_error_message()  # NBB_ERR_TIMEOUT
    assert time.time() - t0 < 60
    assert b"gave up" in lib.nbb_last_error_message()
    from nbb import ics

    p = ics.plummer(2000, seed=1)
    ax, _, _ = nbb_mod.compute_accelerations(p, 0.5, 0.01, 1.0)
    assert np.all(np.isfinite(ax))
