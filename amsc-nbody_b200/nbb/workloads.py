"""Measurements of the secondary workloads (one JSON object each).

  disk      disk + bulge, N = 2^20, eps = 0.005, dt = 5e-4, 100 steps: FP64 plain
            and mixed step times, force error of both on 4096 seeded targets
  blobs     64 Gaussian blobs, N = 2^22, eps = 1e-3, dt = 1e-4, 20 steps, for
            theta in {0.3, 0.5, 0.7}: step times and force errors per theta
  ensemble  512 Plummer spheres, N log-uniform in [1024, 131072], per-system
            eps = 0.01 (4096 / N)^(1/3), theta = 0.5, dt = 1e-3, 50 steps: one
            segmented graph step for all systems against one simulation per
            system; interactions/s and per-step latency
  adjoint   Plummer N = 65536, theta = 0.5, eps = 0.01, dt = 1e-3, 1000 steps,
            checkpoints every 32, loss = mean squared distance of the final
            positions to a target rollout (velocities perturbed by N(0, 0.01^2)):
            forward / backward times of the mixed and FP64 rollouts, the
            gradients against central finite differences of the frozen-structure
            FP64 rollout on 64 seeded coordinates, and the tree adjoint against
            the FP64 direct-sum adjoint at N = 4096

Every input is synthetic and seeded (nbb.ics).  Device times are CUDA events
on the simulations' stream; force errors are against the library's FP64
direct-summation kernel.
"""
from __future__ import annotations

import time

import numpy as np

from . import _lib, api, ics

ERROR_TARGETS = 4096


def _torch():
    import torch

    return torch


def _targets(n, seed=12345, count=ERROR_TARGETS):
    rng = np.random.Generator(np.random.Philox(seed))
    return np.sort(rng.choice(n, min(count, n), replace=False)).astype(np.int32)


def force_error(p, theta, eps, precision, targets, g=1.0):
    exact = np.stack(api.compute_direct_accelerations(p.mass, p.x, p.y, p.z, g, eps, targets=targets))
    a = np.stack(api.compute_accelerations(p, theta, eps, g, precision=precision))[:, targets]
    rel = np.linalg.norm(a - exact, axis=0) / np.linalg.norm(exact, axis=0)
    return {"rms_rel": float(np.sqrt(np.mean(rel ** 2))), "max_rel": float(rel.max()),
            "targets": int(targets.size)}


def _timed_run(sim, stream, steps, warmup=3):
    """ms per step of `steps` graph-replayed steps on `stream` (CUDA events)."""
    torch = _torch()
    sim.set_stream(stream.cuda_stream)
    for _ in range(warmup):
        sim.step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def _forms(p, dt, theta, eps, steps):
    stream = _torch().cuda.Stream()
    res = {}
    for name, prec in (("mixed", _lib.PRECISION_MIXED), ("fp64", _lib.PRECISION_FP64)):
        sim = api.Simulation(p, api.SimulationConfig(dt, theta, eps, 1.0, precision=prec))
        sim.initialize()
        ms = _timed_run(sim, stream, steps)
        st = sim.stats()
        res[name] = {"ms_per_step": ms, "interactions_per_step": int(st.interactions),
                     "interactions_per_s": int(st.interactions) / (ms * 1e-3), "group_size": int(st.group_size)}
        sim.close()
    res["speedup_mixed_vs_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
    return res


def disk(steps=100):
    n = 1 << 20
    p = ics.disk_bulge(n, seed=1)
    res = _forms(p, 5e-4, 0.5, 0.005, steps)
    tg = _targets(n)
    res["force_error"] = {"mixed": force_error(p, 0.5, 0.005, _lib.PRECISION_MIXED, tg),
                          "fp64": force_error(p, 0.5, 0.005, _lib.PRECISION_FP64, tg)}
    return {"workload": "disk+bulge N=2^20 theta=0.5 eps=0.005 dt=5e-4 (seed 1)", "steps": steps, **res}


def blobs(steps=20):
    n = 1 << 22
    p = ics.blobs(n, seed=2)
    tg = _targets(n)
    out = {"workload": "64 Gaussian blobs N=2^22 eps=1e-3 dt=1e-4 (seed 2)", "steps": steps, "theta": {}}
    for theta in (0.3, 0.5, 0.7):
        res = _forms(p, 1e-4, theta, 1e-3, steps)
        res["force_error"] = {"mixed": force_error(p, theta, 1e-3, _lib.PRECISION_MIXED, tg),
                              "fp64": force_error(p, theta, 1e-3, _lib.PRECISION_FP64, tg)}
        out["theta"][str(theta)] = res
    return out


def ensemble(steps=50, n_systems=512):
    torch = _torch()
    ens = ics.plummer_ensemble(n_systems, seed=3)
    sizes = np.diff(ens.offsets)
    out = {"workload": f"{n_systems} Plummer spheres, N log-uniform in [1024, 131072] (seed 3), "
                       "eps_i = 0.01 (4096/N_i)^(1/3), theta=0.5, dt=1e-3",
           "steps": steps, "n_total": int(sizes.sum()), "n_min": int(sizes.min()), "n_max": int(sizes.max())}
    stream = torch.cuda.Stream()
    for name, prec in (("mixed", _lib.PRECISION_MIXED), ("fp64", _lib.PRECISION_FP64)):
        sim = api.EnsembleSimulation(ens, api.SimulationConfig(1e-3, 0.5, 0.0, 1.0, precision=prec))
        sim.initialize()
        ms = _timed_run(sim, stream, steps)
        st = sim.stats()
        seg = {"ms_per_step": ms, "interactions_per_step": int(st.interactions),
               "interactions_per_s": int(st.interactions) / (ms * 1e-3), "group_size": int(st.group_size)}
        sim.close()
        # one simulation per system, each replaying its own graph on the same stream
        singles = []
        for k in range(n_systems):
            lo, hi = ens.offsets[k], ens.offsets[k + 1]
            part = ics.ParticleData(*(np.ascontiguousarray(getattr(ens.particles, f)[lo:hi])
                                      for f in ("mass", "x", "y", "z", "vx", "vy", "vz")))
            s = api.Simulation(part, api.SimulationConfig(1e-3, 0.5, float(ens.softening[k]), 1.0,
                                                          precision=prec))
            s.set_stream(stream.cuda_stream)
            s.initialize()
            s.run(3)
            singles.append(s)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in singles:
            s.run(steps)
        e1.record(stream)
        e1.synchronize()
        ms1 = e0.elapsed_time(e1) / steps
        inter1 = int(sum(s.stats().interactions for s in singles))
        for s in singles:
            s.close()
        out[name] = {"segmented": seg,
                     "per_system": {"ms_per_step": ms1, "interactions_per_step": inter1,
                                    "interactions_per_s": inter1 / (ms1 * 1e-3)},
                     "speedup_segmented_vs_per_system": ms1 / ms}
    return out


def _fd_coords(n, count, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    kinds = ["x", "y", "z", "vx", "vy", "vz", "mass"]
    return [(kinds[int(rng.integers(len(kinds)))], int(rng.integers(n))) for _ in range(count)]


def _perturb(p, which, k, h):
    arrs = {f: np.array(getattr(p, f), dtype=np.float64) for f in ("mass", "x", "y", "z", "vx", "vy", "vz")}
    arrs[which][k] += h
    return ics.ParticleData(arrs["mass"], arrs["x"], arrs["y"], arrs["z"], arrs["vx"], arrs["vy"], arrs["vz"])


def _pick(gm, gx, gv, coords):
    ax = {"x": 0, "y": 1, "z": 2}
    return np.array([gm[k] if w == "mass" else (gx[ax[w], k] if w in ax else gv[ax[w[1]], k]) for w, k in coords])


def _kind_mask(coords, kind):
    names = {"position": ("x", "y", "z"), "velocity": ("vx", "vy", "vz"), "mass": ("mass",)}[kind]
    return np.array([w in names for w, _ in coords])


def adjoint(n=65536, steps=1000, every=32, fd_coords=64, fd_chunk=16, n_direct=4096, h=1e-4, h_mass=0.1):
    torch = _torch()
    p = ics.plummer(n, seed=0)
    rng = np.random.Generator(np.random.Philox(4321))
    pt = ics.ParticleData(p.mass, p.x, p.y, p.z, p.vx + 0.01 * rng.standard_normal(n),
                          p.vy + 0.01 * rng.standard_normal(n), p.vz + 0.01 * rng.standard_normal(n))
    out = {"workload": f"plummer N={n} theta=0.5 eps=0.01 dt=1e-3 steps={steps} checkpoints every {every} "
                       "(seed 0); loss = mean |x_T - x_T(target)|^2, target velocities + N(0, 0.01^2) "
                       "(Philox 4321)", "steps": steps, "checkpoint_every": every}
    stream = torch.cuda.Stream()
    grads = {}
    for name, prec in (("mixed", _lib.PRECISION_MIXED), ("fp64", _lib.PRECISION_FP64)):
        cfg = api.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=prec)
        tsim = api.Simulation(pt, cfg)
        tsim.initialize()
        tsim.run(steps)
        target = np.stack(tsim.download()[:3])
        tsim.close()
        sim = api.Simulation(p, cfg)
        sim.set_stream(stream.cuda_stream)
        sim.initialize()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.rollout(steps, every)
        e1.record(stream)
        e1.synchronize()
        xf = np.stack(sim.download()[:3])
        t0 = time.perf_counter()
        gm, gx, gv = sim.backward(2.0 * (xf - target) / n)
        wall_b = time.perf_counter() - t0
        fwd_ms = e0.elapsed_time(e1)
        out[name] = {"loss": float(np.mean(np.sum((xf - target) ** 2, axis=0))),
                     "forward_ms": fwd_ms, "backward_ms": wall_b * 1e3,
                     "backward_over_forward": wall_b * 1e3 / fwd_ms}
        grads[name] = (gm, gx, gv, target)
        sim.close()
    # central differences of the frozen-structure FP64 rollout (the function
    # the adjoint differentiates) with a Richardson pair (h, 2h) that removes
    # the O(h^2) term; each loss difference is formed from the difference of
    # the two final states, not from two rounded losses
    coords = _fd_coords(n, fd_coords, 777)
    cfg64 = api.SimulationConfig(1e-3, 0.5, 0.01, 1.0)
    target64 = grads["fp64"][3]
    fd = np.zeros(len(coords))
    fd_central = np.zeros(len(coords))
    hs = np.array([h_mass * float(p.mass[k]) if w == "mass" else h for w, k in coords])
    t0 = time.perf_counter()
    for c0 in range(0, len(coords), fd_chunk):
        chunk = coords[c0:c0 + fd_chunk]
        copies = []
        for i, (w, k) in enumerate(chunk):
            for sgn in (1.0, -1.0, 2.0, -2.0):
                copies.append(_perturb(p, w, k, sgn * hs[c0 + i]))
        fin = api.frozen_rollout(p, cfg64, copies, steps)
        for i in range(len(chunk)):
            h = hs[c0 + i]
            d = []
            for j in (0, 2):
                xp, xm = fin[4 * i + j, :3], fin[4 * i + j + 1, :3]
                d.append(np.sum((xp - xm) * (xp + xm - 2.0 * target64)) / n / (2.0 * h * (1 + j // 2)))
            fd_central[c0 + i] = d[0]
            fd[c0 + i] = (4.0 * d[0] - d[1]) / 3.0
    fdinfo = {"coords": len(coords), "h_positions_velocities": h, "h_mass": f"{h_mass} * m",
              "richardson": "(4 D(h) - D(2h)) / 3", "seconds": time.perf_counter() - t0}
    per = {}
    for name in ("fp64", "mixed"):
        gm, gx, gv, _ = grads[name]
        ad = _pick(gm, gx, gv, coords)
        per[name] = ad
        rel = np.abs(ad - fd) / np.abs(fd)
        relc = np.abs(ad - fd_central) / np.abs(fd_central)
        info = {"max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                "within_1e-5": int(np.sum(rel <= 1e-5)), "max_rel_central_only": float(relc.max()),
                "relative_l2": float(np.linalg.norm(ad - fd) / np.linalg.norm(fd))}
        for kind in ("position", "velocity", "mass"):
            sel = _kind_mask(coords, kind)
            if sel.any():
                info[f"max_rel_{kind}"] = float(rel[sel].max())
                # error against the typical gradient of that kind: components far
                # below it sit at the rounding noise of the +-h trajectories
                info[f"max_err_over_median_{kind}"] = float(np.max(np.abs(ad - fd)[sel]) /
                                                            np.median(np.abs(fd[sel])))
        fdinfo[name] = info
    fdinfo["per_coordinate"] = [[w, k, float(fd[i]), float(per["fp64"][i]), float(per["mixed"][i])]
                                for i, (w, k) in enumerate(coords)]
    out["finite_differences"] = fdinfo
    # tree adjoint against the FP64 direct-sum adjoint at n_direct
    pd = ics.plummer(n_direct, seed=0)
    rngd = np.random.Generator(np.random.Philox(99))
    wx = rngd.standard_normal((3, n_direct)) / n_direct
    cmp = {}
    for theta in (0.5, 0.0):
        cfg = api.SimulationConfig(1e-3, theta, 0.01, 1.0)
        sim = api.Simulation(pd, cfg)
        sim.initialize()
        sim.rollout(steps, every)
        gm, gx, gv = sim.backward(wx)
        sim.close()
        _, dm, dx, dv = api.direct_rollout_adjoint(pd, cfg, steps, wx)
        cmp[str(theta)] = {k: float(np.linalg.norm(a - b) / np.linalg.norm(b))
                           for k, a, b in (("mass", gm, dm), ("positions", gx, dx), ("velocities", gv, dv))}
    out["direct_sum_adjoint"] = {"n": n_direct, "steps": steps, "loss": "linear, N(0,1)/N weights on x_T",
                                 "relative_l2_difference_by_theta": cmp}
    return out


WORKLOADS = {"disk": disk, "blobs": blobs, "ensemble": ensemble, "adjoint": adjoint}
