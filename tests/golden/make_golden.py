"""Generate golden fixtures by running the reference itself.

Runs the unmodified sytrams/AMSC-Nbody CUDA sources (built into
oracle/_ref/libnbody_ref.so by ``make -C oracle ref`` in a container that has
the reference sources) on a GPU and stores every intermediate of the
reference pipeline for small seeded workloads:

  plummer4096.npz   config-0 Plummer sphere N=4096 (G=1, theta=0.5,
                    eps=0.01): Bbox, Morton keys + permutation, leaf groups,
                    Karras tree, radix-to-octree plan, octree topology,
                    geometry, mass/COM, accelerations, and the state after
                    10 KDK steps of dt=1e-3.
  blobs4096.npz     clustered blobs N=4096 (large multi-particle leaves).
  dupes1024.npz     1024 particles on 97 distinct points (duplicate keys).
  radix_random.npz  Karras trees of the reference test-suite's random key
                    sets (tests/unit/cuda/tree_builder_test.cu:602-642 sizes,
                    std::mt19937(0xC0FFEE) keys, forced duplicates).

Usage (needs a GPU and the built reference):  python tests/golden/make_golden.py
The fixtures are committed; tests read them without the reference present.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "amsc-nbody_b200"))

import pyoracle  # noqa: E402
from nbb import ics  # noqa: E402

KEEP = ["keys", "idx", "uniq", "gfirst", "gcount", "left", "right", "rfirst", "rlast", "plen",
        "rparent", "plan_level", "plan_count", "plan_offset", "children", "oparent", "olevel",
        "oprefix", "ofirst", "ocount", "child_count", "cx", "cy", "cz", "half", "mass", "comx",
        "comy", "comz", "ax", "ay", "az"]


def mt19937_raw(seed: int, count: int) -> np.ndarray:
    """The first `count` outputs of std::mt19937(seed)."""
    bg = np.random.MT19937()
    bg._legacy_seeding(seed)
    return bg.random_raw(count).astype(np.uint32)


def reference_random_keys():
    """tree_builder_test.cu:602-642: sorted random keys per size, with
    keys[i] = keys[i-1] for i = 5, 16, 27, ... (one shared generator)."""
    bg = np.random.MT19937()
    bg._legacy_seeding(0xC0FFEE)
    out = {}
    for n in (3, 5, 7, 16, 31, 64, 257):
        keys = np.sort(bg.random_raw(n).astype(np.uint32))
        for i in range(5, n, 11):
            keys[i] = keys[i - 1]
        out[n] = keys
        # the test shuffles indices with the same generator afterwards; that
        # consumption is not reproduced, so only the first size is exact
        break
    return out


def pipeline_fixture(p, theta, soft, g, steps=0, dt=0.0):
    r = pyoracle.ref_pipeline(p.mass, p.x, p.y, p.z, theta=theta, soft=soft, g=g)
    out = {k: r[k] for k in KEEP}
    out["box"] = r["box"]
    out["n_groups"] = np.int64(r["n_groups"])
    out["n_octree"] = np.int64(r["n_octree"])
    for f in ("mass", "x", "y", "z", "vx", "vy", "vz"):
        out["in_" + f] = getattr(p, f)
    if steps:
        ms = np.zeros(steps, np.float32)
        st = pyoracle.ref_simulate(p, steps, dt, theta, soft, g, step_ms=ms)
        for k, v in zip(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"), st):
            out[f"traj_{k}"] = v
        out["traj_steps"] = np.int64(steps)
        out["traj_dt"] = np.float64(dt)
    out["theta"] = np.float64(theta)
    out["soft"] = np.float64(soft)
    out["g"] = np.float64(g)
    return out


def main():
    if not pyoracle.ref_available():
        raise SystemExit("oracle/_ref/libnbody_ref.so missing: build it with make -C oracle ref")
    fixtures = {
        "plummer4096": pipeline_fixture(ics.plummer(4096, seed=0), 0.5, 0.01, 1.0, steps=10, dt=1e-3),
        "blobs4096": pipeline_fixture(ics.blobs(4096, seed=2), 0.5, 1e-3, 1.0),
    }
    rng = np.random.Generator(np.random.Philox(7))
    pts = rng.uniform(-1.0, 1.0, (97, 3))
    pick = rng.integers(0, 97, 1024)
    d = ics.ParticleData(rng.uniform(0.5, 1.5, 1024), pts[pick, 0].copy(), pts[pick, 1].copy(),
                         pts[pick, 2].copy(), np.zeros(1024), np.zeros(1024), np.zeros(1024))
    fixtures["dupes1024"] = pipeline_fixture(d, 0.7, 0.05, 1.0)
    radix = {}
    for n, keys in reference_random_keys().items():
        t = pyoracle.ref_radix_tree(keys)
        radix[f"keys_{n}"] = keys
        for k, v in t.items():
            radix[f"{k}_{n}"] = v
    # wider coverage: further seeded key sets with duplicates
    for n in (2, 4, 100, 1000):
        keys = np.sort(mt19937_raw(1000 + n, n))
        keys[3::7] = keys[2::7][: keys[3::7].size]
        keys = np.sort(keys)
        t = pyoracle.ref_radix_tree(keys)
        radix[f"keys_{n}"] = keys
        for k, v in t.items():
            radix[f"{k}_{n}"] = v
    fixtures["radix_random"] = radix
    for name, data in fixtures.items():
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **data)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
