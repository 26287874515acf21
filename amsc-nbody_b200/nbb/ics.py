"""Seeded synthetic initial conditions for the benchmark workloads.

All generators use numpy's counter-based Philox bit generator, so a (recipe,
n, seed) triple always yields the same float64 SoA state.  Units: G = 1 and
total mass 1 unless stated.  The reference's own benchmark uses Gaussian
"spiral" blobs from ``data/generate_galaxy.py``; the recipes here follow the
benchmark configurations of this project (Plummer sphere, disk + bulge,
clustered blobs, ensembles of Plummer spheres).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class ParticleData:
    """Planar float64 particle state, the same layout as the reference's
    ``Particles`` / ``DeviceParticlesView`` (src/particle.hpp:85-118)."""

    mass: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray

    def __len__(self) -> int:
        return int(self.mass.shape[0])

    def copy(self) -> "ParticleData":
        return ParticleData(*(np.array(a, dtype=np.float64, copy=True) for a in self.arrays()))

    def arrays(self):
        return (self.mass, self.x, self.y, self.z, self.vx, self.vy, self.vz)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


def _isotropic(rng: np.random.Generator, n: int):
    cos_t = rng.uniform(-1.0, 1.0, n)
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    return sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t


def _plummer_radii(rng, n: int, a: float, r_max: float) -> np.ndarray:
    """Radii from the inverse cumulative mass profile M(r)/M = r^3/(r^2+a^2)^1.5,
    redrawing any radius at or beyond r_max."""
    r = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        u = rng.uniform(0.0, 1.0, todo.size)
        u = np.clip(u, 1e-300, 1.0)
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        ok = np.isfinite(rr) & (rr < r_max)
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    return r


def _ahw_speed_fraction(rng, n: int) -> np.ndarray:
    """Aarseth-Henon-Wielen rejection sampling of q = v / v_escape from
    g(q) = q^2 (1 - q^2)^(7/2), whose maximum is below 0.1."""
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        x1 = rng.uniform(0.0, 1.0, todo.size)
        x2 = rng.uniform(0.0, 1.0, todo.size)
        ok = 0.1 * x2 < x1 * x1 * (1.0 - x1 * x1) ** 3.5
        q[todo[ok]] = x1[ok]
        todo = todo[~ok]
    return q


def _plummer_parts(rng, n: int, total_mass: float, a: float, r_max_over_a: float = 10.0):
    r = _plummer_radii(rng, n, a, r_max_over_a * a)
    ux, uy, uz = _isotropic(rng, n)
    q = _ahw_speed_fraction(rng, n)
    v = q * np.sqrt(2.0 * total_mass) * (r * r + a * a) ** -0.25
    wx, wy, wz = _isotropic(rng, n)
    return r * ux, r * uy, r * uz, v * wx, v * wy, v * wz


def _centre(p: ParticleData) -> ParticleData:
    m = p.mass
    tot = m.sum()
    for a in ("x", "y", "z", "vx", "vy", "vz"):
        arr = getattr(p, a)
        arr -= (m * arr).sum() / tot
    return p


def plummer(n: int, seed: int = 0, a: float = 1.0, total_mass: float = 1.0) -> ParticleData:
    """Plummer sphere: equal masses summing to ``total_mass``, scale radius a,
    radii truncated at r < 10a, isotropic directions, velocities from the
    isotropic distribution function by AHW rejection, centre of mass position
    and velocity subtracted."""
    rng = _rng(seed)
    x, y, z, vx, vy, vz = _plummer_parts(rng, n, total_mass, a)
    p = ParticleData(np.full(n, total_mass / n), x, y, z, vx, vy, vz)
    return _centre(p)


def disk_bulge(n: int, seed: int = 1, disk_fraction: float = 0.8, r_disk: float = 1.0,
               h_disk: float = 0.1, a_bulge: float = 0.2, dispersion: float = 0.1) -> ParticleData:
    """Exponential disk (surface density ~ exp(-R/r_disk), sech^2 vertical
    profile of scale height h_disk) holding ``disk_fraction`` of the particles,
    plus a Plummer bulge (a = a_bulge, r < 10a).  Equal masses summing to 1.
    Disk particles move on circles at v_c = sqrt(M(<R)/R) from the enclosed
    (spherically counted) mass, plus Gaussian dispersion of
    ``dispersion * v_c`` per component; bulge velocities follow the bulge's own
    Plummer distribution function (AHW rejection)."""
    rng = _rng(seed)
    nd = int(round(disk_fraction * n))
    nb = n - nd
    m = np.full(n, 1.0 / n)
    # R pdf ~ R exp(-R/r_disk): Gamma(2, r_disk)
    R = rng.gamma(2.0, r_disk, nd)
    phi = rng.uniform(0.0, 2.0 * np.pi, nd)
    u = rng.uniform(-1.0, 1.0, nd)
    u = np.clip(u, -1.0 + 1e-15, 1.0 - 1e-15)
    zd = h_disk * np.arctanh(u)
    xd, yd = R * np.cos(phi), R * np.sin(phi)
    xb, yb, zb, vxb, vyb, vzb = _plummer_parts(rng, nb, nb / n, a_bulge)
    x = np.concatenate([xd, xb])
    y = np.concatenate([yd, yb])
    z = np.concatenate([zd, zb])
    r_all = np.sqrt(x * x + y * y + z * z)
    order = np.argsort(r_all, kind="stable")
    cum = np.cumsum(m[order])
    r_sorted = r_all[order]
    # enclosed mass at each disk particle's cylindrical radius
    enc = np.interp(R, r_sorted, cum, left=0.0, right=1.0)
    vc = np.sqrt(np.maximum(enc, 0.0) / np.maximum(R, 1e-12))
    sig = dispersion * vc
    vxd = -np.sin(phi) * vc + sig * rng.standard_normal(nd)
    vyd = np.cos(phi) * vc + sig * rng.standard_normal(nd)
    vzd = sig * rng.standard_normal(nd)
    p = ParticleData(m, x, y, z, np.concatenate([vxd, vxb]), np.concatenate([vyd, vyb]),
                     np.concatenate([vzd, vzb]))
    return _centre(p)


def blobs(n: int, seed: int = 2, n_blobs: int = 64, half_width: float = 50.0,
          sigma_range=(0.01, 1.0), mass_sigma: float = 0.5) -> ParticleData:
    """Clustered precision stress: ``n_blobs`` Gaussian blobs with centres
    uniform in [-half_width, half_width]^3, per-blob sigma log-uniform in
    ``sigma_range``, multinomial (equal-weight) populations, log-normal
    (mu = 0, sigma = mass_sigma) masses normalised to total 1, zero velocity."""
    rng = _rng(seed)
    centres = rng.uniform(-half_width, half_width, (n_blobs, 3))
    lo, hi = np.log(sigma_range[0]), np.log(sigma_range[1])
    sig = np.exp(rng.uniform(lo, hi, n_blobs))
    counts = rng.multinomial(n, np.full(n_blobs, 1.0 / n_blobs))
    blob = np.repeat(np.arange(n_blobs), counts)
    pos = centres[blob] + sig[blob, None] * rng.standard_normal((n, 3))
    m = rng.lognormal(0.0, mass_sigma, n)
    m /= m.sum()
    zero = np.zeros(n)
    return ParticleData(m, np.ascontiguousarray(pos[:, 0]), np.ascontiguousarray(pos[:, 1]),
                        np.ascontiguousarray(pos[:, 2]), zero.copy(), zero.copy(), zero.copy())


@dataclasses.dataclass
class Ensemble:
    """Independent systems stored back to back; system s owns particles
    [offsets[s], offsets[s+1])."""

    particles: ParticleData
    offsets: np.ndarray  # int64, n_systems + 1
    softening: np.ndarray  # per-system epsilon

    @property
    def n_systems(self) -> int:
        return int(self.offsets.shape[0] - 1)


def plummer_ensemble(n_systems: int = 512, seed: int = 3, n_min: int = 1024,
                     n_max: int = 131072, eps_ref: float = 0.01, n_ref: int = 4096) -> Ensemble:
    """Ensemble of independent Plummer spheres (each as :func:`plummer`), N
    log-uniform in [n_min, n_max] per system, per-system softening
    eps_ref * (n_ref / N)^(1/3)."""
    rng = _rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_systems))
    sizes = np.clip(np.rint(sizes).astype(np.int64), n_min, n_max)
    parts = [plummer(int(k), seed=int(seed * 100003 + s)) for s, k in enumerate(sizes)]
    offsets = np.zeros(n_systems + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    cat = ParticleData(*(np.concatenate([getattr(p, f) for p in parts])
                         for f in ("mass", "x", "y", "z", "vx", "vy", "vz")))
    eps = eps_ref * (n_ref / sizes.astype(np.float64)) ** (1.0 / 3.0)
    return Ensemble(cat, offsets, eps)
