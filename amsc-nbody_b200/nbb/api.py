"""Python mirror of the reference's public API for the Barnes-Hut step.

Names, argument meaning and error behaviour follow sytrams/AMSC-Nbody:
``Simulation`` (src/simulation.hpp:24-66), ``SimulationConfig``
(src/simulation.hpp:18-22), ``BarnesHutParameters`` (src/barnes_hut.hpp:8-13),
``computeBarnesHutAcceleration`` (src/barnes_hut.hpp:21) and the leapfrog
integrator (src/integrator.hpp:5-7).  Every call goes through the C ABI of
libnbb.so.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from ._lib import check, ptr
from .ics import ParticleData

G_SI = 6.67430e-11  # src/particle.hpp:16


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclasses.dataclass
class SimulationConfig:
    """SimulationConfig{timeStep, theta, softening} plus the gravitational
    constant (the reference's Simulation fixes it to the SI value) and the
    traversal precision of this library."""

    time_step: float
    theta: float
    softening: float
    gravitational_constant: float = G_SI
    precision: int = _lib.PRECISION_FP64
    group_size: int = 0
    use_graph: bool = True
    device: int = 0
    cache_depth: int = -1  # mixed walk: tree levels staged in shared memory; -1 tuned

    def to_c(self) -> _lib.Config:
        return _lib.Config(self.time_step, self.theta, self.softening, self.gravitational_constant,
                           int(self.precision), int(self.group_size), int(bool(self.use_graph)),
                           int(self.device), int(self.cache_depth))


@dataclasses.dataclass
class BarnesHutParameters:
    theta: float = 0.5
    softening: float = 1.0e-6
    gravitational_constant: float = G_SI


class Simulation:
    """Owns the particle state on the GPU and advances it with leapfrog KDK
    (src/simulation.cpp:70-127).  ``particles`` is copied in."""

    def __init__(self, particles: ParticleData, config: SimulationConfig, types=None):
        lib = _lib.load()
        self._lib = lib
        self._handle = C.c_void_p()
        self._n = len(particles)
        arrs = [_f64(a) for a in particles.arrays()]
        t = None if types is None else np.ascontiguousarray(types, dtype=np.uint8)
        cfg = config.to_c()
        check(lib.nbb_sim_create(C.byref(cfg), self._n, *[ptr(a) for a in arrs], ptr(t), 0,
                                 C.byref(self._handle)))
        self.config = config

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.nbb_sim_destroy(h)
            self._handle = None

    def close(self):
        self.__del__()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def initialize(self) -> None:
        check(self._lib.nbb_sim_initialize(self._handle))

    def step(self) -> None:
        check(self._lib.nbb_sim_step(self._handle))

    def run(self, number_of_steps: int) -> None:
        check(self._lib.nbb_sim_run(self._handle, int(number_of_steps)))

    def time(self) -> float:
        return self._lib.nbb_sim_time(self._handle)

    def step_number(self) -> int:
        return int(self._lib.nbb_sim_step_number(self._handle))

    # reference spelling
    stepNumber = step_number

    def particles(self) -> _lib.StateView:
        """Non-owning device view (DeviceParticlesView)."""
        v = _lib.StateView()
        check(self._lib.nbb_sim_state(self._handle, C.byref(v)))
        return v

    def set_stream(self, stream_handle: int | None) -> None:
        check(self._lib.nbb_sim_set_stream(self._handle, C.c_void_p(stream_handle) if stream_handle else None))

    def synchronize(self) -> None:
        check(self._lib.nbb_sim_synchronize(self._handle))

    def upload(self, p: ParticleData | None = None, *, mass=None, x=None, y=None, z=None, vx=None,
               vy=None, vz=None) -> None:
        if p is not None:
            mass, x, y, z, vx, vy, vz = p.arrays()
        check(self._lib.nbb_sim_upload(self._handle, *[ptr(a) for a in (mass, x, y, z, vx, vy, vz)]))

    def download(self, out=None):
        """Positions and velocities to host (new arrays unless ``out`` =
        6 float64 arrays)."""
        if out is None:
            out = [np.empty(self._n) for _ in range(6)]
        check(self._lib.nbb_sim_download(self._handle, *[ptr(a) for a in out]))
        return out

    def step_host(self, p: ParticleData | None = None, *, mass=None, x=None, y=None, z=None, vx=None,
                  vy=None, vz=None, out=None):
        """One step with host state in and out (upload + step + download in
        one call, the positions' copy overlapping the walk).  Returns ``out``
        (6 float64 arrays: x y z vx vy vz; new arrays when None)."""
        if p is not None:
            mass, x, y, z, vx, vy, vz = p.arrays()
        if out is None:
            out = [np.empty(self._n) for _ in range(6)]
        check(self._lib.nbb_sim_step_host(self._handle, *[ptr(a) for a in (mass, x, y, z, vx, vy, vz)],
                                          *[ptr(a) for a in out]))
        return out

    def accelerations(self):
        """Current accelerations copied to host."""
        out = [np.empty(self._n) for _ in range(3)]
        check(self._lib.nbb_sim_download_accel(self._handle, *[ptr(a) for a in out]))
        return out

    def stats(self) -> _lib.Stats:
        s = _lib.Stats()
        check(self._lib.nbb_sim_stats(self._handle, C.byref(s)))
        return s

    PROFILE_STAGES = ("reset", "bbox", "morton_sort_groups", "tree", "traversal")

    def profile(self):
        """Recompute the current force outside the step graph with CUDA events
        between stages; returns ({stage: ms}, Stats).  State is unchanged."""
        ms = (C.c_float * len(self.PROFILE_STAGES))()
        st = _lib.Stats()
        check(self._lib.nbb_sim_profile(self._handle, ms, C.byref(st)))
        return dict(zip(self.PROFILE_STAGES, list(ms))), st

    def diagnostics(self, potential: int = _lib.POTENTIAL_TREE) -> dict:
        """Conserved quantities of the current state (nbb_sim_diagnostics):
        mass, centre of mass, momentum, angular momentum, kinetic, potential
        and total energy."""
        d = _lib.Diagnostics()
        check(self._lib.nbb_sim_diagnostics(self._handle, int(potential), C.byref(d)))
        return {"mass": d.mass, "center_of_mass": np.array(d.center_of_mass[:]),
                "momentum": np.array(d.momentum[:]), "angular_momentum": np.array(d.angular_momentum[:]),
                "kinetic_energy": d.kinetic_energy, "potential_energy": d.potential_energy,
                "total_energy": d.total_energy}

    def capture_frame(self, max_particles: int = 100000, sequence: int = 0) -> bytes:
        """Quantized frame of the current positions (nbb_sim_capture_frame),
        in the reference's version-3 .nbsnap layout; see nbb.frames."""
        size = self._lib.nbb_frame_bytes(self._handle, int(max_particles))
        buf = np.empty(size, np.uint8)
        written = C.c_size_t(0)
        check(self._lib.nbb_sim_capture_frame(self._handle, int(max_particles), int(sequence), ptr(buf), size,
                                              C.byref(written), 0))
        return buf[: written.value].tobytes()

    def rollout(self, steps: int, checkpoint_every: int = 32) -> None:
        """Advance ``steps`` steps keeping (x, v, a) every
        ``checkpoint_every`` steps for :meth:`backward` (nbb_sim_rollout)."""
        check(self._lib.nbb_sim_rollout(self._handle, int(steps), int(checkpoint_every)))

    def backward(self, grad_positions, grad_velocities=None):
        """Gradient of a loss of the last rollout's final state with respect
        to its initial state (nbb_sim_backward).  ``grad_positions`` /
        ``grad_velocities`` are dL/d(final x, y, z) and dL/d(final vx, vy, vz)
        as three arrays (or a (3, n) array).  Returns (grad_mass,
        grad_positions (3, n), grad_velocities (3, n))."""
        n = self._n
        gp = [_f64(a) for a in grad_positions]
        gv = None if grad_velocities is None else [_f64(a) for a in grad_velocities]
        if len(gp) != 3 or any(a.size != n for a in gp) or (gv is not None and (
                len(gv) != 3 or any(a.size != n for a in gv))):
            raise _lib.InvalidArgument(_lib.ERR_INVALID_ARGUMENT, "cotangents must be three arrays of n values")
        gm = np.empty(n)
        gx0 = np.empty((3, n))
        gv0 = np.empty((3, n))
        gvp = [None] * 3 if gv is None else [ptr(a) for a in gv]
        check(self._lib.nbb_sim_backward(self._handle, *[ptr(a) for a in gp], *gvp, ptr(gm),
                                         *[ptr(gx0[k]) for k in range(3)], *[ptr(gv0[k]) for k in range(3)], 0))
        return gm, gx0, gv0

    def export_tree(self, m_capacity: int | None = None) -> dict:
        return _export(lambda e: self._lib.nbb_sim_export(self._handle, C.byref(e)), self._n, m_capacity)


class EnsembleSimulation(Simulation):
    """Independent systems advanced together, one launch per stage
    (nbb_ensemble_create): system k owns particles
    [offsets[k], offsets[k+1]) and has its own softening.  Every Simulation
    method applies; state arrays cover all systems back to back."""

    def __init__(self, ensemble, config: SimulationConfig):
        lib = _lib.load()
        self._lib = lib
        self._handle = C.c_void_p()
        p = ensemble.particles
        self._n = len(p)
        arrs = [_f64(a) for a in p.arrays()]
        offsets = np.ascontiguousarray(ensemble.offsets, dtype=np.int64)
        if offsets.ndim != 1 or offsets.size < 2 or int(offsets[-1]) != self._n:
            raise _lib.InvalidArgument(_lib.ERR_INVALID_ARGUMENT,
                                       "ensemble offsets must end at the particle count "
                                       f"({self._n}), got {offsets[-1] if offsets.size else None}")
        eps = None if ensemble.softening is None else _f64(ensemble.softening)
        cfg = config.to_c()
        check(lib.nbb_ensemble_create(C.byref(cfg), int(offsets.size - 1), ptr(offsets), ptr(eps),
                                      *[ptr(a) for a in arrs], 0, C.byref(self._handle)))
        self.config = config
        self.offsets = offsets


_EXPORT_FIELDS = [
    ("keys", np.uint32, "n"), ("idx", np.uint32, "n"), ("uniq", np.uint32, "n"),
    ("gfirst", np.int32, "n"), ("gcount", np.int32, "n"), ("left", np.int32, "n"),
    ("right", np.int32, "n"), ("rfirst", np.int32, "n"), ("rlast", np.int32, "n"),
    ("plen", np.int32, "n"), ("rparent", np.int32, "2n"), ("plan_level", np.int32, "2n"),
    ("plan_count", np.int32, "2n"), ("plan_offset", np.int32, "2n"),
    ("children", np.int32, "8m"), ("oparent", np.int32, "m"), ("olevel", np.int32, "m"),
    ("oprefix", np.uint32, "m"), ("ofirst", np.int32, "m"), ("ocount", np.int32, "m"),
    ("child_count", np.int32, "m"), ("cx", np.float64, "m"), ("cy", np.float64, "m"),
    ("cz", np.float64, "m"), ("half", np.float64, "m"), ("mass", np.float64, "m"),
    ("comx", np.float64, "m"), ("comy", np.float64, "m"), ("comz", np.float64, "m"),
]


def node_capacity(n: int) -> int:
    """Upper bound of octree nodes for n particles: sum over levels 0..10 of
    min(8^L, n), plus one."""
    return 1 + sum(min(8 ** lvl, n) for lvl in range(11))


def _export(call, n: int, m_capacity: int | None = None, fields=None) -> dict:
    mcap = node_capacity(n) if m_capacity is None else m_capacity
    size = {"n": max(n, 1), "2n": max(2 * n, 1), "m": mcap, "8m": 8 * mcap}
    bufs = {}
    e = _lib.TreeExport()
    e.m_capacity = mcap
    for name, dt, kind in _EXPORT_FIELDS:
        if fields is not None and name not in fields:
            continue
        bufs[name] = np.zeros(size[kind], dt)
        setattr(e, name, ptr(bufs[name]))
    check(call(e))
    g, m = e.n_groups, e.n_octree
    lens = {"keys": n, "idx": n, "uniq": g, "gfirst": g, "gcount": g, "left": g - 1,
            "right": g - 1, "rfirst": g - 1, "rlast": g - 1, "plen": g - 1, "rparent": 2 * g - 1,
            "plan_level": 2 * g - 1, "plan_count": 2 * g - 1, "plan_offset": 2 * g - 1,
            "children": 8 * m}
    out = {k: v[: max(lens.get(k, m), 0)].copy() for k, v in bufs.items()}
    out.update(box=np.array(list(e.box)), n_groups=g, n_octree=m)
    return out


def compute_accelerations(particles_or_arrays, theta: float, softening: float, g: float = 1.0,
                          precision: int = _lib.PRECISION_FP64, export: bool = False,
                          stats: bool = False):  # noqa: D417
    """One rebuild + Barnes-Hut evaluation of caller particles (host arrays):
    the reference's pipeline of src/simulation.cpp:137-198 with an explicit
    G.  Returns (ax, ay, az) [, export dict] [, Stats]."""
    lib = _lib.load()
    if isinstance(particles_or_arrays, ParticleData):
        m, x, y, z = (_f64(a) for a in particles_or_arrays.arrays()[:4])
    else:
        m, x, y, z = (_f64(a) for a in particles_or_arrays)
    n = m.size
    ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
    st = _lib.Stats()
    result = {}

    def call(e):
        return lib.nbb_accel(n, ptr(m), ptr(x), ptr(y), ptr(z), theta, softening, g, int(precision),
                             ptr(ax), ptr(ay), ptr(az), 0, C.byref(e) if e is not None else None,
                             C.byref(st))

    if export:
        result = _export(call, n)
    else:
        check(call(None))
    out = [ax, ay, az]
    if export:
        out.append(result)
    if stats:
        out.append(st)
    return tuple(out)


def compute_direct_accelerations(m, x, y, z, g: float = 1.0, softening: float = 0.0, targets=None):
    """FP64 direct summation on the GPU for the given targets (all when
    None); output k belongs to targets[k]."""
    lib = _lib.load()
    m, x, y, z = (_f64(a) for a in (m, x, y, z))
    t = None if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
    nt = m.size if t is None else t.size
    ax, ay, az = np.zeros(nt), np.zeros(nt), np.zeros(nt)
    check(lib.nbb_accel_direct(m.size, ptr(m), ptr(x), ptr(y), ptr(z), nt, ptr(t), g, softening,
                               ptr(ax), ptr(ay), ptr(az), 0))
    return ax, ay, az


def computeBarnesHutAcceleration(octree: dict, sorted_indices, mass, x, y, z, particle_count: int,
                                 parameters: BarnesHutParameters, particle_order: str = "original"):
    """computeBarnesHutAcceleration on a caller-built octree (reference
    numbering, src/octree_types.hpp:73-104).  ``octree`` holds children,
    parent, firstParticle, particleCount, mass, comX/Y/Z, centerX/Y/Z,
    halfSize (host arrays) and nParticles.  Returns (ax, ay, az)."""
    lib = _lib.load()
    n_nodes = int(np.asarray(octree["parent"]).size)
    n_particles = int(octree.get("nParticles", particle_count))
    if particle_count != n_particles:
        raise _lib.InvalidArgument(_lib.ERR_INVALID_ARGUMENT, "Particle count does not match the octree")
    arrs = {
        "children": np.ascontiguousarray(octree["children"], np.int32),
        "parent": np.ascontiguousarray(octree["parent"], np.int32),
        "first": np.ascontiguousarray(octree["firstParticle"], np.int32),
        "count": np.ascontiguousarray(octree["particleCount"], np.int32),
        "mass": _f64(octree["mass"]), "comx": _f64(octree["comX"]), "comy": _f64(octree["comY"]),
        "comz": _f64(octree["comZ"]), "cx": _f64(octree["centerX"]), "cy": _f64(octree["centerY"]),
        "cz": _f64(octree["centerZ"]), "half": _f64(octree["halfSize"]),
    }
    view = _lib.OctreeView(n_nodes, n_particles, *[ptr(arrs[k]) for k in (
        "children", "parent", "first", "count", "mass", "comx", "comy", "comz", "cx", "cy", "cz",
        "half")])
    idx = np.ascontiguousarray(sorted_indices, np.uint32)
    m, x, y, z = (_f64(a) for a in (mass, x, y, z))
    ax, ay, az = np.zeros(n_particles), np.zeros(n_particles), np.zeros(n_particles)
    order = {"original": 0, "morton": 1}[particle_order]
    check(lib.nbb_accel_octree(C.byref(view), ptr(idx), ptr(m), ptr(x), ptr(y), ptr(z), ptr(ax),
                               ptr(ay), ptr(az), parameters.theta, parameters.softening,
                               parameters.gravitational_constant, order, 0))
    return ax, ay, az


def octree_from_keys(sorted_keys) -> dict:
    """Leaf groups -> Karras tree -> plan -> sparse octree topology for caller
    sorted keys (export dict, geometry/physics fields absent)."""
    lib = _lib.load()
    k = np.ascontiguousarray(sorted_keys, np.uint32)
    n = k.size
    fields = {f for f, _, _ in _EXPORT_FIELDS} - {"child_count", "cx", "cy", "cz", "half", "mass",
                                                  "comx", "comy", "comz", "keys", "idx"}
    return _export(lambda e: lib.nbb_octree_from_keys(ptr(k), n, C.byref(e)), n, fields=fields)


def radix_tree(keys) -> dict:
    """buildTree on caller keys (any 32-bit keys, duplicates allowed)."""
    lib = _lib.load()
    k = np.ascontiguousarray(keys, np.uint32)
    n = k.size
    ni = max(n - 1, 1)
    left, right, rf, rl, pl = (np.zeros(ni, np.int32) for _ in range(5))
    parent = np.zeros(max(2 * n - 1, 1), np.int32)
    check(lib.nbb_radix_tree(ptr(k), n, ptr(left), ptr(right), ptr(rf), ptr(rl), ptr(pl), ptr(parent)))
    s = slice(0, n - 1)
    return dict(left=left[s].copy(), right=right[s].copy(), rangeFirst=rf[s].copy(),
                rangeLast=rl[s].copy(), prefixLength=pl[s].copy(), parent=parent[: 2 * n - 1].copy())


def leapfrog_kick_drift(x, y, z, vx, vy, vz, ax, ay, az, dt: float, stream=None):
    """leapfrogKickDrift on device tensors (torch CUDA float64), in place."""
    lib = _lib.load()
    n = x.numel()
    check(lib.nbb_kick_drift(*[ptr(a) for a in (x, y, z, vx, vy, vz, ax, ay, az)], n, dt, stream))


def leapfrog_kick(vx, vy, vz, ax, ay, az, dt: float, stream=None):
    """leapfrogKick on device tensors (torch CUDA float64), in place."""
    lib = _lib.load()
    n = vx.numel()
    check(lib.nbb_kick(*[ptr(a) for a in (vx, vy, vz, ax, ay, az)], n, dt, stream))


def measure_fma_tflops(precision: int) -> float:
    """Measured SIMT FMA throughput of the current GPU (TFLOP/s)."""
    v = C.c_double(0.0)
    check(_lib.load().nbb_measure_fma_tflops(int(precision), C.byref(v)))
    return v.value


def kernel_launch_count() -> int:
    return int(_lib.load().nbb_kernel_launch_count())


def frozen_rollout(particles: ParticleData, config: SimulationConfig, copies, steps: int):
    """Final states of perturbed copies advanced with the unperturbed
    system's tree structure at every step (nbb_frozen_rollout).  ``copies``
    is a sequence of ParticleData of the same size; returns an array
    (copies, 6, n) of final x, y, z, vx, vy, vz."""
    lib = _lib.load()
    n = len(particles)
    base = [_f64(a) for a in particles.arrays()]
    q = len(copies)
    stack = [np.ascontiguousarray(np.stack([getattr(c, f) for c in copies]), dtype=np.float64)
             for f in ("mass", "x", "y", "z", "vx", "vy", "vz")]
    if any(a.shape != (q, n) for a in stack):
        raise _lib.InvalidArgument(_lib.ERR_INVALID_ARGUMENT, "every copy must hold n particles")
    out = np.empty((6, q, n))
    cfg = config.to_c()
    check(lib.nbb_frozen_rollout(C.byref(cfg), n, *[ptr(a) for a in base], q, *[ptr(a) for a in stack],
                                 int(steps), *[ptr(out[k]) for k in range(6)], 0))
    return np.ascontiguousarray(out.transpose(1, 0, 2))


def direct_rollout_adjoint(particles: ParticleData, config: SimulationConfig, steps: int, grad_positions,
                           grad_velocities=None):
    """FP64 direct-summation rollout and its adjoint
    (nbb_direct_rollout_adjoint).  Returns (final state (6, n), grad_mass,
    grad_positions (3, n), grad_velocities (3, n))."""
    lib = _lib.load()
    n = len(particles)
    arrs = [_f64(a) for a in particles.arrays()]
    gp = [_f64(a) for a in grad_positions]
    keep = None if grad_velocities is None else [_f64(a) for a in grad_velocities]
    gvp = [None] * 3 if keep is None else [ptr(a) for a in keep]
    final = np.empty((6, n))
    gm = np.empty(n)
    gx0 = np.empty((3, n))
    gv0 = np.empty((3, n))
    cfg = config.to_c()
    check(lib.nbb_direct_rollout_adjoint(C.byref(cfg), n, *[ptr(a) for a in arrs], int(steps),
                                         *[ptr(a) for a in gp], *gvp, *[ptr(final[k]) for k in range(6)],
                                         ptr(gm), *[ptr(gx0[k]) for k in range(3)],
                                         *[ptr(gv0[k]) for k in range(3)], 0))
    return final, gm, gx0, gv0


class ConservationMonitor:
    """Relative drift of the conserved quantities of a simulation over time:
    ``record()`` stores the current diagnostics; ``drift()`` gives, for the
    last record, |E - E0| / |E0| for the total energy and |P - P0| / scale,
    |L - L0| / scale for momentum and angular momentum (scale: their initial
    norms, or sum m |v| and sum m |x| |v| when those vanish)."""

    def __init__(self, simulation: Simulation, potential: int = _lib.POTENTIAL_TREE):
        self.sim = simulation
        self.potential = potential
        self.records = []

    def record(self) -> dict:
        d = self.sim.diagnostics(self.potential)
        d["step"] = self.sim.step_number()
        d["time"] = self.sim.time()
        self.records.append(d)
        return d

    def drift(self) -> dict:
        if not self.records:
            raise ValueError("no diagnostics recorded")
        d0, d = self.records[0], self.records[-1]
        e0 = abs(d0["total_energy"]) or 1.0
        p_scale = np.linalg.norm(d0["momentum"]) or 1.0
        l_scale = np.linalg.norm(d0["angular_momentum"]) or 1.0
        return {"energy": abs(d["total_energy"] - d0["total_energy"]) / e0,
                "momentum": float(np.linalg.norm(d["momentum"] - d0["momentum"]) / p_scale),
                "angular_momentum": float(np.linalg.norm(d["angular_momentum"] - d0["angular_momentum"]) / l_scale),
                "steps": d["step"] - d0["step"]}
