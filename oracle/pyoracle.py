"""ctypes bindings for the CPU oracle (liboracle.so) and, where it was built,
the reference harness (_ref/libnbody_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg / reference arm.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnbody_ref.so")

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_Z = C.c_size_t


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def frame_capture(x, y, z, types=None, max_particles=0, sequence=0, step=0, time=0.0):
    """orc_frame_capture: the frame's bytes, or raises ValueError(status)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    n = x.size
    s = n if (max_particles == 0 or max_particles > n) else max_particles
    t = None if types is None else np.ascontiguousarray(types, dtype=np.uint8)
    out = np.zeros(128 + 7 * s, np.uint8)
    r = lib().orc_frame_capture(n, _ptr(x), _ptr(y), _ptr(z), _ptr(t), int(max_particles), int(sequence),
                                int(step), float(time), _ptr(out), out.size)
    if r < 0:
        raise ValueError(r)
    return out[:r].tobytes()


def build_oracle() -> str:
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return ORACLE_SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        L = _lib
        L.orc_bbox.argtypes = [_Z, _P, _P, _P, _P]
        L.orc_morton.argtypes = [_Z, _P, _P, _P, _P, _P, _P]
        L.orc_leaf_groups.argtypes = [_I, _P, _P, _P, _P]
        L.orc_radix_tree.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P]
        L.orc_octree_plan.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P]
        L.orc_octree_build.argtypes = [_I] + [_P] * 8 + [_I] + [_P] * 6
        L.orc_octree_geometry.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P]
        L.orc_octree_mass.argtypes = [_I, _I] + [_P] * 14
        L.orc_bh_accel.argtypes = ([_I, _I] + [_P] * 17 + [_I, _D, _D, _D] + [_P] * 3 + [_I, _P])
        L.orc_direct_accel.argtypes = [_I, _P, _P, _P, _P, _I, _P, _D, _D, _P, _P, _P, _I]
        L.orc_direct_accel.restype = None
        L.orc_kick_drift.argtypes = [_Z] + [_P] * 9 + [_D]
        L.orc_kick_drift.restype = None
        L.orc_kick.argtypes = [_Z] + [_P] * 6 + [_D]
        L.orc_kick.restype = None
        L.orc_pipeline.argtypes = [_Z, _P, _P, _P, _P, _D, _D, _D, _I, _P]
        L.orc_simulate.argtypes = [_Z] + [_P] * 10 + [_D, _D, _D, _D, _I, _I]
        L.orc_frame_capture.argtypes = [_Z, _P, _P, _P, _P, _Z, C.c_uint64, C.c_uint64, _D, _P, _Z]
        L.orc_frame_capture.restype = C.c_longlong
    return _lib


class OracleError(RuntimeError):
    def __init__(self, stage: str, code: int):
        super().__init__(f"oracle {stage} failed with status {code}")
        self.code = code


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def bbox(x, y, z):
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.zeros(4)
    st = lib().orc_bbox(x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(out))
    if st:
        raise OracleError("bbox", st)
    return out


def morton(x, y, z, box=None):
    x, y, z = _f64(x), _f64(y), _f64(z)
    if box is None:
        box = bbox(x, y, z)
    box = _f64(box)
    keys = np.zeros(x.size, np.uint32)
    idx = np.zeros(x.size, np.uint32)
    st = lib().orc_morton(x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(box), _ptr(keys), _ptr(idx))
    if st:
        raise OracleError("morton", st)
    return keys, idx


def leaf_groups(sorted_keys):
    k = _u32(sorted_keys)
    n = k.size
    uniq = np.zeros(max(n, 1), np.uint32)
    first = np.zeros(max(n, 1), np.int32)
    count = np.zeros(max(n, 1), np.int32)
    g = lib().orc_leaf_groups(n, _ptr(k), _ptr(uniq), _ptr(first), _ptr(count))
    if g <= 0:
        raise OracleError("leaf_groups", g)
    return uniq[:g].copy(), first[:g].copy(), count[:g].copy()


def radix_tree(keys):
    k = _u32(keys)
    n = k.size
    ni = max(n - 1, 1)
    left, right, rf, rl, pl = (np.zeros(ni, np.int32) for _ in range(5))
    parent = np.zeros(2 * n - 1, np.int32)
    st = lib().orc_radix_tree(n, _ptr(k), _ptr(left), _ptr(right), _ptr(rf), _ptr(rl), _ptr(pl),
                              _ptr(parent))
    if st:
        raise OracleError("radix_tree", st)
    s = slice(0, n - 1)
    return dict(left=left[s].copy(), right=right[s].copy(), rangeFirst=rf[s].copy(),
                rangeLast=rl[s].copy(), prefixLength=pl[s].copy(), parent=parent)


def octree_plan(uniq, tree):
    u = _u32(uniq)
    g = u.size
    nr = 2 * g - 1
    level, count, offset = (np.zeros(nr, np.int32) for _ in range(3))
    m = C.c_int(0)
    pl = _i32(tree["prefixLength"]) if g > 1 else np.zeros(1, np.int32)
    st = lib().orc_octree_plan(g, _ptr(u), _ptr(_i32(tree["parent"])), _ptr(pl), _ptr(level),
                               _ptr(count), _ptr(offset), C.byref(m))
    if st:
        raise OracleError("octree_plan", st)
    return dict(radixLevel=level, edgeNodeCount=count, edgeNodeOffset=offset, nOctreeNodes=m.value)


def octree_from_keys(sorted_keys):
    """Leaf groups -> Karras -> plan -> sparse octree topology, as the
    reference's sparse_octree_test pipeline (sparse_octree_test.cu:100-325)."""
    uniq, first, count = leaf_groups(sorted_keys)
    tree = radix_tree(uniq)
    plan = octree_plan(uniq, tree)
    m = plan["nOctreeNodes"]
    children = np.zeros(8 * m, np.int32)
    parent, level, first_p, count_p = (np.zeros(m, np.int32) for _ in range(4))
    prefix = np.zeros(m, np.uint32)
    rf = _i32(tree["rangeFirst"]) if uniq.size > 1 else np.zeros(1, np.int32)
    st = lib().orc_octree_build(uniq.size, _ptr(uniq), _ptr(first), _ptr(count),
                                _ptr(_i32(tree["parent"])), _ptr(rf), _ptr(plan["radixLevel"]),
                                _ptr(plan["edgeNodeCount"]), _ptr(plan["edgeNodeOffset"]), m,
                                _ptr(children), _ptr(parent), _ptr(level), _ptr(prefix),
                                _ptr(first_p), _ptr(count_p))
    if st:
        raise OracleError("octree_build", st)
    return dict(groups=(uniq, first, count), tree=tree, plan=plan,
                octree=dict(children=children, parent=parent, level=level, prefix=prefix,
                            firstParticle=first_p, particleCount=count_p, nNodes=m))


def octree_geometry(level, prefix, box):
    level, prefix, box = _i32(level), _u32(prefix), _f64(box)
    m = level.size
    cx, cy, cz, h = (np.zeros(m) for _ in range(4))
    st = lib().orc_octree_geometry(m, _ptr(level), _ptr(prefix), _ptr(box), _ptr(cx), _ptr(cy),
                                   _ptr(cz), _ptr(h))
    if st:
        raise OracleError("octree_geometry", st)
    return cx, cy, cz, h


def bh_accel(octree: dict, idx, m, x, y, z, theta, soft, g, morton_ordered=False, n_threads=0):
    """Traversal on a caller octree dict with keys children, parent,
    firstParticle, particleCount, mass, comX/Y/Z, centerX/Y/Z, halfSize."""
    n = int(np.asarray(m).size)
    o = {k: (np.ascontiguousarray(v)) for k, v in octree.items()}
    nn = o["parent"].size
    ax, ay, az = np.zeros(n), np.zeros(n), np.zeros(n)
    inter = C.c_int64(0)
    st = lib().orc_bh_accel(nn, n, _ptr(_i32(o["children"])), _ptr(_i32(o["parent"])),
                            _ptr(_i32(o["firstParticle"])), _ptr(_i32(o["particleCount"])),
                            _ptr(_f64(o["mass"])), _ptr(_f64(o["comX"])), _ptr(_f64(o["comY"])),
                            _ptr(_f64(o["comZ"])), _ptr(_f64(o["centerX"])),
                            _ptr(_f64(o["centerY"])), _ptr(_f64(o["centerZ"])),
                            _ptr(_f64(o["halfSize"])), _ptr(_u32(idx)), _ptr(_f64(m)),
                            _ptr(_f64(x)), _ptr(_f64(y)), _ptr(_f64(z)), int(morton_ordered),
                            theta, soft, g, _ptr(ax), _ptr(ay), _ptr(az), n_threads,
                            C.byref(inter))
    if st:
        raise OracleError("bh_accel", st)
    return ax, ay, az


def direct_accel(m, x, y, z, g=1.0, soft=0.0, targets=None, n_threads=0):
    m, x, y, z = _f64(m), _f64(x), _f64(y), _f64(z)
    n = m.size
    t = None if targets is None else _i32(targets)
    nt = n if t is None else t.size
    ax, ay, az = np.zeros(nt), np.zeros(nt), np.zeros(nt)
    lib().orc_direct_accel(n, _ptr(m), _ptr(x), _ptr(y), _ptr(z), nt, _ptr(t), g, soft, _ptr(ax),
                           _ptr(ay), _ptr(az), n_threads)
    return ax, ay, az


def kick_drift(x, y, z, vx, vy, vz, ax, ay, az, dt):
    arrs = [_f64(a).copy() for a in (x, y, z, vx, vy, vz)]
    acc = [_f64(a) for a in (ax, ay, az)]
    lib().orc_kick_drift(arrs[0].size, *[_ptr(a) for a in arrs], *[_ptr(a) for a in acc], dt)
    return arrs


def kick(vx, vy, vz, ax, ay, az, dt):
    arrs = [_f64(a).copy() for a in (vx, vy, vz)]
    acc = [_f64(a) for a in (ax, ay, az)]
    lib().orc_kick(arrs[0].size, *[_ptr(a) for a in arrs], *[_ptr(a) for a in acc], dt)
    return arrs


class _PipelineOut(C.Structure):
    _fields_ = [("box", C.c_double * 4)] + [(f, _P) for f in (
        "keys", "idx", "uniq", "gfirst", "gcount", "left", "right", "rfirst", "rlast", "plen",
        "rparent", "plan_level", "plan_count", "plan_offset")] + [("m_capacity", C.c_int)] + [
        (f, _P) for f in ("children", "oparent", "olevel", "oprefix", "ofirst", "ocount",
                          "child_count", "cx", "cy", "cz", "half", "mass", "comx", "comy", "comz",
                          "ax", "ay", "az")] + [("n_groups", C.c_int), ("n_octree", C.c_int),
                                                 ("interactions", C.c_int64)]


# field name -> (dtype, size kind) shared with the reference harness layout
PIPELINE_FIELDS = [
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
    ("ax", np.float64, "n"), ("ay", np.float64, "n"), ("az", np.float64, "n"),
]


def trim_pipeline(bufs: dict, n: int, g: int, m: int) -> dict:
    """Cut capacity-sized buffers down to their valid lengths."""
    lens = {"keys": n, "idx": n, "uniq": g, "gfirst": g, "gcount": g, "left": g - 1,
            "right": g - 1, "rfirst": g - 1, "rlast": g - 1, "plen": g - 1, "rparent": 2 * g - 1,
            "plan_level": 2 * g - 1, "plan_count": 2 * g - 1, "plan_offset": 2 * g - 1,
            "children": 8 * m, "ax": n, "ay": n, "az": n}
    out = {}
    for k, v in bufs.items():
        out[k] = v[: lens.get(k, m)].copy()
    return out


def alloc_pipeline(n: int, m_capacity: int | None = None, with_accel=True):
    mcap = 10 * n + 1 if m_capacity is None else m_capacity
    sizes = {"n": max(n, 1), "2n": max(2 * n, 1), "m": mcap, "8m": 8 * mcap}
    bufs = {}
    for name, dt, kind in PIPELINE_FIELDS:
        if name in ("ax", "ay", "az") and not with_accel:
            continue
        bufs[name] = np.zeros(sizes[kind], dt)
    return bufs, mcap


def pipeline(m, x, y, z, theta=0.5, soft=0.01, g=1.0, n_threads=0, with_accel=True):
    """Full rebuild + (optional) force evaluation; returns a dict of every
    intermediate trimmed to its valid size, plus box, n_groups, n_octree,
    interactions."""
    m, x, y, z = _f64(m), _f64(x), _f64(y), _f64(z)
    n = m.size
    bufs, mcap = alloc_pipeline(n, with_accel=with_accel)
    o = _PipelineOut()
    o.m_capacity = mcap
    for name, arr in bufs.items():
        setattr(o, name, _ptr(arr))
    st = lib().orc_pipeline(n, _ptr(m), _ptr(x), _ptr(y), _ptr(z), theta, soft, g, n_threads,
                            C.byref(o))
    if st:
        raise OracleError("pipeline", st)
    out = trim_pipeline(bufs, n, o.n_groups, o.n_octree)
    out.update(box=np.array(list(o.box)), n_groups=o.n_groups, n_octree=o.n_octree,
               interactions=o.interactions)
    return out


def simulate(p, steps, dt, theta, soft, g=1.0, n_threads=0):
    """initialize() + steps x step() on copies of the state; returns
    (x, y, z, vx, vy, vz, ax, ay, az)."""
    m = _f64(p.mass)
    st_arr = [_f64(a).copy() for a in (p.x, p.y, p.z, p.vx, p.vy, p.vz)]
    acc = [np.zeros(m.size) for _ in range(3)]
    st = lib().orc_simulate(m.size, _ptr(m), *[_ptr(a) for a in st_arr], *[_ptr(a) for a in acc],
                            dt, theta, soft, g, steps, n_threads)
    if st:
        raise OracleError("simulate", st)
    return (*st_arr, *acc)


# ----------------------------------------------------------- reference ---

_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        _ref = C.CDLL(REF_SO)
        _ref.ref_pipeline.argtypes = [_Z, _P, _P, _P, _P, _D, _D, _D, _P]
        _ref.ref_simulate.argtypes = [_Z] + [_P] * 10 + [_D, _D, _D, _D, _I, _P]
        _ref.ref_radix_tree.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P]
        _ref.ref_last_error.restype = C.c_char_p
        _ref.ref_capture_frame.argtypes = [_Z, _P, _P, _P, _P, _Z, C.c_uint64, C.c_uint64, _D, C.c_char_p,
                                           C.c_char_p, _Z]
        _ref.ref_capture_last_error.restype = C.c_char_p
    return _ref


def ref_capture_frame(x, y, z, types, max_particles, sequence, step, time, directory):
    """The reference's DeviceFrameWriter + FrameSpool: returns the frame file's
    bytes (written under `directory`), or raises with the reference's message."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    t = np.ascontiguousarray(types, dtype=np.uint8)
    path = C.create_string_buffer(4096)
    st = ref_lib().ref_capture_frame(x.size, _ptr(x), _ptr(y), _ptr(z), _ptr(t), int(max_particles),
                                     int(sequence), int(step), float(time), directory.encode(), path, 4096)
    if st:
        raise RuntimeError(ref_lib().ref_capture_last_error().decode())
    with open(path.value.decode(), "rb") as f:
        return f.read()


class _RefOut(C.Structure):
    _fields_ = [("box", C.c_double * 4)] + [(f, _P) for f in (
        "keys", "idx", "uniq", "gfirst", "gcount", "left", "right", "rfirst", "rlast", "plen",
        "rparent", "plan_level", "plan_count", "plan_offset")] + [("m_capacity", C.c_int)] + [
        (f, _P) for f in ("children", "oparent", "olevel", "oprefix", "ofirst", "ocount",
                          "child_count", "cx", "cy", "cz", "half", "mass", "comx", "comy", "comz",
                          "ax", "ay", "az")] + [("n_groups", C.c_int), ("n_octree", C.c_int)]


def ref_pipeline(m, x, y, z, theta=0.5, soft=0.01, g=1.0, with_accel=True):
    m, x, y, z = _f64(m), _f64(x), _f64(y), _f64(z)
    n = m.size
    bufs, mcap = alloc_pipeline(n, with_accel=with_accel)
    o = _RefOut()
    o.m_capacity = mcap
    for name, arr in bufs.items():
        setattr(o, name, _ptr(arr))
    st = ref_lib().ref_pipeline(n, _ptr(m), _ptr(x), _ptr(y), _ptr(z), theta, soft, g, C.byref(o))
    if st:
        raise RuntimeError("reference pipeline: " + ref_lib().ref_last_error().decode())
    out = trim_pipeline(bufs, n, o.n_groups, o.n_octree)
    out.update(box=np.array(list(o.box)), n_groups=o.n_groups, n_octree=o.n_octree)
    return out


def ref_simulate(p, steps, dt, theta, soft, g=1.0, step_ms=None):
    m = _f64(p.mass)
    st_arr = [_f64(a).copy() for a in (p.x, p.y, p.z, p.vx, p.vy, p.vz)]
    acc = [np.zeros(m.size) for _ in range(3)]
    ms = np.zeros(max(steps, 1), np.float32)
    st = ref_lib().ref_simulate(m.size, _ptr(m), *[_ptr(a) for a in st_arr],
                                *[_ptr(a) for a in acc], dt, theta, soft, g, steps, _ptr(ms))
    if st:
        raise RuntimeError("reference simulate: " + ref_lib().ref_last_error().decode())
    if step_ms is not None:
        step_ms[:] = ms[:steps]
    return (*st_arr, *acc)


def ref_radix_tree(keys):
    k = _u32(keys)
    n = k.size
    ni = max(n - 1, 1)
    left, right, rf, rl, pl = (np.zeros(ni, np.int32) for _ in range(5))
    parent = np.zeros(2 * n - 1, np.int32)
    st = ref_lib().ref_radix_tree(n, _ptr(k), _ptr(left), _ptr(right), _ptr(rf), _ptr(rl),
                                  _ptr(pl), _ptr(parent))
    if st:
        raise RuntimeError("reference radix tree: " + ref_lib().ref_last_error().decode())
    s = slice(0, n - 1)
    return dict(left=left[s].copy(), right=right[s].copy(), rangeFirst=rf[s].copy(),
                rangeLast=rl[s].copy(), prefixLength=pl[s].copy(), parent=parent)
