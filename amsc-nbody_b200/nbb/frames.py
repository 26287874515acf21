"""Quantized position frames (the reference's .nbsnap version-3 layout).

``Simulation.capture_frame`` returns a frame as bytes (built on the GPU by
nbb_sim_capture_frame); ``FrameSpool`` stores frames the way the reference's
spool does (src/streaming/frame.cpp:123-133, 341-500: run-<session>-frame-
<sequence, 20 digits>.nbsnap, written to a .part file and renamed, plus a
run-<session>.complete marker); ``read_header`` / ``read_positions`` /
``read_types`` decode a frame as the reference's readers do
(frame.cpp:520-720).  Headless: no viewer or network is involved.
"""
from __future__ import annotations

import os
import re
import struct
import time

import numpy as np

MAGIC = b"NBSNAP01"
QUANTIZED_MAX = 65535


def read_header(frame: bytes) -> dict:
    if frame[:8] != MAGIC:
        raise ValueError("not an N-body frame")
    version, header_bytes, sequence, step, sim_time, source, count, scalar, comps, payload = struct.unpack_from(
        "<IIQQdQQIIQ", frame, 8)
    h = dict(version=version, header_bytes=header_bytes, sequence=sequence, simulation_step=step,
             simulation_time=sim_time, source_particle_count=source, particle_count=count, scalar_bytes=scalar,
             components=comps, payload_bytes=payload, particle_type_bytes=0)
    if header_bytes >= 120:
        b = struct.unpack_from("<6d", frame, 72)
        h["bounds_min"], h["bounds_max"] = tuple(b[:3]), tuple(b[3:])
    if version == 3 and header_bytes == 128:
        h["particle_type_bytes"] = struct.unpack_from("<Q", frame, 120)[0]
    return h


def read_quantized(frame: bytes) -> np.ndarray:
    h = read_header(frame)
    return np.frombuffer(frame, dtype="<u2", count=3 * h["particle_count"], offset=h["header_bytes"]).reshape(-1, 3)


def read_positions(frame: bytes) -> np.ndarray:
    """float32 (count, 3): min + range * q / 65535, min where an axis collapses."""
    h = read_header(frame)
    q = read_quantized(frame).astype(np.float64)
    lo = np.array(h["bounds_min"])
    rng = np.array(h["bounds_max"]) - lo
    out = np.where(rng == 0.0, lo, lo + rng * q / QUANTIZED_MAX)
    return out.astype(np.float32)


def read_types(frame: bytes) -> np.ndarray:
    h = read_header(frame)
    if h["particle_type_bytes"] == 0:
        return np.zeros(h["particle_count"], np.uint8)
    off = h["header_bytes"] + 6 * h["particle_count"]
    return np.frombuffer(frame, dtype=np.uint8, count=h["particle_count"], offset=off).copy()


class FrameSampler:
    """At most `rate` frames per wall-clock second, skipping missed intervals
    (frame.cpp:151-176)."""

    def __init__(self, samples_per_second: float = 60.0):
        if not np.isfinite(samples_per_second) or samples_per_second <= 0.0:
            raise ValueError("Frame sample rate must be finite and positive")
        self.rate = samples_per_second
        self.interval = 1.0 / samples_per_second
        self.next_time = 0.0
        self.sequence = 0

    def is_due(self, elapsed: float) -> bool:
        if not np.isfinite(elapsed) or elapsed < 0.0:
            raise ValueError("Frame sampling time must be finite and non-negative")
        tol = np.finfo(float).eps * max(1.0, abs(elapsed)) * 8.0
        if elapsed + tol < self.next_time:
            return False
        skipped = np.floor(max(0.0, elapsed - self.next_time) / self.interval)
        self.next_time += (skipped + 1.0) * self.interval
        return True

    def take_sequence(self) -> int:
        s = self.sequence
        self.sequence += 1
        return s


class FrameSpool:
    def __init__(self, directory: str, session_id: str | None = None):
        if not directory:
            raise ValueError("Frame spool directory cannot be empty")
        self.session_id = session_id or f"{int(time.time() * 1e6)}-{os.getpid()}"
        if not re.fullmatch(r"[A-Za-z0-9_-]+", self.session_id):
            raise ValueError("Frame session id may contain only letters, numbers, '-' and '_'")
        self.directory = directory
        os.makedirs(directory, exist_ok=True)

    def frame_path(self, sequence: int) -> str:
        return os.path.join(self.directory, f"run-{self.session_id}-frame-{sequence:020d}.nbsnap")

    def write(self, frame: bytes) -> str:
        path = self.frame_path(read_header(frame)["sequence"])
        if os.path.exists(path):
            raise RuntimeError("Refusing to overwrite queued frame: " + path)
        with open(path + ".part", "wb") as f:
            f.write(frame)
        os.replace(path + ".part", path)
        return path

    def mark_complete(self) -> str:
        path = os.path.join(self.directory, f"run-{self.session_id}.complete")
        if not os.path.exists(path):
            with open(path + ".part", "w") as f:
                f.write(self.session_id + "\n")
            os.replace(path + ".part", path)
        return path
