"""Frame capture: the oracle's restatement against the known answers of the
reference's frame tests (tests/unit/cpu/streaming_frame_test.cpp), and the
headless spool / sampler / reader in nbb.frames."""
import os

import numpy as np
import pytest


def _two_of_twenty():
    # 20 particles sampled down to 2 (indices 0 and 10); bounds and the
    # quantized payload of streaming_frame_test.cpp:99-147
    x = np.zeros(20); y = np.zeros(20); z = np.zeros(20)
    lo, hi = (-2.5, 3.5, -5.0), (1.25, 4.75, 6.125)
    x[:], y[:], z[:] = 0.0, 4.0, 0.0
    x[0], y[0], z[0] = hi[0], lo[1], lo[2]
    x[10], y[10], z[10] = lo[0], hi[1], hi[2]
    types = np.zeros(20, np.uint8)
    types[0], types[10] = 1, 4
    return x, y, z, types, lo, hi


def test_oracle_frame_matches_reference_known_answer(oracle):
    from nbb import frames

    x, y, z, types, lo, hi = _two_of_twenty()
    # non-sampled particles lie inside the bounds of the sampled two
    x[1:10] = x[11:] = -1.0
    y[1:10] = y[11:] = 4.0
    z[1:10] = z[11:] = 0.0
    frame = oracle.frame_capture(x, y, z, types, max_particles=2, sequence=7, step=42, time=0.5)
    assert len(frame) == 128 + 6 * 2 + 2
    h = frames.read_header(frame)
    assert (h["version"], h["header_bytes"], h["sequence"], h["simulation_step"]) == (3, 128, 7, 42)
    assert h["simulation_time"] == 0.5
    assert (h["source_particle_count"], h["particle_count"], h["components"], h["scalar_bytes"]) == (20, 2, 3, 2)
    assert (h["payload_bytes"], h["particle_type_bytes"]) == (14, 2)
    assert h["bounds_min"] == lo and h["bounds_max"] == hi
    assert frames.read_quantized(frame).ravel().tolist() == [65535, 0, 0, 0, 65535, 65535]
    assert frames.read_positions(frame).ravel().tolist() == [1.25, 3.5, -5.0, -2.5, 4.75, 6.125]
    assert frames.read_types(frame).tolist() == [1, 4]


def test_oracle_frame_collapsed_axis_quantizes_to_zero(oracle):
    from nbb import frames

    x = np.full(5, 8.0); y = np.linspace(-1.0, 3.0, 5); z = np.full(5, 5.0)
    frame = oracle.frame_capture(x, y, z, np.zeros(5, np.uint8))
    q = frames.read_quantized(frame)
    assert np.all(q[:, 0] == 0) and np.all(q[:, 2] == 0)
    assert q[:, 1].tolist() == [0, 16384, 32768, 49151, 65535]
    pos = frames.read_positions(frame)
    assert np.all(pos[:, 0] == 8.0) and np.all(pos[:, 2] == 5.0)
    assert abs(pos[2, 1] - 1.0) <= 4.0 / 65535.0


def test_oracle_frame_errors(oracle):
    x = np.zeros(4); y = np.zeros(4); z = np.zeros(4)
    bad = x.copy(); bad[2] = np.nan
    with pytest.raises(ValueError, match="-2"):
        oracle.frame_capture(bad, y, z, np.zeros(4, np.uint8))
    with pytest.raises(ValueError, match="-3"):
        oracle.frame_capture(x, y, z, np.array([0, 1, 5, 0], np.uint8))


def test_sampler_follows_the_reference_schedule():
    from nbb.frames import FrameSampler

    s = FrameSampler(60.0)
    assert s.is_due(0.0) and s.take_sequence() == 0
    assert not s.is_due(0.01)
    assert s.is_due(1.0 / 60.0) and s.take_sequence() == 1
    assert not s.is_due(0.02)
    assert s.is_due(2.0 / 60.0) and s.take_sequence() == 2
    s = FrameSampler(60.0)
    assert s.is_due(0.0) and s.is_due(10.0) and not s.is_due(10.0)
    with pytest.raises(ValueError):
        FrameSampler(0.0)
    with pytest.raises(ValueError):
        FrameSampler().is_due(-1.0)


def test_spool_names_publishes_and_refuses_overwrite(oracle, tmp_path):
    from nbb.frames import FrameSpool

    x, y, z, types, _, _ = _two_of_twenty()
    frame = oracle.frame_capture(x, y, z, types, sequence=3)
    spool = FrameSpool(str(tmp_path), "test-session")
    path = spool.write(frame)
    assert os.path.basename(path) == "run-test-session-frame-00000000000000000003.nbsnap"
    assert not os.path.exists(path + ".part")
    with open(path, "rb") as f:
        assert f.read() == frame
    with pytest.raises(RuntimeError):
        spool.write(frame)
    marker = spool.mark_complete()
    assert os.path.basename(marker) == "run-test-session.complete"
    with pytest.raises(ValueError):
        FrameSpool(str(tmp_path), "bad id")
