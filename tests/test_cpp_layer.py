"""The C++ layer with the reference's names (nbb_simulation.hpp) and the
command-line driver: host-only parts on the CPU, the rest on the GPU."""
import os
import struct
import subprocess

import pytest

from conftest import PKG, ROOT

INC = [f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(PKG, 'cpp')}"]
CLI = os.path.join(PKG, "nbody")


def _compile(src, out, extra=()):
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", *INC, src, *extra, "-o", out])


def test_particle_file_loader(tmp_path):
    # tests/unit/cpu/particle_file_test.cpp of the reference, on the header
    exe = str(tmp_path / "particle_file_test")
    _compile(os.path.join(ROOT, "tests", "cpp", "particle_file_test.cpp"), exe,
             [f"-L{PKG}", "-lnbb", f"-Wl,-rpath,{PKG}"])
    out = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"


def _run_cli(*args):
    assert os.path.exists(CLI), "build the CLI with make -C amsc-nbody_b200"
    return subprocess.run([CLI, *args], capture_output=True, text=True)


def test_cli_argument_handling(tmp_path):
    # tests/scripts/simulation_cli_test.cmake:1-80 of the reference
    r = _run_cli("--help")
    assert r.returncode == 0 and "Usage:" in r.stdout
    assert "--time-step DT" in r.stdout and "--softening VALUE" in r.stdout
    r = _run_cli()
    assert r.returncode == 2 and "--input is required" in r.stderr
    r = _run_cli("--unknown")
    assert r.returncode == 2 and "Unknown option: --unknown" in r.stderr
    r = _run_cli("--input", "ignored.bin", "--time-step", "0.25", "--steps", "0")
    assert r.returncode == 2 and "Invalid positive integer for --steps" in r.stderr
    r = _run_cli("--input", str(tmp_path / "missing.bin"), "--time-step", "0.25", "--steps", "2")
    assert r.returncode == 1 and "Could not open particle input file" in r.stderr


def write_one_particle(path):
    """tests/support/write_particle_fixture.cpp: u64 count 1, then
    mass, x, y, z, vx, vy, vz = 2, 1, 2, -1, 2, -3, 0.5."""
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", 1))
        f.write(struct.pack("<7d", 2.0, 1.0, 2.0, -1.0, 2.0, -3.0, 0.5))


@pytest.mark.gpu
def test_cli_runs_a_simulation(tmp_path, nbb_mod):
    # tests/scripts/simulation_cli_test.cmake:82-105
    path = tmp_path / "one.bin"
    write_one_particle(path)
    r = _run_cli("--input", str(path), "--time-step", "0.25", "--steps", "2", "--theta", "0.6",
                 "--softening", "0.03")
    assert r.returncode == 0, r.stderr
    for text in ("Loaded 1 particles", "Simulation complete", "steps: 2", "simulated time: 0.5"):
        assert text in r.stdout


@pytest.mark.gpu
def test_cpp_simulation_layer(tmp_path, nbb_mod):
    exe = str(tmp_path / "shim_test")
    cuda = "/usr/local/cuda"
    _compile(os.path.join(ROOT, "tests", "cpp", "shim_test.cpp"), exe,
             [f"-I{cuda}/include", f"-L{PKG}", "-lnbb", f"-L{cuda}/lib64", "-lcudart",
              f"-Wl,-rpath,{PKG}"])
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"


def test_cli_frame_option_handling(tmp_path):
    # apps/simulation/main.cpp:165-205: frame options; the stream server is not built
    r = _run_cli("--input", "x.bin", "--time-step", "0.25", "--steps", "1", "--sample-rate", "0")
    assert r.returncode == 2 and "--sample-rate must be positive" in r.stderr
    r = _run_cli("--input", "x.bin", "--time-step", "0.25", "--steps", "1", "--stream-max-particles", "-3")
    assert r.returncode == 2 and "--stream-max-particles" in r.stderr
    r = _run_cli("--input", "x.bin", "--time-step", "0.25", "--steps", "1", "--cluster")
    assert r.returncode == 2 and "not part of this build" in r.stderr
    r = _run_cli("--help")
    assert "--stream-dir DIR" in r.stdout and "--sample-rate HZ" in r.stdout


@pytest.mark.gpu
def test_cli_writes_frames(tmp_path, nbb_mod):
    from nbb import frames

    path = tmp_path / "one.bin"
    write_one_particle(path)
    spool = tmp_path / "spool"
    r = _run_cli("--input", str(path), "--time-step", "0.25", "--steps", "3", "--stream-dir", str(spool),
                 "--sample-rate", "1000000")
    assert r.returncode == 0, r.stderr
    assert "frames written: 4" in r.stdout and "particles per frame: 1 of 1" in r.stdout
    names = sorted(os.listdir(spool))
    snaps = [n for n in names if n.endswith(".nbsnap")]
    assert len(snaps) == 4 and any(n.endswith(".complete") for n in names)
    with open(spool / snaps[-1], "rb") as f:
        h = frames.read_header(f.read())
    assert (h["version"], h["sequence"], h["simulation_step"], h["simulation_time"]) == (3, 3, 3, 0.75)


def test_build_api_header_compiles(tmp_path):
    # nbb_build.hpp with the reference's function-level names compiles as C++17
    # without CUDA headers (its buffers go through the C ABI)
    src = tmp_path / "t.cpp"
    src.write_text('#include "nbb_build.hpp"\nint main() { Tree t; MortonLeafGroups g; return t.nLeaves + g.nGroups; }\n')
    subprocess.check_call(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", *INC, str(src)])


BUILD_API_FIELDS = ["box", "keys", "idx", "uniq", "gfirst", "gcount", "left", "right", "rfirst", "rlast", "plen",
                    "rparent", "plan_level", "plan_count", "plan_offset", "children", "oparent", "olevel",
                    "oprefix", "ofirst", "ocount", "child_count", "cx", "cy", "cz", "half", "mass", "comx",
                    "comy", "comz"]
BUILD_API_TYPES = {"box": "<f8", "keys": "<u4", "idx": "<u4", "uniq": "<u4", "oprefix": "<u4", "cx": "<f8",
                   "cy": "<f8", "cz": "<f8", "half": "<f8", "mass": "<f8", "comx": "<f8", "comy": "<f8",
                   "comz": "<f8"}
BUILD_API_THETAS = (0.0, 0.3, 0.5, 0.7, 1.0)


def _read_build_api_output(path):
    import numpy as np

    data = open(path, "rb").read()
    pos, out = 0, {}

    def take(dtype):
        nonlocal pos
        (count,) = struct.unpack_from("<Q", data, pos)
        pos += 8
        a = np.frombuffer(data, dtype=dtype, count=count, offset=pos).copy()
        pos += a.nbytes
        return a

    for f in BUILD_API_FIELDS:
        out[f] = take(BUILD_API_TYPES.get(f, "<i4"))
    for theta in BUILD_API_THETAS:
        out[theta] = [take("<f8") for _ in range(3)]
    assert pos == len(data)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("recipe,n", [("plummer", 20000), ("blobs", 12000), ("plummer", 1)])
def test_build_api_transcription_matches_oracle(tmp_path, nbb_mod, oracle, recipe, n):
    """The reference accuracy harness's call sequence, compiled against
    nbb_build.hpp and run on the GPU: every intermediate and the
    accelerations of each theta equal the oracle's bit for bit."""
    import numpy as np
    from nbb import ics

    exe = str(tmp_path / "build_api_test")
    _compile(os.path.join(ROOT, "tests", "cpp", "build_api_test.cpp"), exe,
             [f"-L{PKG}", "-lnbb", f"-Wl,-rpath,{PKG}"])
    p = ics.plummer(max(n, 2), seed=8) if recipe == "plummer" else ics.blobs(n, seed=9)
    arrays = [np.ascontiguousarray(a[:n], dtype=np.float64) for a in (p.mass, p.x, p.y, p.z)]
    src = tmp_path / "in.bin"
    with open(src, "wb") as f:
        f.write(struct.pack("<Q", n))
        for a in arrays:
            f.write(a.tobytes())
    dst = tmp_path / "out.bin"
    r = subprocess.run([exe, str(src), str(dst)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"
    got = _read_build_api_output(dst)
    for theta in BUILD_API_THETAS:
        ref = oracle.pipeline(*arrays, theta=theta, soft=0.02, g=1.0)
        if theta == BUILD_API_THETAS[0]:
            assert np.array_equal(got["box"], np.asarray(ref["box"]))
            for f in BUILD_API_FIELDS[1:]:
                assert np.array_equal(got[f], ref[f]), f
        for a, b in zip(got[theta], (ref["ax"], ref["ay"], ref["az"])):
            assert np.array_equal(a, b), theta
