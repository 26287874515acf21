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
