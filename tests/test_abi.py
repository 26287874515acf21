"""The C-ABI boundary without a GPU: the library loads, exports every entry
point include/nbb.h declares, and the header compiles as C and C++."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "nbb.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nbb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_simulation_surface():
    names = declared_functions()
    for required in ("nbb_sim_create", "nbb_sim_initialize", "nbb_sim_step", "nbb_sim_run",
                     "nbb_sim_time", "nbb_sim_step_number", "nbb_sim_state", "nbb_sim_destroy",
                     "nbb_accel", "nbb_accel_direct", "nbb_accel_octree", "nbb_kick_drift",
                     "nbb_kick", "nbb_radix_tree", "nbb_octree_from_keys", "nbb_sim_export"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import nbb._lib as L

    assert os.path.exists(L.LIB_PATH), "libnbb.so must be built (make -C amsc-nbody_b200)"
    lib = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_table_matches_header():
    import nbb._lib as L

    declared = set(declared_functions())
    assert set(L.SIGNATURES) <= declared


@pytest.mark.parametrize("lang,flags", [("c", ["-std=c11"]), ("c++", ["-std=c++17"])])
def test_header_compiles(lang, flags, tmp_path):
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    src.write_text('#include "nbb.h"\nint main(void){nbb_config c; nbb_config_default(&c); return 0;}\n')
    cc = "gcc" if lang == "c" else "g++"
    subprocess.check_call([cc, *flags, "-Wall", "-Werror", "-fsyntax-only", "-I",
                           os.path.join(ROOT, "include"), str(src)])


def test_library_fails_loudly_without_device():
    """On a machine without a GPU the library loads and every call reports
    NBB_ERR_NO_DEVICE (or a CUDA error) -- there is no CPU fallback."""
    from conftest import HAS_GPU

    if HAS_GPU:
        pytest.skip("a GPU is present")
    import numpy as np

    import nbb

    with pytest.raises((nbb.NoDevice, nbb.DeviceError)):
        nbb.compute_accelerations((np.ones(4), np.arange(4.0), np.zeros(4), np.zeros(4)), 0.5, 0.01)


# The ctypes mirrors in nbb/_lib.py and the C structs they stand for.
STRUCTS = {"Config": "nbb_config", "StateView": "nbb_state_view", "Stats": "nbb_stats",
           "TreeExport": "nbb_tree_export", "Diagnostics": "nbb_diagnostics", "OctreeView": "nbb_octree_view"}


def test_python_structs_match_the_header_layout(tmp_path):
    """Every struct the Python binding passes through the C ABI has the size
    and field offsets the compiler gives the header's declaration."""
    import nbb._lib as L

    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "nbb.h"', 'int main(void) {']
    for py, c in STRUCTS.items():
        lines.append(f'  printf("{py} sizeof %zu\\n", sizeof({c}));')
        for field, _ in getattr(L, py)._fields_:
            lines.append(f'  printf("{py} {field} %zu\\n", offsetof({c}, {field}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           str(src), "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        py, field, value = line.split()
        got[(py, field)] = int(value)
    for py in STRUCTS:
        cls = getattr(L, py)
        assert got[(py, "sizeof")] == ctypes.sizeof(cls), py
        for field, _ in cls._fields_:
            assert got[(py, field)] == getattr(cls, field).offset, (py, field)
