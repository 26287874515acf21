"""Every file:line citation of the reference in the library, the oracle, the
tests and the documents points inside the cited file.

A citation is `path:line` or `path:first-last` (optionally followed by
`,first-last` ranges), where `path` is the reference file's path within its
project or, when that is unambiguous, its bare file name.  The reference tree
is taken from NBB_REFERENCE or from a `reference` directory beside this
repository; without either the test is skipped.
"""
import collections
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCANNED = ("include", "amsc-nbody_b200", "oracle", "tests", "bench.py", "__graft_entry__.py",
           "DESIGN.md", "INTEGRATION.md", "README.md")
SKIP_DIRS = {"_ref", "_build", "__pycache__", "golden"}
SUFFIXES = (".cu", ".cuh", ".h", ".hpp", ".cpp", ".c", ".py", ".md", "Makefile")
# bare names that exist more than once in the reference mean its top-level file
TOP_LEVEL = {"README.md", "CMakeLists.txt"}
CITATION = re.compile(r"([A-Za-z0-9_./-]+\.(?:cu|hpp|cpp|h|cuh|md|py|cmake|sh|txt))"
                      r":(\d+)(?:[-–](\d+))?((?:,\d+(?:[-–]\d+)?)*)")


def reference_root():
    for path in (os.environ.get("NBB_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if path and os.path.isdir(os.path.join(path, "gpu", "cuda_kernels")):
            return path
    return None


def scanned_files():
    for top in SCANNED:
        path = os.path.join(ROOT, top)
        if os.path.isfile(path):
            yield path
            continue
        for d, dirs, files in os.walk(path):
            dirs[:] = [x for x in dirs if x not in SKIP_DIRS]
            for f in files:
                if f.endswith(SUFFIXES):
                    yield os.path.join(d, f)


def own_names():
    names = set()
    for d, dirs, files in os.walk(ROOT):
        dirs[:] = [x for x in dirs if x not in {".git", "_work", "gpurun_out", "_ref", "_build"}]
        names.update(files)
    return names - TOP_LEVEL


def citations(ref):
    """(citing file, line, text, reference file or None when unresolved,
    [(first, last), ...]) of every reference citation."""
    files = []
    for d, _, fs in os.walk(ref):
        files += [os.path.relpath(os.path.join(d, f), ref) for f in fs]
    by_name = collections.defaultdict(list)
    for f in files:
        by_name[os.path.basename(f)].append(f)
    ours = own_names()
    for path in scanned_files():
        with open(path, errors="replace") as h:
            for ln, line in enumerate(h, 1):
                for m in CITATION.finditer(line):
                    name = m.group(1)
                    base = os.path.basename(name)
                    if base not in by_name or (base in ours and "/" not in name):
                        continue  # not a reference file name, or one of this repository's files
                    if "/" in name:
                        target = [f for f in files if f == name]
                    elif base in TOP_LEVEL:
                        target = [base]
                    else:
                        target = by_name[base]
                    ranges = [(int(m.group(2)), int(m.group(3) or m.group(2)))]
                    for a, b in re.findall(r",(\d+)(?:[-–](\d+))?", m.group(4) or ""):
                        ranges.append((int(a), int(b or a)))
                    resolved = target[0] if len(target) == 1 else None
                    yield os.path.relpath(path, ROOT), ln, m.group(0), resolved, ranges


def test_reference_citations_point_inside_the_cited_files():
    ref = reference_root()
    if ref is None:
        pytest.skip("reference sources not present (set NBB_REFERENCE)")
    lengths = {}
    bad, count = [], 0
    for where, ln, text, target, ranges in citations(ref):
        count += 1
        if target is None:
            bad.append(f"{where}:{ln}: {text} does not name one reference file")
            continue
        if target not in lengths:
            with open(os.path.join(ref, target), "rb") as h:
                lengths[target] = h.read().count(b"\n") + 1
        for first, last in ranges:
            if not 1 <= first <= last <= lengths[target]:
                bad.append(f"{where}:{ln}: {text} outside {target} ({lengths[target]} lines)")
    assert count > 100, count
    assert not bad, "\n".join(bad)
