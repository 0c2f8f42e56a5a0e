"""The neighbour-list layout of the pair kernels, checked on the host.

tests/list_layout_check.cpp includes md-force-routines_b200/csrc/p3m_list_layout.h,
the header nvcc compiles into the list builder and the pair loops, and checks
for TPI 1, 2, 4 and 8 and several list capacities that the writer's index is a
bijection onto the list array, that every read and inner-list store of the pair
kernels lands on the writer's slot of the entry it means, that vector accesses
are aligned, and that a warp's chunk is one contiguous run. A second build with
every reader address moved by one entry must fail.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "list_layout_check.cpp")
INC = os.path.join(ROOT, "md-force-routines_b200", "csrc")


def _build(tmp_path, name, *defs):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / name)
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", INC, *defs, "-o", exe, SRC],
                   check=True)
    return exe


def test_list_layout_reads_match_writes(tmp_path):
    r = subprocess.run([_build(tmp_path, "llc")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok "), r.stdout
    assert int(r.stdout.split()[1]) > 1_000_000


def test_list_layout_check_catches_a_misplaced_read(tmp_path):
    r = subprocess.run([_build(tmp_path, "llc_skew", "-DPLANT_SKEW=1")], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 1, r.stdout
    assert r.stdout.startswith("FAIL"), r.stdout
