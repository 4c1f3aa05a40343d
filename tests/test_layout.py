"""Device layout of the radiation and thermodynamics fields (trg_types.h):
every (field, cell) pair has its own slot, a cell's four optical depths fill
one aligned 32-byte group (the unit the causal sweep reads from a neighbour)
and its two column densities one 16-byte pair.  Compiled on the host."""
import os
import subprocess

import pytest

import common

SRC = os.path.join(common.HERE, "host_harness", "layout_check.cpp")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("layout") / "layout_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", exe, SRC], check=True)
    return exe


@pytest.mark.parametrize("n", [1, 7, 4096, 35937])
def test_layout_is_one_to_one_and_grouped(checker, n):
    r = subprocess.run([checker, str(n)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
