"""The C-ABI library loads and exports every entry point include/torch_b200.h declares."""
import ctypes
import os
import re

import pytest

import common
import torch_b200

HEADER = os.path.join(common.ROOT, "include", "torch_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(trg_[a-z_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("trg_create", "trg_full_step", "trg_run_steps", "trg_component", "trg_get_state",
              "trg_last_error", "trg_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    path = torch_b200.library_path()
    if not os.path.exists(path):
        pytest.fail(f"{path} missing: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    bound = {n for n, _, _ in torch_b200._SIGNATURES}
    assert set(declared_functions()) <= bound


def test_params_struct_matches_header_fields():
    text = open(HEADER).read()
    body = text[text.index("typedef struct trg_params"):text.index("} trg_params;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = re.findall(r"\b([a-zA-Z_][a-zA-Z0-9_]*)\s*(?:\[\d\])?\s*[,;]", body)
    assert names == [f[0] for f in torch_b200.TrgParams._fields_]
