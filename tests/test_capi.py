"""The C-ABI library builds, loads and exports every symbol the public
header declares (no GPU needed: nothing here launches a kernel)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "octopus_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"OCT_API\s+[\w\s\*]+?\b(oct_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "oct_tree_build" in names and "oct_edges_fill" in names and "oct_edges_diff_backward" in names
    assert len(names) >= 16


def test_library_exports_every_declared_symbol(ob):
    lib = ob._lib.load()
    so = ob._lib.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for name in declared():
        assert name in exported, name
        assert getattr(lib, name) is not None
    # the ctypes table covers exactly the declared set
    assert sorted(ob._lib.declared_symbols()) == declared()


def test_version_and_status_strings(ob):
    lib = ob._lib.load()
    assert lib.oct_version() >= 10000
    assert lib.oct_status_string(3) == b"InexactError"
    assert lib.oct_status_string(1) == b"ArgumentError"


def test_null_arguments_are_rejected_without_a_device(ob):
    lib = ob._lib.load()
    assert lib.oct_ctx_create(0, None) == ob._lib.ERR_ARGUMENT
    assert lib.oct_tree_build(None, None, None, 0, 1.0, 0) == ob._lib.ERR_ARGUMENT
    assert lib.oct_edges_count(None, None, None, 0, None) == ob._lib.ERR_ARGUMENT
    assert lib.oct_ctx_destroy(None) == ob._lib.OK
    assert lib.oct_ctx_set_option(None, ob._lib.OPT_WAIT_LIMIT, 10) == ob._lib.ERR_ARGUMENT
    assert lib.oct_ctx_get_option(None, ob._lib.OPT_WAIT_LIMIT, None) == ob._lib.ERR_ARGUMENT
    assert lib.oct_edges_count_noalloc(None, None, None, 1, None, None, None) == ob._lib.ERR_ARGUMENT
    assert lib.oct_ctx_last_error(None) == b""


def test_oracle_is_not_linked_into_the_library(ob):
    out = subprocess.run(["nm", "-D", ob._lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    assert "oracle_" not in out
    ldd = subprocess.run(["ldd", ob._lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in ldd
