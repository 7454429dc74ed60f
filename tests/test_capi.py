"""CPU checks of the C-ABI boundary: the library loads, exports every symbol
include/b40c_bfs.h declares, and rejects bad arguments with cudaError_t codes
(no compute call needs a GPU here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "b40c_bfs.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b40c_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_api():
    syms = declared_symbols()
    for name in ["b40c_problem_create", "b40c_problem_from_host", "b40c_problem_reset",
                 "b40c_problem_extract_results", "b40c_enactor_create", "b40c_enact_search",
                 "b40c_enactor_get_statistics", "b40c_enactor_frontier_type"]:
        assert name in syms


def test_library_exports_every_declared_symbol():
    from back40computing_b200._lib import LIB_PATH, SIGNATURES
    so = ctypes.CDLL(str(LIB_PATH))
    for name in declared_symbols():
        assert hasattr(so, name), f"{name} declared in b40c_bfs.h but not exported"
        assert name in SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_error_string():
    from back40computing_b200 import bfs, graphs
    assert "sm_100a" in bfs.version()
    with pytest.raises(graphs.GraphError, match="invalid width"):
        graphs.grid2d(-3)


def test_invalid_arguments_rejected_without_gpu():
    from back40computing_b200._lib import lib
    L = lib()
    assert L.b40c_enactor_create(7, 0, 0, ctypes.byref(ctypes.c_void_p())) == 1
    assert L.b40c_enactor_set_policy(None, 256, 0, 0, 0, 0) == 1
    assert L.b40c_enactor_frontier_type(None, None) == 1
    assert L.b40c_problem_reset(None, 0, 1.0) == 401
    assert L.b40c_debug_barrier_timeout(0, 10) == 1


def test_product_never_imports_the_oracle():
    for path in (ROOT / "back40computing_b200").rglob("*.py"):
        src = path.read_text()
        assert "oracle" not in re.sub(r"#.*", "", src).replace("oracle/", ""), path


def test_library_is_not_older_than_its_sources():
    """A failed build keeps the previous .so; this catches running it stale."""
    from back40computing_b200 import build
    lib = build.LIB
    assert lib.exists(), "libb40c_bfs.so not built"
    newest = max(p.stat().st_mtime for p in list(build.CSRC.iterdir()) + [build.INCLUDE / "b40c_bfs.h"])
    assert lib.stat().st_mtime >= newest, "libb40c_bfs.so is older than csrc/: rebuild"
