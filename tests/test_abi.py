"""The C ABI library loads on a machine without a GPU and exports every entry
point include/falcondb_b200.h declares; the Python binding covers them all."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "falcondb_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for must in ["fdb_open", "fdb_close", "fdb_sql", "fdb_result_free", "fdb_filter_count", "fdb_aggregate",
                 "fdb_group_by_codes", "fdb_group_by_i64", "fdb_join_build", "fdb_join_probe_agg", "fdb_topk"]:
        assert must in syms


def test_library_exports_every_declared_symbol():
    import falcondb_b200 as F

    lib = ctypes.CDLL(str(F.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_covers_every_symbol():
    import falcondb_b200 as F

    assert sorted(F.EXPORTED) == declared_symbols()
    F.lib()  # signatures applied without error
    assert "sm_100a" in F.version()


def test_rust_binding_in_integration_doc_covers_every_symbol():
    """The Rust `extern "C"` block a FalconDB maintainer would add (the
    integration guide) declares every entry point of the header."""
    doc = (ROOT / "INTEGRATION.md").read_text()
    block = doc[doc.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    bound = set(re.findall(r"pub fn (fdb_[a-z0-9_]+)\(", block))
    assert sorted(set(declared_symbols()) - bound) == []


def test_open_without_gpu_fails_loudly():
    """No CPU fallback: opening a context needs a CUDA device."""
    import falcondb_b200 as F
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(F.FalconError):
        F.Database(0)
    assert F.lib().fdb_last_error()


def test_oracle_library_loads():
    from oracle import oracle as O

    O.lib()
    assert O.hardware_threads() >= 1
