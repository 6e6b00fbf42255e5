"""The C-ABI library loads without a GPU and exports every symbol the
include/*.h headers declare; the oracle library loads too."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols(headers=None):
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        if headers is not None and h.name not in headers:
            continue
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(gpudb_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def engine_symbols():
    return [s for s in declared_symbols() if s not in set(declared_symbols({"gpudb_datagen.h"}))]


def test_headers_declare_entry_points():
    syms = declared_symbols()
    assert "gpudb_create" in syms and "gpudb_query_run" in syms and "gpudb_gen_fact" in syms
    assert len(syms) > 40


def test_library_exports_every_declared_symbol():
    from gpudbmetalcodegen_b200 import _lib
    lib = _lib.load()
    missing = [s for s in engine_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # the data generators live in their own library, which maps no engine code
    dg = _lib.load_datagen()
    missing = [s for s in declared_symbols({"gpudb_datagen.h"}) if not hasattr(dg, s)]
    assert not missing, missing
    assert not hasattr(dg, "gpudb_create") and not hasattr(dg, "gpudb_query_run")
    assert not [s for s in declared_symbols({"gpudb_datagen.h"}) if hasattr(lib, s)]


def test_python_bindings_cover_every_declared_symbol():
    from gpudbmetalcodegen_b200 import _lib
    assert set(engine_symbols()) <= set(_lib.EXPORTED)
    assert set(declared_symbols({"gpudb_datagen.h"})) <= set(_lib.DATAGEN_EXPORTED)


def test_no_gpu_create_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gpudbmetalcodegen_b200.engine import Context
    from gpudbmetalcodegen_b200._lib import GpudbError
    with pytest.raises(GpudbError) as e:
        Context(0)
    assert e.value.status in (-8, -6)


def test_version_and_templates():
    from gpudbmetalcodegen_b200 import _lib, engine
    assert b"sm_100a" in _lib.load().gpudb_version()
    t = engine.templates()
    for name in ("q1", "q6", "join_topk", "groupby", "hashjoin", "mix_topk"):
        assert name in t


def test_oracle_library_loads():
    from oracle import oracle_py
    lib = oracle_py.lib()
    assert hasattr(lib, "oracle_q1") and hasattr(lib, "oracle_join_topk")
