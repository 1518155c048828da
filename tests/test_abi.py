"""CPU checks of the C ABI: the library builds, loads and exports every declared symbol;
argument errors come back as status codes (no GPU needed for these)."""
import ctypes as C
import os
import re

import pytest

from grainrecon_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "grainrecon_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(grc_[a-z_0-9]+)\s*\(", src)))


def test_header_matches_binding_list():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_null_context_is_an_error_not_a_crash():
    L = _lib.load()
    assert L.grc_sync(None) == _lib.GRC_EINVAL
    assert L.grc_forward_comp(None, *([None] * 2), 0, *([None] * 8)) == _lib.GRC_EINVAL
    assert L.grc_grow_indexed_region(None, None, 0, *([None] * 10)) == _lib.GRC_EINVAL
    assert L.grc_last_error(None) == b"NULL context"


def test_ctx_create_without_device_reports_status():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    L = _lib.load()
    h = C.c_void_p()
    assert L.grc_ctx_create(C.byref(h), 0) != _lib.GRC_OK
    assert not h.value


def test_no_cpu_fallback_in_product_path():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "grainrecon_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".h", ".cuh")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in re.sub(r"#.*|//.*", "", txt).replace("the oracle", ""), f


def test_map_key_follows_content_not_address():
    """grc_map_key (a host function): equal contents in different buffers give equal keys; a
    changed sampled value, a different size or a changed value of a fully sampled map change it."""
    import numpy as np
    rng = np.random.default_rng(0)
    a = rng.random(1_000_003).astype(np.float32)
    b = a.copy()
    assert _lib.map_key(a, 4096) == _lib.map_key(b, 4096) != 0
    b[0] += 1  # the first value is always sampled
    assert _lib.map_key(a, 4096) != _lib.map_key(b, 4096)
    b[:] = a
    b[-1] += 1  # and the last
    assert _lib.map_key(a, 4096) != _lib.map_key(b, 4096)
    assert _lib.map_key(a[:-1], 4096) != _lib.map_key(a, 4096)
    small = rng.random(1000).astype(np.float32)
    for i in (1, 500, 998):  # every value of a map no larger than the sample count
        c = small.copy()
        c[i] = -c[i]
        assert _lib.map_key(c, 4096) != _lib.map_key(small, 4096)


def _struct_fields(name):
    """(type, field) pairs of a typedef struct in the header."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct\s*\{(.*?)\}\s*" + name + r"\s*;", src, flags=re.S).group(1)
    return [tuple(m) for m in re.findall(r"(\w+)\s+(\w+)\s*;", body)]


def test_stats_struct_matches_binding():
    """grc_stats is read through ctypes: same fields, same order, same widths."""
    widths = {"int64_t": 8, "double": 8, "int32_t": 4, "int": 4}
    fields = _struct_fields("grc_stats")
    assert [f for _, f in fields] == [f for f, _ in _lib.Stats._fields_]
    assert sum(widths[t] for t, _ in fields) == C.sizeof(_lib.Stats)
