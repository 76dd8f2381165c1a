"""The C-ABI library loads and exports every symbol include/aster_cuda.h
declares; CPU only (no compute call needs a GPU here)."""
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "aster_cuda.h"
LIB = ROOT / "aster_b200" / "libaster_cuda.so"


def declared():
    src = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|int|int64_t)\s+(aster_\w+)\s*\(", src, re.M)))


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


def test_library_built():
    assert LIB.exists(), "run python -m aster_b200.build"


def test_every_declared_symbol_exported():
    names = declared()
    assert len(names) >= 14
    missing = [n for n in names if n not in exported()]
    assert not missing, missing


def test_ctypes_binding_covers_header():
    from aster_b200 import api
    assert set(api.EXPORTS) <= set(declared())
    lib = api.load_library()
    for n in declared():
        assert hasattr(lib, n)


def test_product_does_not_link_the_oracle():
    out = subprocess.run(["ldd", str(LIB)], capture_output=True, text=True).stdout
    assert "oracle" not in out and "aster_ref" not in out


def test_strerror_without_gpu():
    from aster_b200 import api
    lib = api.load_library()
    assert lib.aster_strerror(0) == b"ok"
    assert b"stack" in lib.aster_strerror(5)
    assert lib.aster_version() >= 10000


def test_null_arguments_rejected():
    import ctypes
    from aster_b200 import api
    lib = api.load_library()
    assert lib.aster_ctx_create(None, 0, None) == 1          # ASTER_ERR_INVALID_ARG
    assert lib.aster_ctx_destroy(None) == 1
    assert lib.aster_allpairs(None, None, 0, None) == 1
    assert lib.aster_kdk_steps(None, None, 0, 0, 1) == 1


def test_params_struct_layout():
    import ctypes
    from aster_b200 import api
    assert ctypes.sizeof(api.CParams) == 5 * 8 + 4 * 4
    assert ctypes.sizeof(api.CTreeView) == 13 * 8 + 8


def test_graph_csv_layout():
    """The reference Graph files: "time,data" for one value per sample, a
    "time,Body0,...," header (trailing comma) for per-body graphs."""
    from aster_b200.api import graph_csv
    assert graph_csv([1, 2], [0.5, 0.25]) == "time,data\n1,0.5\n2,0.25\n"
    assert graph_csv([3], [[1.0, 2.0]]) == "time,Body0,Body1,\n3,1.0,2.0\n"
