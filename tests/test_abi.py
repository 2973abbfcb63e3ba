"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(dfm_\w+)\s*\(", src, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def so():
    from delfem_b200 import build, lib
    build.build()
    return ctypes.CDLL(lib.LIB_PATH)


def test_every_declared_symbol_is_exported(so):
    names = declared_symbols()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from delfem_b200 import lib
    assert set(declared_symbols()) == set(lib.PROTOS), set(declared_symbols()) ^ set(lib.PROTOS)


def test_library_loads_and_reports_version(so):
    from delfem_b200 import lib
    L = lib.load()
    assert L.dfm_abi_version() == 1
    assert L.dfm_status_string(lib.WAIT_TIMEOUT) == b"device wait timeout"


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from delfem_b200 import lib
    with pytest.raises(RuntimeError):
        lib.Context(0)
