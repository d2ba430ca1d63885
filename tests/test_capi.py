"""The C-ABI library loads on CPU and exports every symbol include/tdp.h declares."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    txt = (ROOT / "include" / "tdp.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tdp_[a-z0-9_]+)\s*\(", txt)))


def test_header_symbols_exported(pkg):
    L = pkg.tdp.lib()
    names = declared_symbols()
    assert names, "no declarations found"
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(pkg.tdp.EXPORTED)


def test_no_device_is_an_error_not_a_crash(pkg):
    import torch
    if torch.cuda.is_available():
        return
    L = pkg.tdp.lib()
    h = ctypes.c_void_p()
    rc = L.tdp_ctx_create(0, 0, 0, ctypes.byref(h))
    assert rc == 7  # TDP_ERR_NODEV
