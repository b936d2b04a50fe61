"""The C-ABI libraries load without a GPU and export every function include/*.h declares."""
import ctypes
import os
import re

import pytest

from poststackmig3d_b200 import _lib
from poststackmig3d_b200 import host as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(psm_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header,loader", [("psm.h", _lib.cuda), ("psm_host.h", H.host)])
def test_every_declared_symbol_is_exported(header, loader):
    names = declared(header)
    assert names, header
    lib = loader()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_calls_fail_cleanly():
    L = _lib.cuda()
    n = ctypes.c_int(-1)
    assert L.psm_device_count(ctypes.byref(n)) == 0 and n.value >= 0
    assert L.psm_version().startswith(b"poststackmig3d-b200")
    # argument errors are reported without touching a device
    assert L.psm_set_traces(None, None) == -1
    assert L.psm_destroy(None) == 0


def test_binary_usage_message():
    import subprocess
    r = subprocess.run([H.binary_path()], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage:" in r.stderr
