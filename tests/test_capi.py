"""The C ABI library: loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "vann.h")).read()
    return sorted(set(re.findall(r"\b(vann_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import vann

    L = vann.lib()
    names = _declared()
    assert names, "no declarations parsed"
    for n in names:
        assert hasattr(L, n), n
    assert sorted(vann.EXPORTS) == names


def test_status_strings_and_abi_version():
    import vann

    L = vann.lib()
    assert L.vann_abi_version() == vann.ABI_VERSION == 2
    assert L.vann_status_string(0) == b"ok"
    assert L.vann_status_string(5) == b"hop limit reached"


def test_invalid_params_fail_without_touching_the_gpu():
    import vann

    p = vann.Params(130, 64, 100, 1.2, 1000, 600, 500, 0, 0)  # dim not a multiple of 4
    h = ctypes.c_void_p()
    st = vann.lib().vann_create(ctypes.byref(p), ctypes.byref(h))
    assert st == vann.ERR_UNSUPPORTED
    assert b"multiple of 4" in vann.lib().vann_last_error()
    p = vann.Params(128, 200, 100, 1.2, 1000, 600, 500, 0, 0)  # degree > 128
    assert vann.lib().vann_create(ctypes.byref(p), ctypes.byref(h)) == vann.ERR_UNSUPPORTED
