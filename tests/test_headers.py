"""The public headers compile on their own (C and C++) without a GPU."""
import os
import subprocess
import tempfile

from conftest import ROOT


def _compile(src: str, compiler: str, ext: str):
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "t" + ext)
        open(f, "w").write(src)
        r = subprocess.run([compiler, "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                            "-I", "/usr/local/cuda/include", f], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_c_header_is_plain_c():
    _compile('#include "vann.h"\nint main(void){ vann_params p; (void)p; return vann_abi_version() == VANN_ABI_VERSION ? 0 : 1; }\n',
             "gcc", ".c")


def test_cpp_mirror_header_compiles():
    _compile('#include "vann.hpp"\nint main(){ vann::VamanaParams p; (void)p; return 0; }\n', "g++", ".cpp")
