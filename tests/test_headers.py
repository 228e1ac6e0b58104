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


def test_ctypes_mirror_matches_the_c_structs():
    """Every public struct of vann.h has the size and field offsets of its ctypes mirror
    (a mismatch would pass garbage across the ABI without any error)."""
    import ctypes

    import vann

    pairs = [("vann_params", vann.Params), ("vann_search_params", vann.SearchParams), ("vann_info", vann.Info),
             ("vann_server_params", vann.ServerParams), ("vann_server_stats", vann.ServerStats)]
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "vann.h"', "int main(void) {"]
    for cname, py in pairs:
        lines.append(f'    printf("{cname} sizeof() %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("    return 0;\n}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
        open(src, "w").write("\n".join(lines))
        r = subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", src, "-o",
                            exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {(a, b): int(c) for a, b, c in (ln.split() for ln in out if ln)}
    for cname, py in pairs:
        assert got[(cname, "sizeof()")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
