"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares; the Python binding covers the same set."""
import ctypes
import glob
import os
import re
import subprocess

from scp_b200 import native, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(scp_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_abi():
    names = declared_functions()
    assert {"scp_gpu_init", "scp_gpu_step", "scp_gpu_diag", "scp_gpu_free"} <= names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(n for n in declared_functions() if n.startswith("scp_gpu_")) <= set(native.EXPORTS)


def _c_layout(struct, fields, tmp_path):
    src = tmp_path / "layout.c"
    body = "".join(f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields)
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "scp_gpu.h"\n'
                   f'int main(void){{printf("%zu\\n", sizeof({struct}));{body}return 0;}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    return [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]


def test_struct_layouts_match_c(tmp_path):
    for struct, cls in (("scp_gpu_params", params.CParams), ("scp_gpu_info", native.Info),
                        ("scp_gpu_diag_out", native.DiagOut)):
        fields = [f for f, _ in cls._fields_]
        got = _c_layout(struct, fields, tmp_path)
        assert got[0] == ctypes.sizeof(cls), struct
        assert got[1:] == [getattr(cls, f).offset for f in fields], struct


def test_errstr_and_version_without_gpu():
    lib = native.lib()
    assert lib.scp_gpu_abi_version() == 6
    assert lib.scp_gpu_errstr(-4).decode().startswith("gauged periodic")
    assert lib.scp_gpu_errstr(0).decode() == "ok"


def test_init_rejects_bad_params_without_touching_gpu():
    lib = native.lib()
    p = params.Params(N=2).to_c()
    h = ctypes.c_void_p()
    arr = (ctypes.c_void_p * 24)()
    assert lib.scp_gpu_init(ctypes.byref(p), arr, ctypes.byref(h)) == -1
