"""The C ABI on CPU: the library loads, exports every declared symbol, and
the ctypes structures match the header's layout (checked by compiling the
header with gcc).  No compute calls: there is no GPU here."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from magritte_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "magritte_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:mgr_status|const char \*)\s*(mgr_\w+)\s*\(", src, re.M)))


def test_header_declarations_match_binding_list():
    assert set(declared_functions()) == set(_capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mgr_\w+)", out))
    assert set(declared_functions()) <= exported


def test_version_string():
    assert b"sm_100a" in _capi.load().mgr_version()


def _cuda_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda_present(), reason="checks the no-device error path")
def test_create_without_device_reports_cuda_error():
    lib = _capi.load()
    h = C.c_void_p()
    assert lib.mgr_create(0, C.byref(h)) == 5
    assert not h.value
    assert lib.mgr_destroy(None) == 1


def test_struct_layout_matches_header():
    """offsetof/sizeof of every struct field from gcc vs the ctypes mirror."""
    structs = {"mgr_model_desc": _capi.ModelDesc, "mgr_colpar_desc": _capi.ColparDesc,
               "mgr_ali_opts": _capi.AliOpts, "mgr_mlp": _capi.MlpDesc,
               "mgr_train_opts": _capi.TrainOpts, "mgr_tuning": _capi.Tuning}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-o", exe, src], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    for line in out.strip().splitlines():
        cname, field, value = line.split()
        cls = structs[cname]
        got = C.sizeof(cls) if field == "sizeof" else getattr(cls, field).offset
        assert got == int(value), (cname, field, got, value)
