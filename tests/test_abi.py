"""The C ABI: header declarations, library exports and the ctypes table agree (no GPU needed)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wql3d.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(wql3d_\w+)\s*\(", src, flags=re.M))


@pytest.fixture(scope="module")
def lib_path():
    from waveqlab3d_q_gpu_b200 import build
    return build.build()


def test_header_declares_the_entry_points():
    names = declared()
    assert "wql3d_domain_create" in names and "wql3d_run" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (wql3d_\w+)", out))
    missing = declared() - exported
    assert not missing, missing


def test_library_loads_and_binds_all_symbols(lib_path):
    from waveqlab3d_q_gpu_b200 import _lib
    L = _lib.load()
    for name in declared():
        assert hasattr(L, name)
    assert set(_lib.SIGNATURES) == declared()


def test_errors_without_device_are_status_codes(lib_path):
    """Argument checks return WQL3D_EINVAL with a message instead of exiting."""
    import ctypes as C
    from waveqlab3d_q_gpu_b200 import _lib
    L = _lib.load()
    assert L.wql3d_domain_create(None, None) == -1
    assert b"null" in L.wql3d_last_error()
    assert L.wql3d_scale_rate_array(None, 10, 1.0, None) == -1
    assert L.wql3d_update_state_array(None, None, 0, 1.0, None) == 0
    d = _lib.DomainDesc()
    d.abi_version = 999
    h = C.c_void_p()
    assert L.wql3d_domain_create(C.byref(d), C.byref(h)) == -1
    assert b"ABI" in L.wql3d_last_error()


def test_descriptor_layout_matches_header(lib_path, tmp_path):
    """sizeof/offsetof of the descriptors in C equal the ctypes mirror."""
    import ctypes as C
    from waveqlab3d_q_gpu_b200 import _lib
    prog = tmp_path / "layout.c"
    fields = [f for f, _ in _lib.DomainDesc._fields_]
    bfields = [f for f, _ in _lib.BlockDesc._fields_]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wql3d.h"', 'int main(void){',
             'printf("%zu %zu\\n", sizeof(wql3d_domain_desc), sizeof(wql3d_block_desc));']
    for f in fields:
        lines.append(f'printf("%zu\\n", offsetof(wql3d_domain_desc, {f}));')
    for f in bfields:
        lines.append(f'printf("%zu\\n", offsetof(wql3d_block_desc, {f}));')
    lines.append("return 0;}")
    prog.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == C.sizeof(_lib.DomainDesc) and vals[1] == C.sizeof(_lib.BlockDesc)
    offs = vals[2:]
    assert offs[:len(fields)] == [getattr(_lib.DomainDesc, f).offset for f in fields]
    assert offs[len(fields):] == [getattr(_lib.BlockDesc, f).offset for f in bfields]
