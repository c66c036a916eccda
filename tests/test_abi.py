"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import re
import subprocess
from pathlib import Path

from cpp_projects_b200 import _capi

ROOT = Path(__file__).resolve().parent.parent


def declared_in_headers():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(bfs_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_loads():
    lib = _capi.lib()
    assert lib.bfs_version().decode().startswith("bfs-b200")


def test_every_declared_symbol_is_exported():
    names = declared_in_headers()
    assert len(names) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", str(_capi.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (bfs_[a-z0-9_]+)", out))
    missing = sorted(names - exported)
    assert not missing, f"declared but not exported: {missing}"


def test_every_declared_symbol_has_a_binding():
    names = declared_in_headers()
    missing = sorted(n for n in names if n not in _capi.declared_symbols())
    assert not missing, f"declared in include/ but not bound in _capi: {missing}"


def test_bad_arguments_return_status_not_crash():
    lib = _capi.lib()
    plan = ctypes.c_void_p()
    desc = _capi.FdmtDesc(fmin=1600.0, fmax=1200.0, nchan=64, ncols=128, max_dt=64)
    st = lib.bfs_fdmt_plan_create_host(ctypes.byref(desc), ctypes.byref(plan))
    assert st == _capi.BFS_ERR_ARG
    assert b"fmin" in lib.bfs_last_error()
    desc = _capi.FdmtDesc(fmin=1200.0, fmax=1600.0, nchan=1, ncols=128, max_dt=64)
    assert lib.bfs_fdmt_plan_create_host(ctypes.byref(desc), ctypes.byref(plan)) == _capi.BFS_ERR_ARG


def test_header_is_plain_c(tmp_path):
    """include/bfs.h is a C header: it compiles as pedantic C99 and links
    against the library from a C program (no C++ types in the interface)."""
    src = tmp_path / "use.c"
    src.write_text('#include "bfs.h"\n#include <stdio.h>\n'
                   'int main(void) { bfs_guppi_session s; bfs_cand c; (void)s; (void)c;\n'
                   '  printf("%s\\n", bfs_version()); return 0; }\n')
    exe = tmp_path / "use"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", str(src),
                        "-I", str(ROOT / "include"), "-L", str(_capi.LIB_PATH.parent), "-lbfs_b200",
                        f"-Wl,-rpath,{_capi.LIB_PATH.parent}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.startswith("bfs-b200")
