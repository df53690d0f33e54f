"""CPU checks of the C ABI: the library loads, exports every declared entry
point, and rejects bad arguments without touching a GPU."""
import ctypes as C
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(gl):
    lib = gl.load()
    names = gl._native.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert b"sm_100a" in lib.gpulsm_version()


def test_exported_symbols_match_nm(gl):
    out = subprocess.run(["nm", "-D", "--defined-only", gl._native.LIB_PATH], capture_output=True, text=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    for name in gl._native.header_functions():
        assert name in exported, name


def test_null_arguments_are_invalid(gl):
    lib = gl.load()
    N = gl._native
    assert lib.gpulsm_dict_create(None, None) == N.ERR_INVALID_ARGUMENT
    assert b"null" in lib.gpulsm_last_error()
    assert lib.gpulsm_dict_insert(None, None, None, 1, None) == N.ERR_INVALID_ARGUMENT
    assert lib.gpulsm_flix_create(None, None) == N.ERR_INVALID_ARGUMENT
    with pytest.raises(gl.InvalidArgument):
        N.check(lib.gpulsm_dict_lookup(None, None, 1, None, None, None))
    with pytest.raises(ValueError):
        N.check(lib.gpulsm_sort_pairs(None, None, None, None, 10, 48, 0, 32, None))
    assert lib.gpulsm_sort_pairs(None, None, None, None, 0, 32, 0, 32, None) == N.OK  # empty sort


def test_error_classes_map_reference_exceptions(gl):
    N = gl._native
    assert issubclass(gl.InvalidArgument, ValueError)
    assert issubclass(gl.OutOfDeviceMemory, MemoryError)
    assert issubclass(gl.CapacityError, RuntimeError)
    for code, cls in N._ERRORS.items():
        e = cls("x", code)
        assert e.status == code


def test_config_struct_layout_matches_header(gl):
    N = gl._native
    assert C.sizeof(N.DictConfig) == 8 * 3 + 4 * 4
    assert C.sizeof(N.FlixConfig) == 4 * 4 + 8


def test_every_ctypes_struct_matches_the_c_header(gl, tmp_path):
    """Size and every field offset of the ctypes mirrors, against a C program
    compiled from include/gpulsm.h (a field missing from the header fails the
    compile)."""
    N = gl._native
    pairs = [(N.DictConfig, "gpulsm_dict_config"), (N.FlixConfig, "gpulsm_flix_config"),
             (N.ServeStats, "gpulsm_serve_stats"), (N.LoadSpec, "gpulsm_load_spec")]
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "gpulsm.h"', "int main(void) {"]
    for cls, ctype in pairs:
        lines.append(f'  printf("{ctype} sizeof %zu\\n", sizeof({ctype}));')
        for name, _ in cls._fields_:
            lines.append(f'  printf("{ctype} {name} %zu\\n", offsetof({ctype}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(((a, b), int(c)) for a, b, c in
               (line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines()))
    for cls, ctype in pairs:
        assert got[(ctype, "sizeof")] == C.sizeof(cls), ctype
        for name, _ in cls._fields_:
            assert got[(ctype, name)] == getattr(cls, name).offset, (ctype, name)


def test_no_cpu_fallback_when_library_missing(tmp_path):
    """Importing the package from a copy without libgpulsm.so must fail loudly."""
    import shutil

    dst = tmp_path / "gpu-lsm-tree_b200"
    shutil.copytree(os.path.join(ROOT, "gpu-lsm-tree_b200"), dst,
                    ignore=shutil.ignore_patterns("*.so", "_build", "__pycache__"))
    shutil.copytree(os.path.join(ROOT, "include"), tmp_path / "include")
    code = ("import importlib,sys; sys.path.insert(0, %r); m = importlib.import_module('gpu-lsm-tree_b200');"
            "\ntry:\n  m.load()\nexcept ImportError as e:\n  print('LOUD', e)" % str(tmp_path))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert "LOUD" in r.stdout and "no CPU fallback" in r.stdout


def test_sort_entries_reject_partial_overlap_before_touching_memory(gl):
    """Both sort entries allow keys_out == keys_in (in place) but reject a
    partial overlap of any two buffers; the check is pointer arithmetic only,
    made before any pointer is dereferenced, so fake addresses are safe here."""
    lib = gl.load()
    N = gl._native
    base = 1 << 40
    for fn in (lib.gpulsm_sort_pairs, lib.gpulsm_sort_pairs_noalloc):
        # keys_out starts 4 bytes into keys_in: partial overlap
        assert fn(base, None, base + 4, None, 100, 32, 0, 32, None) == N.ERR_INVALID_ARGUMENT
        assert b"overlap" in lib.gpulsm_last_error()
        # values_out overlapping keys_out
        assert fn(base, base + 4096, base + 8192, base + 8192 + 64, 100, 32, 0, 32, None) == N.ERR_INVALID_ARGUMENT
        assert b"overlap" in lib.gpulsm_last_error()
