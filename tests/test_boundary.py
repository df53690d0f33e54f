"""The reference-side boundary: include/gpulsmopt_b200.cuh keeps class
GPULSMOpt's surface (GPULSMOpt.cuh:5599-5881) over the C ABI, and FliX's own
GPULSMOpt adapter (FliX/impl_gpulsmopt.cuh:137-311) builds against it with its
one include line redirected (oracle/Makefile, oracle/flix_adapter_shim.cu)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libflix_gpulsmopt_adapter.so")
REFERENCE = os.environ.get("GPULSM_REFERENCE")


def _declared_abi():
    with open(os.path.join(ROOT, "include", "gpulsm.h")) as f:
        text = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    return set(re.findall(r"\b(gpulsm_[a-z0-9_]+)\s*\(", text))


def test_shim_header_uses_only_declared_entry_points():
    with open(os.path.join(ROOT, "include", "gpulsmopt_b200.cuh")) as f:
        used = set(re.findall(r"\b(gpulsm_[a-z0-9_]+)\s*\(", f.read()))
    assert used and used <= _declared_abi(), used - _declared_abi()


@pytest.mark.skipif(not os.path.exists(ADAPTER), reason="adapter not built (oracle/Makefile with a reference checkout)")
def test_built_adapter_binds_only_to_the_c_abi():
    """The FliX adapter library resolves its dictionary calls in libgpulsm.so:
    every gpulsm_* symbol it imports is declared in include/gpulsm.h, and it
    carries no GPULSMOpt engine of its own."""
    und = subprocess.run(["nm", "-D", "--undefined-only", ADAPTER], capture_output=True, text=True).stdout
    imported = {line.split()[-1] for line in und.splitlines() if "gpulsm_" in line}
    assert {"gpulsm_dict_create", "gpulsm_dict_insert", "gpulsm_dict_lookup", "gpulsm_dict_range_sum",
            "gpulsm_dict_successor", "gpulsm_dict_erase", "gpulsm_dict_bulk_build"} <= imported
    assert imported <= _declared_abi()
    defined = subprocess.run(["nm", "-DC", "--defined-only", ADAPTER], capture_output=True, text=True).stdout
    assert "gpulsmopt2_detail" not in defined  # no reference engine code inside


@pytest.mark.skipif(not REFERENCE, reason="GPULSM_REFERENCE does not name a reference checkout")
def test_adapter_compiles_against_the_shim(tmp_path):
    """nvcc -c of FliX/impl_gpulsmopt.cuh with its GPULSMOpt include redirected to
    gpulsmopt_b200.cuh (the maintainer's one-line edit, made in a temporary copy)."""
    src = open(os.path.join(REFERENCE, "FliX", "impl_gpulsmopt.cuh")).read()
    edited = src.replace('#include "../GPULSMOpt.cuh"', '#include "gpulsmopt_b200.cuh"')
    assert edited != src
    (tmp_path / "FliX").mkdir()
    (tmp_path / "FliX" / "impl_gpulsmopt.cuh").write_text(edited)
    os.symlink(os.path.join(REFERENCE, "gpu_dictionary_adapter.cuh"), tmp_path / "gpu_dictionary_adapter.cuh")
    out = tmp_path / "adapter.o"
    r = subprocess.run(["nvcc", "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                        "arch=compute_100a,code=sm_100a", f"-I{tmp_path / 'FliX'}",
                        f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(REFERENCE, 'FliX')}",
                        f"-I{REFERENCE}", f"-I{os.path.join(REFERENCE, 'FliX', 'nvtx_stub')}", "-c",
                        os.path.join(ROOT, "oracle", "flix_adapter_shim.cu"), "-o", str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
