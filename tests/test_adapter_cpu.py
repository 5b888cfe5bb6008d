"""The reference's kernel-layer templates compile against yq_forward.cu.

yallasql_b200/adapter/yq_forward.cu defines YallaSQL::Kernel::launch_* with
the reference's own signatures (include/kernels/comparison_operators_kernel.hpp:8,
prefix_sum.hpp:26-29, radix_sort_kernel.hpp:23, :83-89) by forwarding to
libyq_ops.so. This compiles it against the reference's headers (with the
stand-ins for its logger and DuckDB types in oracle/ref_stubs) and checks that
every instantiation the reference's own src/kernels/*.cu provide for those
entry points is defined, so the reference's operators link against it.
Skipped where the reference sources are absent.
"""
import os
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "yallasql_b200", "adapter", "yq_forward.cu")

EXPECTED = (
    [f"launch_conditional_operators<{t}, YallaSQL::Kernel::{op}<{t}> >"
     for t in ("int", "float", "long", "YallaSQL::Kernel::String")
     for op in ("LEOperator", "GEOperator", "LEQOperator", "GEQOperator", "EQOperator", "NEQOperator")]
    + ["launch_conditional_operators<bool, YallaSQL::Kernel::ANDOperator>",
       "launch_conditional_operators<bool, YallaSQL::Kernel::OROperator>",
       "launch_prefix_sum_mask(bool*, unsigned int*, unsigned int, CUstream_st*&)",
       "launch_prefix_sum<unsigned int>",
       "launch_radix_sort<YallaSQL::Kernel::AscOp<unsigned int>, unsigned int, 256ul>",
       "launch_radix_sort<YallaSQL::Kernel::AscOp<unsigned long>, unsigned long, 256ul>",
       "launch_radix_sort<YallaSQL::Kernel::AscOpString, YallaSQL::Kernel::String",
       "launch_radix_sort<YallaSQL::Kernel::DescOp<unsigned int>, unsigned int, 256ul>",
       "launch_radix_sort<YallaSQL::Kernel::DescOp<unsigned long>, unsigned long, 256ul>",
       "launch_radix_sort<YallaSQL::Kernel::DescOpString, YallaSQL::Kernel::String",
       "launch_int_to_uint32(int*, unsigned int*, int)",
       "launch_uint32_to_int(unsigned int*, int*, int)",
       "launch_float_to_uint32(float*, unsigned int*, int)",
       "launch_uint32_to_float(unsigned int*, float*, int)"])


def _ref_or_skip():
    ref = oracle.reference_sources()
    if not ref:
        pytest.skip("reference sources not present (set YQ_REFERENCE_SOURCES)")
    return ref


def test_forwarding_file_compiles_against_reference_headers(tmp_path):
    ref = _ref_or_skip()
    obj = tmp_path / "yq_forward.o"
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    cmd = [nvcc, "-std=c++20", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-w",
           "-I", os.path.join(ROOT, "oracle", "ref_stubs"), "-I", os.path.join(ref, "include"),
           "-I", os.path.join(ROOT, "include"), "-c", ADAPTER, "-o", str(obj)]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout
    syms = subprocess.run(["nm", "-C", "--defined-only", str(obj)], stdout=subprocess.PIPE, text=True,
                          check=True).stdout
    defined = [ln for ln in syms.splitlines() if " T " in ln or " W " in ln]
    text = "\n".join(defined)
    missing = [e for e in EXPECTED if e not in text]
    assert not missing, missing


def test_forwarding_library_exports_the_test_entry_points():
    """oracle/_ref/libyq_forward.so (built by `make -C oracle ref`) loads and
    exports the harness the GPU tests call (no device work here)."""
    path = os.path.join(ROOT, "oracle", "_ref", "libyq_forward.so")
    if not os.path.exists(path):
        _ref_or_skip()
        pytest.skip("libyq_forward.so not built")
    import ctypes
    lib = ctypes.CDLL(path)
    for name in ("fwd_compare_i32", "fwd_compare_f32", "fwd_compare_i64", "fwd_compare_str", "fwd_logic",
                 "fwd_prefix_sum_mask", "fwd_prefix_sum_u32", "fwd_radix_sort_u32", "fwd_radix_sort_u64",
                 "fwd_radix_sort_str", "fwd_float_to_uint32", "fwd_int_to_uint32"):
        assert hasattr(lib, name), name
