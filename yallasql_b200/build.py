"""Build the in-tree shared libraries for sm_100a.

``libyq_ops.so``    CUDA kernels + the C ABI declared in ``include/yq_ops.h``.
``libyq_engine.so`` C++ operator layer (Batch / CacheManager / operators)
                    declared in ``include/yq_engine.h``, linked against
                    libyq_ops.so.

Objects are compiled in parallel and only when a source or header changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
ENGINE = os.path.join(PKG, "engine")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
              "-I", INCLUDE, "-diag-suppress", "177"]
OPS_LIB = os.path.join(PKG, "libyq_ops.so")
ENGINE_LIB = os.path.join(PKG, "libyq_engine.so")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers(d: str) -> list[str]:
    out = []
    for base in (d, INCLUDE):
        for f in os.listdir(base):
            if f.endswith((".cuh", ".h", ".hpp")):
                out.append(os.path.join(base, f))
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout)


_INCLUDE_RE = None


def _includes(path: str, seen: set[str]) -> set[str]:
    """Local headers `path` includes, transitively (quoted #include lines)."""
    global _INCLUDE_RE
    import re
    if _INCLUDE_RE is None:
        _INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)
    try:
        with open(path) as f:
            text = f.read()
    except OSError:
        return seen
    for name in _INCLUDE_RE.findall(text):
        dep = os.path.normpath(os.path.join(os.path.dirname(path), name))
        if dep not in seen and os.path.exists(dep):
            seen.add(dep)
            _includes(dep, seen)
    return seen


def _compile_all(srcs: list[str], extra: list[str], headers: list[str]) -> list[str]:
    os.makedirs(BUILD, exist_ok=True)
    objs, jobs = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        deps = sorted(_includes(s, set())) if s.endswith((".cu", ".cpp")) else headers
        if _stale(o, [s] + deps):
            jobs.append([nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    return objs


# Device headers the runtime-compiled kernels include (jit.cu), by the name
# each is #included under.
JIT_HEADERS = [("row_kernels.cuh", os.path.join(CSRC, "row_kernels.cuh")),
               ("yq_agg.cuh", os.path.join(CSRC, "yq_agg.cuh")),
               ("yq_hash.cuh", os.path.join(CSRC, "yq_hash.cuh")),
               ("yq_lookback.cuh", os.path.join(CSRC, "yq_lookback.cuh")),
               ("yq_stage.cuh", os.path.join(CSRC, "yq_stage.cuh")),
               ("yq_vm.cuh", os.path.join(CSRC, "yq_vm.cuh")),
               ("yq_common.cuh", os.path.join(CSRC, "yq_common.cuh")),
               ("../../include/yq_ops.h", os.path.join(INCLUDE, "yq_ops.h"))]


def _jit_headers_source() -> str:
    """A C++ file holding the JIT device headers as string literals."""
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "jit_headers.gen.cpp")
    if not _stale(out, [p for _, p in JIT_HEADERS] + [os.path.abspath(__file__)]):
        return out
    parts = ["// Generated by yallasql_b200/build.py: device headers for runtime compilation.\n"]
    names, texts = [], []
    for i, (name, path) in enumerate(JIT_HEADERS):
        with open(path) as f:
            text = f.read()
        if ")YQJIT\"" in text:
            raise RuntimeError(f"{path} contains the raw-string delimiter")
        parts.append(f'static const char h{i}[] = R"YQJIT({text})YQJIT";\n')
        names.append(f'"{name}"')
        texts.append(f"h{i}")
    parts.append(f"extern const int yq_jit_header_count = {len(JIT_HEADERS)};\n")
    parts.append("extern const char* const yq_jit_header_names[] = {" + ", ".join(names) + "};\n")
    parts.append("extern const char* const yq_jit_header_texts[] = {" + ", ".join(texts) + "};\n")
    with open(out, "w") as f:
        f.write("".join(parts))
    return out


def build_ops(verbose: bool = False) -> str:
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    srcs.append(_jit_headers_source())
    headers = _headers(CSRC)
    objs = _compile_all(srcs, [], headers)
    if _stale(OPS_LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", OPS_LIB] + objs + ["-ldl"])
        if verbose:
            print("built", OPS_LIB)
    return OPS_LIB


def build_engine(verbose: bool = False) -> str:
    if not os.path.isdir(ENGINE):
        return ""
    srcs = sorted(os.path.join(ENGINE, f) for f in os.listdir(ENGINE) if f.endswith((".cpp", ".cu")))
    if not srcs:
        return ""
    headers = _headers(ENGINE)
    objs = _compile_all(srcs, [], headers)
    if _stale(ENGINE_LIB, objs + [OPS_LIB]):
        _run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", ENGINE_LIB] + objs +
             ["-L", PKG, "-lyq_ops", "-Xlinker", "-rpath,$ORIGIN"])
        if verbose:
            print("built", ENGINE_LIB)
    return ENGINE_LIB


def build(verbose: bool = False) -> None:
    build_ops(verbose)
    build_engine(verbose)


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
