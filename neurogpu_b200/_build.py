"""In-tree build of libngpu.so (CUDA for sm_100a) with nvcc.

The shared library is written next to this file so that it travels with the
repository snapshot; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libngpu.so"
INCLUDE = HERE.parent / "include"

# kernel headers the runtime specialisation (ngpu_jit.h) compiles with NVRTC,
# embedded in the library as text
JIT_HEADERS = ["ngpu_math.cuh", "param_fold.cuh", "node_classes.cuh", "channels_ttpc.cuh", "channels_mainen.cuh", "sim_kernels.cuh"]
JIT_INC = CSRC / "jit_sources.inc"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: libngpu.so cannot be built")


def _sources() -> list[Path]:
    return (sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) +
            [INCLUDE / "ngpu.h"])


def write_jit_sources(chunk: int = 8000) -> Path:
    """csrc/jit_sources.inc: the JIT_HEADERS as C++ raw-string chunks."""
    delim = "NGPUJITSRC"
    out = ["// Generated by neurogpu_b200/_build.py from the kernel headers; do not edit.",
           "namespace ngpu_jit {", "struct JitFile {", "    const char* name;", "    int n_chunks;",
           "    const char* const* chunks;", "};"]
    for k, name in enumerate(JIT_HEADERS):
        text = (CSRC / name).read_text()
        if f"){delim}" in text:
            raise RuntimeError(f"{name} contains the raw-string delimiter")
        parts, cur = [], ""
        for line in text.splitlines(keepends=True):
            if len(cur) + len(line) > chunk and cur:
                parts.append(cur)
                cur = ""
            cur += line
        parts.append(cur)
        out.append(f"static const char* const kJitChunks{k}[] = {{")
        out += [f'    R"{delim}({p}){delim}",' for p in parts]
        out.append("};")
    out.append("static const JitFile kJitFiles[] = {")
    for k, name in enumerate(JIT_HEADERS):
        out.append(f'    {{"{name}", (int)(sizeof(kJitChunks{k}) / sizeof(kJitChunks{k}[0])), kJitChunks{k}}},')
    out.append("};")
    out.append(f"static const int kJitFileCount = {len(JIT_HEADERS)};")
    out.append("}  // namespace ngpu_jit")
    text = "\n".join(out) + "\n"
    if not JIT_INC.exists() or JIT_INC.read_text() != text:
        JIT_INC.write_text(text)
    return JIT_INC


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _sources() if p.exists())


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile csrc/ngpu.cu into libngpu.so (no-op when up to date)."""
    if not force and not needs_build():
        return LIB
    write_jit_sources()
    cmd = [_nvcc(), *NVCC_FLAGS, *(extra_flags or []), str(CSRC / "ngpu.cu"), "-o", str(LIB), "-ldl"]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
    print(LIB)
