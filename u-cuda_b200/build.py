"""Build of the engine library (libucb.so) for sm_100a.

Steps:
  1. embed csrc/kernels/*.cuh (device sources compiled at run time by NVRTC) into a
     generated C++ file;
  2. compile csrc/*.cpp and csrc/*.cu with nvcc (-gencode arch=compute_100a,code=sm_100a)
     into ucb/libucb.so, linked against NVRTC; the CUDA driver is loaded at run time.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
GEN = CSRC / "_gen"
OUT = PKG / "ucb" / "libucb.so"
INCLUDE = PKG.parent / "include"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
DELIM = "UCBSRC"


def cutlass_include() -> Path:
    """CUTLASS / CuTe header tree (the sm100 UMMA and TMEM atoms of the MLP GEMM):
    $UCB_CUTLASS_INCLUDE, else the copy vendored with the flashinfer package."""
    env = os.environ.get("UCB_CUTLASS_INCLUDE")
    if env:
        return Path(env)
    import sysconfig
    cand = Path(sysconfig.get_paths()["purelib"]) / "flashinfer" / "data" / "cutlass" / "include"
    if not (cand / "cute" / "tensor.hpp").exists():
        raise RuntimeError(f"CUTLASS headers not found at {cand}; set UCB_CUTLASS_INCLUDE")
    return cand


def embed_headers() -> Path:
    GEN.mkdir(parents=True, exist_ok=True)
    heads = sorted((CSRC / "kernels").glob("*.cuh"))
    lines = ['#include <string>', '#include <utility>', '#include <vector>', 'namespace ucb {',
             'const std::vector<std::pair<std::string, std::string>>& device_headers() {',
             '    static const std::vector<std::pair<std::string, std::string>> h = {']
    for p in heads:
        text = p.read_text()
        if f"){DELIM}\"" in text:
            raise RuntimeError(f"delimiter collision in {p}")
        lines.append(f'        {{"{p.name}", R"{DELIM}({text}){DELIM}"}},')
    lines += ['    };', '    return h;', '}', '}  // namespace ucb', '']
    out = GEN / "embedded_headers.cpp"
    new = "\n".join(lines)
    if not out.exists() or out.read_text() != new:
        out.write_text(new)
    return out


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cu")) + [embed_headers()]


def needs_build(srcs) -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = list(srcs) + list((CSRC / "kernels").glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = True) -> Path:
    srcs = sources()
    if not force and not needs_build(srcs):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = str(CUDA / "bin" / "nvcc")
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-lineinfo",
              "-gencode", "arch=compute_100a,code=sm_100a",
              f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA / 'include'}"]
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.name + ".o")
        objs.append(o)
        if not force and o.exists() and o.stat().st_mtime > max(
                [s.stat().st_mtime] + [p.stat().st_mtime for p in CSRC.glob("*.h")] +
                [p.stat().st_mtime for p in INCLUDE.glob("*.h")]):
            continue
        cmd = [nvcc] + common + ["-c", str(s), "-o", str(o)]
        if s.suffix == ".cu":
            cmd += [f"-I{cutlass_include()}", "--expt-relaxed-constexpr"]
            cmd += ["-Xptxas", "-v"] if os.environ.get("UCB_PTXAS_VERBOSE") else []
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"--- {s.name}\n{out.decode()}\n")
        elif verbose and out.strip():
            sys.stderr.write(out.decode())
    if failed:
        raise RuntimeError("nvcc compilation failed")
    link = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(OUT)] + \
        [str(o) for o in objs] + [f"-L{CUDA / 'lib64'}", "-lnvrtc", "-ldl", "-lpthread",
                                  "-Xlinker", f"-rpath,{CUDA / 'lib64'}"]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(OUT)
