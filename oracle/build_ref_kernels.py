"""Builds the reference's own integrator kernels, unchanged, for the GPU parity pin.

TEST INFRASTRUCTURE (part of the oracle): the product never loads what this writes.

What it does, for each case in CASES:
  1. reads the reference's NVRTC template (kernels/lle2d.template.cu, ls2d.template.cu,
     bifurcation1d.template.cu) and its four headers (cudaLibrary.cu, cudaLibrary.cuh,
     cudaMacros.cuh, configCUDA.h) where they lie in the reference tree;
  2. substitutes {{AMOUNT_OF_X}}, {{KRS_BODY}} and {{PAR_OR_VAR}} by plain string
     replacement, as `replace_all` does (U-CUDA/parametric_engine.cpp:554-562, used by
     compile_if_needed :1549-1551 and compile_lle_2d_if_needed :2496-2498);
  3. compiles with NVRTC, the headers passed as virtual header sources under their own
     names and the reference's options (parametric_engine.cpp:1581-1604:
     --gpu-architecture, --std=c++17, -default-device, -I<CUDA include>), registering
     the kernel names as name expressions and recording their lowered names
     (:1574-1575, :1619-1620, :2520, :2553).

Two builds per case:
  * "stock"  -- the reference's options as they are (FMA contraction on, NVRTC's default);
  * "nofma"  -- the same plus --fmad=false, which makes every floating-point operation of
               the kernel round once, as the oracle's restatement (g++ -ffp-contract=off)
               and the engine's exact form do, so the three can be compared bit for bit.
The one deliberate difference from the reference's pipeline: it asks NVRTC for PTX of
compute_<cc> and lets the driver JIT it at load time (cuModuleLoadDataEx, :1631); this
recipe asks NVRTC for a CUBIN of sm_100 directly (the same front end and the same ptxas
optimisation level), because the GPU machine that runs the tests has no reference tree.

The KRS bodies are the reference codegen's own output for each system, taken from the
golden fixture tests/golden/codegen_cases.json (itself generated by the reference's
sysparse.cpp + codegen.cpp, see tests/golden/make_golden.py).

Usage:
    python oracle/build_ref_kernels.py <reference U-CUDA directory> [out dir]
Out dir defaults to oracle/_ref. Writes refk_<case>_<variant>.cubin and refk_manifest.json.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

# (case name, template file, golden codegen case, amountOfX, par_or_var, kernel names)
CASES = [
    ("lle2d_rossler_pov1", "lle2d.template.cu", "rossler_config", 3, 1, ["LLEKernelCUDA"]),
    ("lle2d_lorenz_pov0", "lle2d.template.cu", "library_Lorenz", 3, 0, ["LLEKernelCUDA"]),
    ("lle2d_rossler_pov2", "lle2d.template.cu", "rossler_config", 3, 2, ["LLEKernelCUDA"]),
    ("ls2d_hyper_rossler_pov1", "ls2d.template.cu", "hyper_rossler_swept", 4, 1, ["LSKernelCUDA"]),
    ("ls2d_lorenz_pov1", "ls2d.template.cu", "library_Lorenz", 3, 1, ["LSKernelCUDA"]),
    ("bif1d_lorenz_pov1", "bifurcation1d.template.cu", "library_Lorenz", 3, 1,
     ["calculateDiscreteModelCUDA", "peakFinderCUDA"]),
    ("bif1d_rossler_pov0", "bifurcation1d.template.cu", "rossler_config", 3, 0,
     ["calculateDiscreteModelCUDA", "peakFinderCUDA"]),
]
VARIANTS = {"stock": [], "nofma": ["--fmad=false"]}
HEADERS = ["cudaLibrary.cu", "cudaLibrary.cuh", "cudaMacros.cuh", "configCUDA.h"]


def _nvrtc():
    lib = C.CDLL(str(CUDA / "lib64" / "libnvrtc.so"))
    lib.nvrtcGetErrorString.restype = C.c_char_p
    return lib


def _read(p: Path) -> str:
    # the reference's sources are UTF-8 with a byte-order mark; NVRTC gets them as bytes
    return p.read_bytes().decode("utf-8-sig")


def _replace_all(s: str, old: str, new: str) -> str:
    return s.replace(old, new)


def compile_case(nv, src: str, headers: dict, names: list[str], extra: list[str]):
    prog = C.c_void_p()
    hsrc = (C.c_char_p * len(headers))(*[v.encode() for v in headers.values()])
    hnam = (C.c_char_p * len(headers))(*[k.encode() for k in headers.keys()])
    r = nv.nvrtcCreateProgram(C.byref(prog), src.encode(), b"bifurcation1d.cu", len(headers), hsrc, hnam)
    if r:
        raise RuntimeError(f"nvrtcCreateProgram: {nv.nvrtcGetErrorString(r).decode()}")
    for n in names:
        nv.nvrtcAddNameExpression(prog, n.encode())
    opts = ["--gpu-architecture=sm_100", "--std=c++17", "-default-device", f"-I{CUDA / 'include'}"] + extra
    copts = (C.c_char_p * len(opts))(*[o.encode() for o in opts])
    r = nv.nvrtcCompileProgram(prog, len(opts), copts)
    logsz = C.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, C.byref(logsz))
    log = C.create_string_buffer(max(logsz.value, 1))
    nv.nvrtcGetProgramLog(prog, log)
    if r:
        raise RuntimeError(f"NVRTC compile failed:\n{log.value.decode(errors='replace')}")
    lowered = {}
    for n in names:
        p = C.c_char_p()
        nv.nvrtcGetLoweredName(prog, n.encode(), C.byref(p))
        lowered[n] = p.value.decode() if p.value else n
    sz = C.c_size_t()
    nv.nvrtcGetCUBINSize(prog, C.byref(sz))
    buf = C.create_string_buffer(sz.value)
    nv.nvrtcGetCUBIN(prog, buf)
    nv.nvrtcDestroyProgram(C.byref(prog))
    return buf.raw[:sz.value], lowered


def build(ref_dir: Path, out_dir: Path, force: bool = False) -> Path:
    tdir = ref_dir / "kernels"
    if not (tdir / "lle2d.template.cu").exists():
        raise FileNotFoundError(f"no reference kernel templates under {tdir}")
    headers = {h: _read(ref_dir / h) for h in HEADERS}
    golden = {c["name"]: c for c in json.loads((ROOT / "tests" / "golden" / "codegen_cases.json")
                                               .read_text())["cases"]}
    jobs = []
    key = hashlib.sha256("".join(headers.values()).encode())
    key.update(json.dumps([CASES, VARIANTS]).encode())
    for name, tmpl, gcase, nx, pov, kernels in CASES:
        body = golden[gcase]["schemes"]["RK4"]
        src = _read(tdir / tmpl)
        src = _replace_all(src, "{{AMOUNT_OF_X}}", str(nx))
        src = _replace_all(src, "{{KRS_BODY}}", body)
        src = _replace_all(src, "{{PAR_OR_VAR}}", str(pov))
        key.update(src.encode())
        jobs.append((name, tmpl, gcase, nx, pov, kernels, body, src))
    key = key.hexdigest()
    mpath = out_dir / "refk_manifest.json"
    if not force and mpath.exists():
        old = json.loads(mpath.read_text())
        if old.get("key") == key and all((out_dir / v["cubin"]).exists()
                                         for c in old["cases"].values() for v in c["variants"].values()):
            return mpath
    out_dir.mkdir(parents=True, exist_ok=True)
    nv = _nvrtc()

    def one(job, var):
        name, tmpl, gcase, nx, pov, kernels, body, src = job
        cubin, lowered = compile_case(nv, src, headers, kernels, VARIANTS[var])
        fn = f"refk_{name}_{var}.cubin"
        (out_dir / fn).write_bytes(cubin)
        return name, var, {"cubin": fn, "options_extra": VARIANTS[var], "kernels": lowered}

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        done = list(ex.map(lambda jv: one(*jv), [(j, v) for j in jobs for v in VARIANTS]))
    manifest = {"generator": "oracle/build_ref_kernels.py", "arch": "sm_100", "key": key, "cases": {}}
    for name, tmpl, gcase, nx, pov, kernels, body, src in jobs:
        manifest["cases"][name] = {"template": tmpl, "system": gcase, "amountOfX": nx, "par_or_var": pov,
                                   "body_sha256": hashlib.sha256(body.encode()).hexdigest(), "variants": {}}
    for name, var, entry in done:
        manifest["cases"][name]["variants"][var] = entry
    mpath.write_text(json.dumps(manifest, indent=1))
    print(f"built {len(done)} reference kernel modules into {out_dir}")
    return mpath


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(__doc__)
    ref = Path(sys.argv[1])
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else HERE / "_ref"
    print(build(ref, out))
