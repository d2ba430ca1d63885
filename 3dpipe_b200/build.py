"""Build recipe for the tdp library (in-tree, sm_100a only).

Compiles every CUDA source under csrc/ with nvcc for sm_100a and every C++ host
source under src/ with g++, links them into 3dpipe_b200/libtdp.so, and links the
`tdbase` command-line front end (src/join/tdbase_main.cpp) against it into
3dpipe_b200/bin/tdbase.  Rebuilds only what is out of date.

    python 3dpipe_b200/build.py [-j N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
OBJ = PKG / "_build"
LIB = PKG / "libtdp.so"
BIN = PKG / "bin" / "tdbase"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = shutil.which("g++") or "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(PKG / "src")]
# bounds_kernels.cu, prep_kernels.cu: no contraction of a*b+c into an FMA, so
# their values are those of the same expressions rounded one operation at a
# time (as on the host)
PER_FILE_FLAGS = {"bounds_kernels.cu": ["-fmad=false"], "prep_kernels.cu": ["-fmad=false"]}
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-function",
             "-I", str(ROOT / "include"), "-I", str(PKG / "src"),
             "-I", "/usr/local/cuda/include"]


def _sources():
    cu = sorted((PKG / "csrc").glob("*.cu"))
    cpp = sorted(p for p in (PKG / "src").rglob("*.cpp") if p.name != "tdbase_main.cpp")
    return cu, cpp


def _headers():
    hs = list((PKG / "csrc").glob("*.cuh")) + list((PKG / "src").rglob("*.h")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _obj_for(src: Path) -> Path:
    rel = src.relative_to(PKG).with_suffix(".o")
    return OBJ / str(rel).replace(os.sep, "__")


def _compile(src: Path, force: bool, hdr_time: float) -> Path:
    obj = _obj_for(src)
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
        return obj
    obj.parent.mkdir(parents=True, exist_ok=True)
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, *PER_FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
    else:
        cmd = [CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    cu, cpp = _sources()
    hdr_time = _headers()
    jobs = jobs or min(8, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr_time), cu + cpp))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        # link beside the library and rename over it, so a reader never sees a half-written file
        tmp = LIB.with_name(LIB.name + ".tmp")
        cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    main = PKG / "src" / "join" / "tdbase_main.cpp"
    if main.exists():
        BIN.parent.mkdir(parents=True, exist_ok=True)
        if force or not BIN.exists() or BIN.stat().st_mtime < max(LIB.stat().st_mtime, main.stat().st_mtime):
            cmd = [CXX, *CXX_FLAGS, str(main), "-o", str(BIN), "-L", str(PKG), "-ltdp",
                   f"-Wl,-rpath,$ORIGIN/..", "-lpthread"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


def build_oracle(with_reference: bool = True) -> None:
    """Build the FP64 oracle (test infrastructure) and, when the reference tree
    is present, the reference's own CPU code into oracle/_ref/."""
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    ref_env = os.environ.get("TDP_REFERENCE")
    if not ref_env:
        # the oracle recipe names the reference tree it reads by default
        r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "print-ref"], capture_output=True, text=True)
        ref_env = r.stdout.strip() if r.returncode == 0 else ""
    ref = Path(ref_env) if ref_env else Path("/nonexistent")
    if with_reference and (ref / "src" / "geometry" / "computing_cpu.cpp").exists():
        r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REF={ref}"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference build failed:\n{r.stdout}\n{r.stderr}")
        # the reference's own GPU join (a comparison baseline, never on a test
        # or product path): a failure here is reported, not fatal
        r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "refgpu", f"REF={ref}"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            print(f"note: the reference GPU join (oracle/_ref/tdbase_ref_gpu) did not build:\n{r.stderr[-2000:]}",
                  file=sys.stderr)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    a = ap.parse_args()
    build(force=a.force, jobs=a.j, verbose=True)
    if not a.no_oracle:
        build_oracle()
    sys.exit(0)
