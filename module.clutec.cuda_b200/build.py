"""Builds libctstereo.so in place for sm_100a with nvcc.

Every .cu / .cpp file under csrc/ is compiled to an object file in
_build/ (in parallel) and linked into module.clutec.cuda_b200/libctstereo.so,
which is what ctstereo.py loads. The seeded stereo-pair generator (gen/) is a
separate host-only library, libctsynth.so, built with g++.
Run: python module.clutec.cuda_b200/build.py
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libctstereo.so"
SYNTH_SRC = PKG / "gen" / "synth.cpp"
SYNTH_LIB = PKG / "libctsynth.so"
INCLUDE = PKG.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-I", str(INCLUDE), "-I", str(CSRC),
          "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr"]


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _deps_digest(src: Path) -> str:
    h = hashlib.sha1()
    h.update(src.read_bytes())
    for hdr in sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))):
        h.update(hdr.read_bytes())
    h.update(" ".join(ARCH + COMMON).encode())
    return h.hexdigest()


def _compile(src: Path, verbose_ptxas: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    stamp = BUILD / (src.name + ".sha1")
    digest = _deps_digest(src)
    if obj.exists() and stamp.exists() and stamp.read_text() == digest and not verbose_ptxas:
        return obj
    cmd = [NVCC] + ARCH + COMMON + ["-c", str(src), "-o", str(obj)]
    if verbose_ptxas and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas and r.stderr:
        sys.stderr.write(r.stderr)
    stamp.write_text(digest)
    return obj


def build_synth() -> Path:
    """libctsynth.so (the generator) from gen/synth.cpp, rebuilt when older
    than its sources."""
    deps = [SYNTH_SRC, INCLUDE / "ctsynth.h", INCLUDE / "ctstereo.h"]
    if SYNTH_LIB.exists() and SYNTH_LIB.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return SYNTH_LIB
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    tmp = SYNTH_LIB.with_suffix(".so.tmp")
    r = subprocess.run([cxx, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-I", str(INCLUDE),
                        str(SYNTH_SRC), "-o", str(tmp)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {SYNTH_SRC.name}:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, SYNTH_LIB)
    return SYNTH_LIB


def build(verbose_ptxas: bool = False) -> Path:
    build_synth()
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + [
        "-Xcompiler", "-fopenmp", "-lgomp", "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
