"""Builds oracle/_ref/libctref.so: the reference's own census-transform and
cross-check kernel bodies, compiled for the host CPU (test infrastructure:
it pins the oracle's restatement of those rows to the reference's code).

The reference cannot be built as a library here (its include chains need the
missing CluTec.Core headers and the OpenGL interop header), so this recipe
takes the kernel namespaces themselves from the reference sources, in place,
at build time:

  CluTec.Cuda.ImgProc/CensusTransform.cu          namespace Kernel (Const, Transform)
  CluTec.Cuda.MultiView/CrossCheckDisparityMaps.h  namespace CrossCheckDisparityMaps
                                                   minus class CDriver
  CluTec.Cuda.MultiView/CrossCheckDisparityMaps.cu namespace Kernel (Const, c_xPars, Transform)
  CluTec.Cuda.MultiView/DisparityId.h              included unchanged
  CluTec.Cuda.ImgProc/Kernel.Algo.ArraySum_W32H16.h template struct AlgoArraySum_W32H16

and compiles them, in one translation unit fed to g++ on standard input,
against refshim.h (host stand-ins for the CUDA built-ins and the missing
CluTec types) and harness.inc (the extern "C" entry points). Nothing taken
from the reference is written to disk; the only output is the shared
library. Usage: python oracle/ref/build_ref.py [reference root]
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE.parent / "_ref"
OUT = OUT_DIR / "libctref.so"
DEFAULT_REF = Path("/root/reference")


def _skip_to_code(text: str, i: int) -> int:
    """Index of the end of a comment or literal starting at i, or i."""
    if text.startswith("//", i):
        j = text.find("\n", i)
        return len(text) if j < 0 else j
    if text.startswith("/*", i):
        j = text.find("*/", i + 2)
        return len(text) if j < 0 else j + 2
    if text[i] in "\"'":
        q, j = text[i], i + 1
        while j < len(text) and text[j] != q:
            j += 2 if text[j] == "\\" else 1
        return j + 1
    return i


def block(text: str, head: str, start: int = 0) -> tuple[int, int]:
    """(begin, end) of the first `head ... { ... }` at or after start, from
    the head to the matching closing brace (comments and literals skipped)."""
    b = text.find(head, start)
    if b < 0:
        raise ValueError(f"'{head}' not found")
    i, depth = text.index("{", b), 0
    while i < len(text):
        j = _skip_to_code(text, i)
        if j != i:
            i = j
            continue
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return b, i + 1
        i += 1
    raise ValueError(f"unbalanced braces after '{head}'")


def namespace_body(text: str, name: str) -> str:
    b, e = block(text, f"namespace {name}")
    inner = text[b:e]
    return inner[inner.index("{") + 1:-1]


def translation_unit(ref: Path) -> str:
    ct = (ref / "CluTec.Cuda.ImgProc/CensusTransform.cu").read_text(errors="replace")
    cch = (ref / "CluTec.Cuda.MultiView/CrossCheckDisparityMaps.h").read_text(errors="replace")
    ccu = (ref / "CluTec.Cuda.MultiView/CrossCheckDisparityMaps.cu").read_text(errors="replace")
    b, e = block(ct, "namespace Kernel")
    census_kernel = ct[b:e]
    hdr = namespace_body(cch, "CrossCheckDisparityMaps")
    cb, ce = block(hdr, "class CDriver")
    hdr = hdr[:cb] + hdr[ce:].lstrip().removeprefix(";")
    b, e = block(ccu, "namespace Kernel")
    cc_kernel = ccu[b:e]
    asum = (ref / "CluTec.Cuda.ImgProc/Kernel.Algo.ArraySum_W32H16.h").read_text(errors="replace")
    sb, se = block(asum, "struct AlgoArraySum_W32H16")
    tb = asum.rfind("template", 0, sb)  # the struct's template head
    array_sum = asum[tb:se] + ";"
    return "\n".join([
        '#include "refshim.h"',
        '#include "DisparityId.h"',
        "namespace Clu { namespace Cuda { namespace CensusTransform {",
        census_kernel,
        "}}}",
        "namespace Clu { namespace Cuda { namespace CrossCheckDisparityMaps {",
        hdr,
        cc_kernel,
        "}}}",
        "namespace Clu { namespace Cuda { namespace Kernel {",
        array_sum,
        "}}}",
        '#include "harness.inc"',
        "",
    ])


def build(ref: Path = DEFAULT_REF) -> Path:
    if not (ref / "CluTec.Cuda.ImgProc/CensusTransform.cu").exists():
        raise FileNotFoundError(f"reference sources not found under {ref}")
    OUT_DIR.mkdir(exist_ok=True)
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [cxx, "-std=c++20", "-pthread", "-O1", "-fPIC", "-shared", "-w", "-x", "c++",
           "-I", str(HERE), "-I", str(ref / "CluTec.Cuda.MultiView"), "-o", str(OUT), "-"]
    r = subprocess.run(cmd, input=translation_unit(ref), text=True, capture_output=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed:\n{r.stderr[-4000:]}")
    return OUT


if __name__ == "__main__":
    print(build(Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_REF))
