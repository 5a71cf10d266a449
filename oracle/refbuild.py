"""Builds the reference's own force arithmetic for the host, as a checker of the oracle.

TEST INFRASTRUCTURE ONLY (like the rest of oracle/): nothing in the product loads it.

The reference (TauferLab/fen-zi) is one CUDA translation unit that does not compile
with CUDA 12 (legacy texture references), but its force terms are plain per-atom
kernels: one thread per atom, no shared memory or barriers on the paths compiled
here.  This recipe takes, unmodified, the functions below from the reference
sources where they lie, and compiles them as host C++ against a shim
(oracle/ref_shim.h) that supplies the CUDA vector types, the texture fetches as
plain array reads and the device constants as globals:

  src/cucomplexops.cu                  float3/float4 operators (whole file)
  src/globals.h                        struct dihedralParameter
  src/bonded_forces.cu:22-51           bondInteraction
  src/bonded_forces.cu:57-118          angleInteraction
  src/bonded_forces.cu:124-221         improperInteraction
  src/bonded_forces.cu:226-386         torsionInteraction
  src/bonded_forces.cu:389-...         torsionInteraction_c36
  src/bonded_forces.cu:597-1381        bondedforce (bonds, Ewald exclusion, angles,
                                       Urey-Bradley, dihedrals + 1-4, impropers)
  src/bonded_forces.cu:1384-...        bondedforce_c36
  src/mdcuda.cu:519-553                ewaldCorrection
  src/nonbonded_forces.cu:25-245       nonbondforce (the USE_NEW_NONBOND kernel)
  src/cell_based_kernels.cu:1769-1826  BCMultiply (PME influence function)
  src/cell_based_kernels.cu:1829-1947  InitDeviceConstants (B-spline moduli, Gaussian)

Two builds come out of the same text:
  oracle/_ref/libfzref32.so  the reference's FP32 arithmetic (host libm in place of
                             the GPU's intrinsics);
  oracle/_ref/libfzref64.so  the same statements in FP64 (`float` mapped to double and
                             the `f` suffix of floating literals dropped while
                             extracting), so the reference's formulas can be compared
                             with the FP64 oracle to rounding level.
The extracted text and the libraries are written only to oracle/_ref/ (git-ignored),
together with a copy of the reference's complete example deck
tests/examples_fenzi/dmpc_small for the GPU tests (it is input data of the reference,
not committed here).

Usage: python oracle/refbuild.py [reference_root]   (default $FENZI_REFERENCE or
/root/reference).  Without the reference tree it does nothing and says so.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC_OUT = os.path.join(OUT, "src")
CXX = "/usr/bin/g++"

# (file, kind, name): kind "func" = first definition of a function/kernel by name
PIECES = [
    ("globals.h", "struct", "dihedralParameter"),
    ("mdcuda.cu", "func", "ewaldCorrection"),
    ("bonded_forces.cu", "func", "bondInteraction"),
    ("bonded_forces.cu", "func", "angleInteraction"),
    ("bonded_forces.cu", "func", "improperInteraction"),
    ("bonded_forces.cu", "func", "torsionInteraction"),
    ("bonded_forces.cu", "func", "torsionInteraction_c36"),
    ("bonded_forces.cu", "func", "bondedforce"),
    ("bonded_forces.cu", "func", "bondedforce_c36"),
    ("nonbonded_forces.cu", "func", "nonbondforce"),
    ("cell_based_kernels.cu", "func", "BCMultiply"),
    ("cell_based_kernels.cu", "func", "InitDeviceConstants"),
]
# improperInteraction sits inside #ifdef IMPROPER in the source; the extracted
# feature switches below define it.
# The reference's own macro definitions the pieces use (src/defs.in.h:52-68, 87-93,
# 116-128, 157, 163-164, 172-175, 181-190); DIHED_SHAREDMEM (src/defs.in.h:132) is left out:
# it only stages the same dihedral parameter table in shared memory.
DEFINES = ["__my_fadd", "__my_fmul", "__my_fdiv", "__my_fsin", "__my_fcos", "__my_fasin", "__my_facos",
           "__my_fsqrt", "__my_frsqrt", "__mycopysignf", "__my_add3", "__my_add4", "__my_mul3", "__my_mul4",
           "TWO_OVER_SQRT_PI", "CCTWO_OVER_SQRT_PI", "NBPART", "BPART", "NBXMOD", "VSWITCH", "PME_CALC",
           "UREY_BRADLEY", "IMPROPER", "CC", "MAXDPRM", "MAX_DIHED_TYPE", "COMPUTE_GLOBAL_THREADID",
           "PI", "NUM_SPLINE_SAMPLES", "MAXFFT_X", "MAXFFT_Y", "MAXFFT_Z", "M2", "M3", "M4"]


def _code_mask(text: str) -> list[bool]:
    """True for characters outside comments and string/char literals."""
    mask = [True] * len(text)
    i, n = 0, len(text)
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            j = text.find("\n", i)
            j = n if j < 0 else j
            for k in range(i, j):
                mask[k] = False
            i = j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            j = n if j < 0 else j + 2
            for k in range(i, j):
                mask[k] = False
            i = j
        elif c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            for k in range(i, min(j + 1, n)):
                mask[k] = False
            i = j + 1
        else:
            i += 1
    return mask


def _match_brace(text: str, mask: list[bool], open_at: int) -> int:
    depth = 0
    for k in range(open_at, len(text)):
        if not mask[k]:
            continue
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return k
    raise ValueError("unbalanced braces")


def extract_function(text: str, name: str) -> str:
    """The first definition of `name`: from the start of its declaration line to the
    closing brace of its body (preprocessor lines inside are kept)."""
    mask = _code_mask(text)
    for m in re.finditer(r"\b%s\s*\(" % re.escape(name), text):
        if not mask[m.start()]:
            continue
        # parameter list: match parentheses, skipping comments
        depth, k = 0, m.end() - 1
        while True:
            if mask[k]:
                if text[k] == "(":
                    depth += 1
                elif text[k] == ")":
                    depth -= 1
                    if depth == 0:
                        break
            k += 1
        j = k + 1
        while j < len(text) and (not mask[j] or text[j] in " \t\r\n"):
            j += 1
        if text[j] != "{":
            continue  # a call or a prototype, not the definition
        line_start = text.rfind("\n", 0, m.start()) + 1
        end = _match_brace(text, mask, j)
        return text[line_start:end + 1] + "\n"
    raise KeyError(name)


def extract_struct(text: str, name: str) -> str:
    mask = _code_mask(text)
    m = re.search(r"struct\s+%s\s*\{" % re.escape(name), text)
    end = _match_brace(text, mask, m.end() - 1)
    semi = text.index(";", end)
    return text[m.start():semi + 1] + "\n"


_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)[fF]\b")


def to_double(code: str) -> str:
    """Drops the `f` suffix of floating literals outside comments (FP64 build)."""
    mask = _code_mask(code)
    out, last = [], 0
    for m in _FLOAT_LIT.finditer(code):
        if not mask[m.start()]:
            continue
        # a bare integer with an f suffix is not a C literal; only decimal forms reach here
        out.append(code[last:m.start()])
        out.append(m.group(1))
        last = m.end()
    out.append(code[last:])
    return "".join(out)


def extract_defines(text: str, names) -> str:
    """The first `#define NAME ...` line of each name, with its continuation lines."""
    lines = text.splitlines(True)
    out = []
    for name in names:
        pat = re.compile(r"^\s*#\s*define\s+%s\b" % re.escape(name))
        for k, ln in enumerate(lines):
            if pat.match(ln) and "@" not in ln:
                block = [ln]
                while block[-1].rstrip().endswith("\\") and k + len(block) < len(lines):
                    block.append(lines[k + len(block)])
                out.append("".join(block))
                break
        else:
            raise KeyError(name)
    return "".join(out)


def strip_includes(code: str) -> str:
    return "".join(ln for ln in code.splitlines(True) if not ln.lstrip().startswith("#include"))


def build(ref_root: str) -> bool:
    src = os.path.join(ref_root, "src")
    if not os.path.isdir(src):
        print(f"refbuild: no reference tree at {ref_root}; skipped")
        return False
    os.makedirs(SRC_OUT, exist_ok=True)
    texts = {}
    parts = []
    defs = extract_defines(open(os.path.join(src, "defs.in.h")).read(), DEFINES)
    ops = strip_includes(open(os.path.join(src, "cucomplexops.cu")).read())
    parts.append(("cucomplexops.cu (whole)", ops))
    for fname, kind, name in PIECES:
        if fname not in texts:
            texts[fname] = open(os.path.join(src, fname)).read()
        t = texts[fname]
        code = extract_struct(t, name) if kind == "struct" else extract_function(t, name)
        parts.append((f"{fname}: {name}", code))
    for variant in ("32", "64"):
        with open(os.path.join(SRC_OUT, f"ref_defs{variant}.inc"), "w") as f:
            f.write("// generated by oracle/refbuild.py from src/defs.in.h; not committed\n")
            f.write(to_double(defs) if variant == "64" else defs)
        path = os.path.join(SRC_OUT, f"ref_pieces{variant}.inc")
        with open(path, "w") as f:
            f.write("// generated by oracle/refbuild.py from the reference sources; not committed\n")
            for label, code in parts:
                f.write(f"\n// ---- {label}\n")
                f.write(to_double(code) if variant == "64" else code)
        lib = os.path.join(OUT, f"libfzref{variant}.so")
        cmd = [CXX, "-O2", "-fPIC", "-shared", "-std=c++17", "-w", "-fno-fast-math", "-ffp-contract=off",
               f"-DFZREF_VARIANT={variant}", "-I", HERE, "-I", SRC_OUT,
               os.path.join(HERE, "ref_harness.cpp"), "-o", lib]
        subprocess.check_call(cmd)
    deck = os.path.join(ref_root, "tests", "examples_fenzi", "dmpc_small")
    if os.path.isdir(deck):
        dst = os.path.join(OUT, "dmpc_small")
        shutil.rmtree(dst, ignore_errors=True)
        shutil.copytree(deck, dst, ignore=shutil.ignore_patterns(".svn"))
    return True


def default_root() -> str:
    return os.environ.get("FENZI_REFERENCE", "/root/reference")


if __name__ == "__main__":
    ok = build(sys.argv[1] if len(sys.argv) > 1 else default_root())
    print("refbuild:", "built oracle/_ref" if ok else "nothing built")
