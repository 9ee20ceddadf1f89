"""build_dropin.py -- TEST INFRASTRUCTURE ONLY.

Builds CPS with the B200 bridge linked in, as INTEGRATION.md tells a CPS
maintainer to: the bridge header and source given there, and CPS's own
lattice/f_dwf_base/f_dwf_base.C, lattice/f_mobius/f_mobius.C and
lattice/f_wilson/f_wilson.C with the USE_B200 branch blocks given there
inserted at the top of the functions each block names, compiled with
-DUSE_B200.  They are linked, ahead of the rest of CPS (oracle/_ref/libcps.a
from oracle/build_ref.sh), with the reference harness (oracle/ref_harness.C,
also compiled with -DUSE_B200) and cps_public_b200/libcpsb200.so into
oracle/_ref/cpsref_b200.  Running a harness request through that binary runs
CPS's own Lattice::FmatEvlInv / FmatEvlMInv / FmatInv, which then hand the
solve to the library.

Usage: python oracle/build_dropin.py [path-to-cps_pp]   (default $CPS_REFERENCE, else /root/reference/cps_pp)

Everything is written under oracle/_ref/ (git-ignored); the reference tree is
only read.  The patched copies of the three CPS files live in
oracle/_ref/b200/src/ and are never committed.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
B200 = os.path.join(OUT, "b200")
CXXFLAGS = ["-O2", "-fopenmp", "-DUSE_OMP", "-w", "-std=gnu++11", "-DUSE_B200"]

# CPS files that receive branches: path under src/util/lattice, and the class
# names whose member functions the blocks name
FILES = {
    "f_dwf_base/f_dwf_base.C": "FdwfBase",
    "f_mobius/f_mobius.C": "Fmobius",
    "f_wilson/f_wilson.C": "Fwilson",
}


def cpp_blocks(text: str) -> list[str]:
    return re.findall(r"```cpp\n(.*?)```", text, re.S)


def bridge_sources(blocks: list[str]) -> tuple[str, str]:
    hdr = [b for b in blocks if b.startswith("// include/util/b200_bridge.h")]
    src = [b for b in blocks if b.startswith("// util/dirac_op/b200_bridge.C")]
    if len(hdr) != 1 or len(src) != 1:
        raise SystemExit("INTEGRATION.md: expected one bridge header block and one bridge source block")
    return "#pragma once\n" + hdr[0], src[0]


def branch_blocks(blocks: list[str]) -> list[tuple[list[tuple[str, str, int]], str]]:
    """Blocks whose first line names the functions they open, e.g.
    '// FdwfBase::FmatEvlInv (f_dwf_base.C:189), Fwilson::FmatEvlInv (f_wilson.C:159)'
    followed by an #ifdef USE_B200 ... #endif body.  Returns
    [([(class, function, line), ...], body)]."""
    out = []
    for b in blocks:
        first, _, rest = b.partition("\n")
        if not rest.startswith("#ifdef USE_B200"):
            continue
        targets = [(c, f, int(ln)) for c, f, ln in re.findall(r"(\w+)::(\w+) \(\w+\.C:(\d+)\)", first)]
        if not targets:
            raise SystemExit(f"INTEGRATION.md: branch block names no function: {first}")
        out.append((targets, rest))
    return out


def find_body_open(text: str, cls: str, func: str, line: int) -> int:
    """Offset just past the '{' that opens the definition of cls::func that
    starts on `line` (1-based) of the unpatched file."""
    starts = [m for m in re.finditer(r"^int\s+%s::%s\s*\(" % (cls, func), text, re.M)]
    for m in starts:
        ln = text.count("\n", 0, m.start()) + 1
        if ln == line:
            brace = text.index("{", m.end())
            return brace + 1
    found = [text.count("\n", 0, m.start()) + 1 for m in starts]
    raise SystemExit(f"{cls}::{func} does not start on line {line} (definitions at {found})")


def patch(text: str, path: str, cls: str, branches) -> str:
    inserts = []
    for targets, body in branches:
        for c, f, ln in targets:
            if c == cls:
                inserts.append((find_body_open(text, c, f, ln), body, ln))
    if not inserts:
        raise SystemExit(f"no branch targets in {path}")
    # from the end, so earlier offsets stay valid; #line keeps CPS's own line
    # numbers for the code after each insertion
    for off, body, _ in sorted(inserts, reverse=True):
        resume = text.count("\n", 0, off) + 1
        text = text[:off] + "\n" + body + '#line %d "%s"\n' % (resume, path) + text[off:]
    inc = text.index("CPS_START_NAMESPACE")
    return text[:inc] + "#ifdef USE_B200\n#include <util/b200_bridge.h>\n#endif\n" + text[inc:]


def run(cmd: list[str]) -> None:
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise SystemExit(f"failed: {' '.join(cmd)}\n{p.stderr[-4000:]}")


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CPS_REFERENCE", "/root/reference/cps_pp")
    if not os.path.isdir(os.path.join(ref, "src")):
        raise SystemExit(f"build_dropin.py: reference tree {ref} not found")
    lib = os.path.join(ROOT, "cps_public_b200", "libcpsb200.so")
    for need in (os.path.join(OUT, "libcps.a"), lib):
        if not os.path.exists(need):
            raise SystemExit(f"build_dropin.py: {need} missing (oracle/build_ref.sh, python -m cps_public_b200.build)")
    blocks = cpp_blocks(open(os.path.join(ROOT, "INTEGRATION.md")).read())
    hdr, src = bridge_sources(blocks)
    branches = branch_blocks(blocks)
    os.makedirs(os.path.join(B200, "include", "util"), exist_ok=True)
    os.makedirs(os.path.join(B200, "src"), exist_ok=True)
    os.makedirs(os.path.join(B200, "obj"), exist_ok=True)
    with open(os.path.join(B200, "include", "util", "b200_bridge.h"), "w") as f:
        f.write(hdr)
    with open(os.path.join(B200, "src", "b200_bridge.C"), "w") as f:
        f.write(src)
    inc = ["-I" + os.path.join(B200, "include"), "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(HERE, "ref_config"), "-I" + os.path.join(ref, "include")]
    objs = []
    for rel, cls in FILES.items():
        path = os.path.join(ref, "src", "util", "lattice", rel)
        patched = patch(open(path).read(), path, cls, branches)
        dst = os.path.join(B200, "src", os.path.basename(rel))
        with open(dst, "w") as f:
            f.write(patched)
        obj = os.path.join(B200, "obj", os.path.basename(rel) + ".o")
        run(["g++", "-x", "c++", *CXXFLAGS, *inc, "-c", dst, "-o", obj])
        objs.append(obj)
    obj = os.path.join(B200, "obj", "b200_bridge.o")
    run(["g++", "-x", "c++", *CXXFLAGS, *inc, "-c", os.path.join(B200, "src", "b200_bridge.C"), "-o", obj])
    objs.append(obj)
    harness = os.path.join(B200, "obj", "ref_harness.o")
    run(["g++", "-x", "c++", *CXXFLAGS, *inc, "-c", os.path.join(HERE, "ref_harness.C"), "-o", harness])
    stubs = os.path.join(OUT, "stubs.o")
    libdir = os.path.dirname(lib)
    exe = os.path.join(OUT, "cpsref_b200")
    # the patched objects come first: their definitions win over the archive's
    run(["g++", "-fopenmp", harness, *objs, *( [stubs] if os.path.exists(stubs) else []),
         os.path.join(OUT, "libcps.a"), "-L" + libdir, "-lcpsb200",
         "-Wl,-rpath," + os.path.relpath(libdir, OUT).join(["$ORIGIN/", ""]), "-Wl,--allow-multiple-definition",
         "-lm", "-o", exe])
    print("built", exe)


if __name__ == "__main__":
    main()
