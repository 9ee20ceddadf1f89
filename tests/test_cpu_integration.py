"""The CPS-side binding shown in INTEGRATION.md compiles against CPS's own
sources: the bridge header and source as written there, CPS's f_dwf_base.C,
f_mobius.C and f_wilson.C with the USE_B200 branch blocks inserted at the top
of the functions each block names (the patching oracle/build_dropin.py does for
the linked build), and the operator-level branch inside a DiracOpDwf member.
Every block must be used: each branch block names at least one function, and
every named function is found on the line the block cites.  Skipped where the
reference tree is not present."""
import os
import shutil
import subprocess

import pytest

from oracle import build_dropin

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference():
    from __graft_entry__ import REFERENCE
    if not os.path.isdir(os.path.join(REFERENCE, "include")):
        pytest.skip("reference tree not present")
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    return REFERENCE


def syntax_ok(tmp_path, name, source, ref):
    path = tmp_path / name
    path.write_text(source)
    cmd = ["g++", "-x", "c++", "-std=gnu++11", "-fsyntax-only", "-w", "-DUSE_B200", f"-I{tmp_path / 'include'}",
           f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(ROOT, 'oracle', 'ref_config')}",
           f"-I{os.path.join(ref, 'include')}", str(path)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.fixture
def bridge(tmp_path):
    ref = reference()
    blocks = build_dropin.cpp_blocks(open(os.path.join(ROOT, "INTEGRATION.md")).read())
    hdr, src = build_dropin.bridge_sources(blocks)
    (tmp_path / "include" / "util").mkdir(parents=True)
    (tmp_path / "include" / "util" / "b200_bridge.h").write_text(hdr)
    return tmp_path, ref, blocks, src


def test_bridge_source_compiles(bridge):
    tmp_path, ref, blocks, src = bridge
    syntax_ok(tmp_path, "b200_bridge.C", src, ref)


def test_branches_compile_in_the_cps_files(bridge):
    tmp_path, ref, blocks, _ = bridge
    branches = build_dropin.branch_blocks(blocks)
    calls = {"b200_fmat_evl_inv", "b200_fmat_evl_minv", "b200_fmat_inv"}
    assert calls == {c for _, body in branches for c in calls if c in body}
    named = {(c, f) for targets, _ in branches for c, f, _ in targets}
    assert len(named) == 9, named   # FmatEvlInv, FmatEvlMInv, FmatInv of three lattice classes
    for rel, cls in build_dropin.FILES.items():
        path = os.path.join(ref, "src", "util", "lattice", rel)
        patched = build_dropin.patch(open(path).read(), path, cls, branches)
        assert patched.count("#ifdef USE_B200") == 1 + sum(1 for t, _ in branches for c, _, _ in t if c == cls)
        syntax_ok(tmp_path, os.path.basename(rel), patched, ref)


def test_operator_branch_compiles(bridge):
    tmp_path, ref, blocks, _ = bridge
    mdagm = [b for b in blocks if b.startswith("// DiracOpDwf::MatPcDagMatPc")]
    assert len(mdagm) == 1
    tu = f"""#include <config.h>
#include <util/b200_bridge.h>
#include <util/lattice.h>
#include <util/dirac_op.h>
CPS_START_NAMESPACE
struct OperatorCheck : public DiracOpDwf {{
  void mdagm(Vector *out, Vector *in, Float *dot_prd) {{
{mdagm[0]}
  }}
}};
CPS_END_NAMESPACE
"""
    syntax_ok(tmp_path, "operator.C", tu, ref)
