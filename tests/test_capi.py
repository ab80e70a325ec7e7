"""CPU tests of the drop-in boundary: libzkb200.so loads and exports every symbol declared in
include/zkb200.h (no compute calls: this container has no GPU)."""
import ctypes
import os
import re

import zkutil as Z

HEADER = os.path.join(Z.ROOT, "include", "zkb200.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:void|zkg_status|int|float|uint64_t|const char\s*\*)\s*\*?\s*(\w+)\s*\(",
                                 txt, flags=re.M)))


def test_header_declares_all_reference_entry_points():
    syms = declared_symbols()
    for curve in ("bn128", "bls12_381"):
        for fam, kinds in (("proj", ("proj", "affine")), ("jac", ("jac", "affine"))):
            for coeff in ("std", "mont"):
                for kind in kinds:
                    assert "%s_G1_%s_MSM_%s_coeff_%s_out" % (curve, fam, coeff, kind) in syms
        assert "%s_poly_mont_ntt_forward" % curve in syms
        assert "%s_poly_mont_ntt_inverse" % curve in syms


def test_library_exports_every_declared_symbol(zk):
    L = ctypes.CDLL(zk.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert len(declared_symbols()) >= 30


def test_reference_signatures_match_reference_headers():
    """each drop-in prototype equals the reference header's (when the reference tree is present)"""
    d = os.environ.get("ZKB_REFERENCE_DIR") or os.path.join(os.path.dirname(Z.ROOT), "reference")
    ref = os.path.join(d, "lib", "cbits", "curves")
    if not os.path.isdir(ref):
        import pytest
        pytest.skip("reference tree not available")
    mine = open(HEADER).read()
    norm = lambda s: re.sub(r"\s+", "", s.replace("extern", ""))
    for sub in ("g1/proj/bn128_G1_proj.h", "g1/jac/bn128_G1_jac.h", "poly/mont/bn128_poly_mont.h",
                "g1/proj/bls12_381_G1_proj.h", "g1/jac/bls12_381_G1_jac.h", "poly/mont/bls12_381_poly_mont.h"):
        for line in open(os.path.join(ref, sub)):
            if re.search(r"_MSM_(std|mont)_coeff_(proj|jac|affine)_out\(|_ntt_(forward|inverse)\(", line):
                assert norm(line) in norm(mine), line


def test_window_rule_without_gpu(zk):
    L = zk.lib()
    assert L.zkg_msm_window_for(0, 1 << 22) >= 12
    assert L.zkg_msm_window_for(1, 1 << 10) >= 2
