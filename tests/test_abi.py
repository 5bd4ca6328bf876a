"""The C-ABI library loads and exports every symbol include/snapi_cuda.h declares (no GPU call)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(snapi_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_all_declared_symbols():
    from snapi_b200 import build as b
    path = b.build_cuda()
    lib = ctypes.CDLL(path)
    names = declared_functions(os.path.join(ROOT, "include", "snapi_cuda.h"))
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_zeeman_pattern_from_library(oracle_lib):
    """snapi_zeeman_pattern (host code of the library) equals the oracle's restatement."""
    import snapi_b200 as sb
    for ju2, jl2, gu, gl in ((4, 4, 1.5, 1.83), (0, 2, 0.0, 2.5), (6, 4, 1.2, 1.0), (2, 4, 0.5, 1.1), (0, 0, 1, 1)):
        a = sb.zeeman_pattern(ju2, jl2, gu, gl)
        b = oracle_lib.zeeman_pattern(ju2, jl2, gu, gl)
        assert a.split == b.split
        for g in range(3):
            assert a.ncomp[g] == b.ncomp[g]
            for i in range(a.ncomp[g]):
                assert abs(a.S[g][i] - b.S[g][i]) < 1e-15 and abs(a.D[g][i] - b.D[g][i]) < 1e-15
