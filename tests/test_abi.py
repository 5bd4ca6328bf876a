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


def test_ctypes_mirror_matches_header_layout(tmp_path):
    """Every ctypes structure of the Python mirror has the size and field offsets the C compiler
    gives the header's struct (a mismatch would pass garbage through the ABI without an error)."""
    import subprocess
    from snapi_b200 import api, eos_tables as et
    structs = {api.SnapiLine: "snapi_line", api.SnapiProblem: "snapi_problem", api.SnapiLmOpts: "snapi_lm_opts",
               api.F0Info: "snapi_f0_info", api.CubeJob: "snapi_cube_job", api.CubeStats: "snapi_cube_stats",
               api.CubeSynthJob: "snapi_cube_synth_job", api.SnapiAliProblem: "snapi_ali_problem",
               api.SnapiAliColumns: "snapi_ali_columns", api.SnapiAliBB: "snapi_ali_bb",
               api.SnapiAliSetupTables: "snapi_ali_setup_tables", api.SnapiAliSetupOut: "snapi_ali_setup_out",
               et.SnapiPartition: "snapi_partition",
               et.SnapiEosLevel: "snapi_eos_level", et.SnapiEosAtom: "snapi_eos_atom",
               et.SnapiEosMolecule: "snapi_eos_molecule", et.SnapiEosLine: "snapi_eos_line",
               et.SnapiEosModel: "snapi_eos_model"}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "snapi_cuda.h"', "int main(void) {"]
    expect = []
    for cls, cname in structs.items():
        lines.append('  printf("%%zu\\n", sizeof(%s));' % cname)
        expect.append(ctypes.sizeof(cls))
        for fname, _ in cls._fields_:  # a trailing underscore stands for a Python keyword
            lines.append('  printf("%%zu\\n", offsetof(%s, %s));' % (cname, fname.rstrip("_")))
            expect.append(getattr(cls, fname).offset)
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == expect
