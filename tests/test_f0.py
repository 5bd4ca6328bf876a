"""ANA .f0 files (snapi_f0_*: host code of libsnapi_cuda) against the reference's own reader and
writer (cmlib/ana_read.cc, cmlib/ana_write.cc, fileio.cc), and the layout of the master's invert
job cubes (master/job.cc:306-334, 575-597).  No GPU: these calls do not touch the device."""
import ctypes
import os

import numpy as np
import pytest

from conftest import load_fixture


@pytest.fixture(scope="module")
def api():
    from snapi_b200 import api as A
    from snapi_b200 import build as b
    b.build_cuda()
    return A


@pytest.fixture(scope="module")
def fx():
    return load_fixture("f0_ref")


def _names(fx, key):
    return [str(n) for n in fx[key]]


def test_writer_bytes_match_reference(api, fx, tmp_path):
    """snapi_f0_write reproduces ana_fzwrite byte for byte: every type, 1-4 dimensions, no header,
    one block, exactly 255 characters, 256 (two blocks), 600 (three) and 4000 (clipped to 15)."""
    for n in _names(fx, "w_names"):
        hdr = bytes(fx["w_%s_header" % n]).decode() if int(fx["w_%s_has_header" % n]) else None
        p = tmp_path / (n + ".f0")
        api.f0_write(str(p), fx["w_%s_data" % n], header=hdr, type=int(fx["w_%s_type" % n]))
        assert p.read_bytes() == bytes(fx["w_%s_bytes" % n]), n


def _check_read(api, path, typ, dims, header, data, name):
    h = api.f0_stat(path)
    assert h["type"] == typ, name
    assert h["dims"] == tuple(int(d) for d in dims), name
    assert h["header"].encode("latin-1") == header, name
    raw = api.f0_read(path)
    assert raw.tobytes() == data, name


def test_reader_matches_reference(api, fx, tmp_path):
    """snapi_f0_stat / snapi_f0_read return what ana_fzread returns (type, dimensions, header text
    of all blocks, elements in native byte order) for the reference-written files, hand-made headers
    (big-endian data, reversed synch pattern, both, two header blocks) and the reference's own test
    files."""
    for n in _names(fx, "w_names"):
        p = tmp_path / ("w_" + n + ".f0")
        p.write_bytes(bytes(fx["w_%s_bytes" % n]))
        d = fx["w_%s_data" % n]
        hdr = bytes(fx["w_%s_header" % n])[:15 * 255]
        _check_read(api, str(p), int(fx["w_%s_type" % n]), d.shape[::-1], hdr, d.tobytes(), n)
    for n in _names(fx, "r_names"):
        p = tmp_path / ("r_" + n + ".f0")
        p.write_bytes(bytes(fx["r_%s_file" % n]))
        _check_read(api, str(p), int(fx["r_%s_type" % n]), fx["r_%s_dims" % n], bytes(fx["r_%s_header" % n]),
                    bytes(fx["r_%s_data" % n]), n)


def test_stat_flags(api, fx, tmp_path):
    cases = {"be_data": (1, 0, 1), "rev_synch": (1, 1, 1), "rev_synch_be": (0, 1, 1), "f64_2blk": (0, 0, 2)}
    for n, (swap, rev, nhb) in cases.items():
        p = tmp_path / (n + ".f0")
        p.write_bytes(bytes(fx["r_%s_file" % n]))
        h = api.f0_stat(str(p))
        assert (h["swap"], h["reversed_synch"], h["nhb"]) == (swap, rev, nhb), n
        assert h["data_offset"] == 512 * nhb and h["compressed"] == 0
    p = tmp_path / "f64_2blk.f0"
    assert api.f0_stat(str(p))["header"] == "x" * 255 + "tail"


def test_read_converts_and_slices(api, fx, tmp_path):
    d16 = fx["w_i16_2d_3blk_data"]
    p = tmp_path / "i16.f0"
    p.write_bytes(bytes(fx["w_i16_2d_3blk_bytes"]))
    assert np.array_equal(api.f0_read(str(p), out_type=api.F0_FLOAT64), d16.astype(np.float64))
    assert np.array_equal(api.f0_read(str(p), out_type=api.F0_FLOAT32), d16.astype(np.float32))
    assert np.array_equal(api.f0_read(str(p), first=5, count=9), d16.ravel()[5:14])
    p = tmp_path / "be.f0"
    p.write_bytes(bytes(fx["r_be_data_file"]))
    ref = np.frombuffer(bytes(fx["r_be_data_data"]), np.float32)
    assert np.array_equal(api.f0_read(str(p), out_type=api.F0_FLOAT64).ravel(), ref.astype(np.float64))
    with pytest.raises(api.SnapiError):
        api.f0_read(str(p), out_type=api.F0_INT16)  # only the file's type, float32 or float64


def test_streaming_writer(api, tmp_path):
    """snapi_f0_create / write_at (ranges in any order) / close give the snapi_f0_write file;
    close reports missing elements (ana_file::~ana_file), ranges outside the file are refused."""
    L = api.lib()
    a = np.arange(5 * 7 * 3, dtype=np.float64).reshape(5, 7, 3)
    ref = tmp_path / "ref.f0"
    api.f0_write(str(ref), a, header="stream")
    dims = (ctypes.c_longlong * 3)(3, 7, 5)
    st = ctypes.c_int(0)
    out = tmp_path / "s.f0"
    f = L.snapi_f0_create(str(out).encode(), api.F0_FLOAT64, 3, dims, b"stream", ctypes.byref(st))
    assert f and st.value == 0
    flat = a.ravel()
    for lo in (90, 40, 0, 60):
        hi = {90: 105, 40: 60, 0: 40, 60: 90}[lo]
        assert L.snapi_f0_write_at(f, lo, hi - lo, flat[lo:].ctypes.data) == 0
    assert L.snapi_f0_write_at(f, 100, 6, flat.ctypes.data) != 0
    assert L.snapi_f0_close(f) == 0
    assert out.read_bytes() == ref.read_bytes()
    f = L.snapi_f0_create(str(tmp_path / "part.f0").encode(), api.F0_FLOAT64, 3, dims, None, ctypes.byref(st))
    assert L.snapi_f0_write_at(f, 0, 10, flat.ctypes.data) == 0
    assert L.snapi_f0_close(f) != 0
    assert b"10 of 105" in L.snapi_f0_error()


def test_errors(api, fx, tmp_path):
    good = bytes(fx["w_f32_3d_bytes"])
    cases = {
        "missing": None,
        "short_header": good[:300],
        "bad_synch": b"\x00\x01\x02\x03" + good[4:],
        "truncated_data": good[:-4],
        "compressed": good[:4] + bytes([good[4] | 1]) + good[5:],
        "bad_type": good[:7] + bytes([9]) + good[8:],
        "bad_ndim": good[:8] + bytes([0]) + good[9:],
        "too_many_blocks": good[:6] + bytes([16]) + good[7:],
    }
    for n, blob in cases.items():
        p = tmp_path / (n + ".f0")
        if blob is not None:
            p.write_bytes(blob)
        with pytest.raises(api.SnapiError):
            api.f0_read(str(p))
    with pytest.raises(api.SnapiError):
        api.f0_write(str(tmp_path / "x.f0"), np.zeros((2, 2)), type=7)


def test_job_output_layouts(api, fx, tmp_path):
    """The invert job's outputs as the reference's write_file calls lay them out: the node cube
    (3-D overload, float32, element (x, y, p) at (p * ny + y) * nx + x) and the fitted spectra
    (4-D overload, float64 S[x][y][s][l] as is)."""
    nodes, spec = fx["cw_nodes"], fx["cw_spec"]
    p = tmp_path / "inverted_nodes.f0"
    api.f0_write(str(p), np.ascontiguousarray(nodes.transpose(2, 1, 0)).astype(np.float32))
    assert p.read_bytes() == bytes(fx["cw_nodes_file"])
    p = tmp_path / "inverted_spectra.f0"
    api.f0_write(str(p), spec)
    assert p.read_bytes() == bytes(fx["cw_spec_file"])


def job_window(cube, sub, obs_qs, synth_qs):
    """The invert job's cube steps restated in numpy (read_file + transpose gives S[x][y][s][l];
    normalize multiplies by synth_qs / obs_qs in float64; extract cuts the 1-based inclusive
    subfield and window)."""
    xl, xh, yl, yh, ll, lh = [int(v) for v in sub]
    S = cube.astype(np.float64) * (synth_qs / obs_qs)
    return np.ascontiguousarray(S[xl - 1:xh, yl - 1:yh, :, ll - 1:lh])


def test_job_cube_steps_restated(api, fx, tmp_path):
    """The numpy restatement of the job's cube steps reproduces the reference's extracted, scaled
    window (float32 and float64 cubes) and its cube_to_invert.f0 byte for byte."""
    for tag in ("f32", "f64"):
        p = tmp_path / ("cube_%s.f0" % tag)
        p.write_bytes(bytes(fx["cube_%s_file" % tag]))
        cube = api.f0_read(str(p))
        assert cube.ndim == 4 and cube.shape[2] == 4
        qs = fx["cube_%s_qs" % tag]
        S = job_window(cube, fx["cube_sub"], qs[0], qs[1])
        assert np.array_equal(S, fx["cube_%s_S" % tag]), tag
        c2i = tmp_path / ("c2i_%s.f0" % tag)
        api.f0_write(str(c2i), S)
        assert c2i.read_bytes() == bytes(fx["cube_%s_c2i" % tag]), tag


def test_streaming_writer_concurrent_ranges(api, tmp_path):
    """snapi_f0_write_at from several host threads at once (positioned writes of disjoint ranges, as
    the invert job's writer thread and a caller's own threads may issue them) gives the same file as
    one snapi_f0_write."""
    import threading
    L = api.lib()
    a = np.random.default_rng(7).standard_normal((64, 4, 201)).astype(np.float64)
    ref = tmp_path / "ref.f0"
    api.f0_write(str(ref), a)
    dims = (ctypes.c_longlong * 3)(201, 4, 64)
    st = ctypes.c_int(0)
    out = tmp_path / "par.f0"
    f = L.snapi_f0_create(str(out).encode(), api.F0_FLOAT64, 3, dims, None, ctypes.byref(st))
    flat = a.ravel()
    per = 4 * 201
    rc = []

    def work(k):
        for px in range(k, 64, 8):
            rc.append(L.snapi_f0_write_at(f, px * per, per, flat[px * per:].ctypes.data))

    threads = [threading.Thread(target=work, args=(k,)) for k in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert rc and all(r == 0 for r in rc)
    assert L.snapi_f0_close(f) == 0
    assert out.read_bytes() == ref.read_bytes()
