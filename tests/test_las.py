"""LAS ingest: header parsing and record extents on the host (no GPU work)."""
import struct

import numpy as np
import pytest

from gpupdal_b200 import las


def _cloud(n=1000, seed=3):
    rng = np.random.default_rng(seed)
    return tuple(rng.integers(-50000, 50000, n).astype(np.int32) for _ in range(3))


@pytest.mark.parametrize("version,fmt,extra", [((1, 2), 1, 0), ((1, 2), 3, 5), ((1, 3), 2, 0),
                                               ((1, 4), 6, 7), ((1, 4), 0, 0)])
def test_header_fields(tmp_path, version, fmt, extra):
    x, y, z = _cloud()
    p = tmp_path / "a.las"
    rl = las.write_las(p, x, y, z, scale=(0.001, 0.001, 0.001), offset=(5e5, 4e6, 10.0),
                       version=version, point_format=fmt, extra_bytes=extra)
    f = las.LasFile(p)
    h = f.info
    assert (h["version_major"], h["version_minor"]) == version
    assert h["point_format"] == fmt and not h["compressed"]
    assert h["point_record_length"] == rl
    assert h["point_count"] == len(x)
    assert h["scale"] == (0.001, 0.001, 0.001) and h["offset"] == (5e5, 4e6, 10.0)
    assert h["offset_to_points"] == {(1, 2): 227, (1, 3): 235, (1, 4): 375}[version]
    assert h["max"][0] == pytest.approx(x.max() * 0.001 + 5e5)
    assert h["min"][2] == pytest.approx(z.min() * 0.001 + 10.0)
    rx, ry, rz = f.raw_xyz()
    assert np.array_equal(rx, x) and np.array_equal(ry, y) and np.array_equal(rz, z)


def test_las14_count_beyond_legacy_field(tmp_path):
    x, y, z = _cloud(64)
    p = tmp_path / "b.las"
    las.write_las(p, x, y, z, version=(1, 4), point_format=6)
    raw = bytearray(p.read_bytes())
    assert struct.unpack_from("<I", raw, 107)[0] == 0  # formats 6-10 leave the legacy count 0
    assert las.header(bytes(raw[:375]))["point_count"] == 64


def test_rejects_bad_headers(tmp_path):
    x, y, z = _cloud(16)
    p = tmp_path / "c.las"
    las.write_las(p, x, y, z)
    raw = bytearray(p.read_bytes())
    with pytest.raises(las.LasError):
        las.header(bytes(raw[:200]))            # shorter than a 1.0 header
    bad = bytearray(raw)
    bad[0:4] = b"LASX"
    with pytest.raises(las.LasError):
        las.header(bytes(bad))
    bad = bytearray(raw)
    bad[104] = 11                               # no such point format
    with pytest.raises(las.LasError):
        las.header(bytes(bad))
    bad = bytearray(raw)
    struct.pack_into("<H", bad, 105, 8)         # record shorter than X, Y, Z
    with pytest.raises(las.LasError):
        las.header(bytes(bad))


def test_compressed_and_truncated_files(tmp_path):
    x, y, z = _cloud(16)
    p = tmp_path / "d.las"
    las.write_las(p, x, y, z)
    raw = bytearray(p.read_bytes())
    laz = bytearray(raw)
    laz[104] |= 0x80
    q = tmp_path / "d.laz"
    q.write_bytes(bytes(laz))
    h = las.header(bytes(laz))
    assert h["compressed"] == 1 and h["point_format"] == 1
    with pytest.raises(las.LasError, match="LAZ"):
        las.LasFile(q)
    t = tmp_path / "e.las"
    t.write_bytes(bytes(raw[:-5]))
    with pytest.raises(las.LasError, match="exceed"):
        las.LasFile(t)


def test_reference_las_fixture(tmp_path):
    # the reference's test/data/las/simple.las (LAS 1.2, format 3), stored as
    # its header block and point records: the header fields, and the raw
    # X/Y/Z the golden outputs were made from
    from tests import _util as U
    g = U.golden("las_simple")
    p = tmp_path / "simple.las"
    p.write_bytes(g["las_header"].tobytes() + g["las_records"].tobytes())
    f = las.LasFile(p)
    h = f.info
    assert (h["version_major"], h["version_minor"], h["point_format"]) == (1, 2, 3)
    assert h["point_record_length"] == 34 and h["point_count"] == 1065
    assert f.scale == (0.01, 0.01, 0.01) and all(o == 0 for o in f.offset)
    rx, ry, rz = f.raw_xyz()
    assert np.array_equal(rx, g["x"]) and np.array_equal(ry, g["y"]) and np.array_equal(rz, g["z"])
    assert h["min"][0] == pytest.approx(g["x"].min() * 0.01)
    assert h["max"][1] == pytest.approx(g["y"].max() * 0.01)


def test_header_parser_survives_mutations():
    # every truncation of the reference's simple.las header block, and every
    # byte of it set to 0x00, 0xFF and a random value: the parser rejects the
    # header or returns one whose fields hold together
    from tests import _util as U
    hdr = bytes(U.golden("las_simple")["las_header"])
    rng = np.random.default_rng(11)

    def check(b):
        try:
            h = las.header(b)
        except las.LasError:
            return
        assert h["point_record_length"] >= 12
        assert h["point_format"] <= 10
        assert h["compressed"] in (0, 1)

    for n in range(len(hdr) + 1):
        check(hdr[:n])
    for i in range(len(hdr)):
        for v in (0x00, 0xFF, int(rng.integers(0, 256))):
            b = bytearray(hdr)
            b[i] = v
            check(bytes(b))
