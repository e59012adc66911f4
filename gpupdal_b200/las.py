"""LAS point files as tile input: the header through the library's parser
(nbg_las_header) and the point records handed whole to nbg_tile_upload_las,
which decodes X/Y/Z on the device.

Follows the fork's direct LAS hydration (src/pdal/PdgNeighborhood.cpp:
1115-1192): the file is mapped, its record extent checked against the mapped
size, the records copied to the device and the raw int32 coordinates decoded
there (src/io/las/LasKernels.cu:266-321); coordinates stay the file's raw
integers with its scale and offset.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi


class LasError(ValueError):
    pass


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())


def header(data) -> dict:
    """Parses a LAS public header block (bytes-like or uint8 array holding at
    least the header) into a dict of nbg_las_info's fields."""
    lib = abi.load_library()
    buf = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    info = abi.LasInfo()
    rc = lib.nbg_las_header(_ptr(buf), int(buf.nbytes), ctypes.byref(info))
    if rc != abi.NBG_OK:
        raise LasError("not a LAS 1.0-1.4 header (signature, point format or record length)")
    out = {f: getattr(info, f) for f, _ in abi.LasInfo._fields_ if f != "reserved"}
    for f in ("scale", "offset", "min", "max"):
        out[f] = tuple(out[f])
    return out


class LasFile:
    """A LAS file mapped read-only; `records` is the point records' bytes
    (point_count x point_record_length, uint8)."""

    def __init__(self, path):
        self.path = str(path)
        self.map = np.memmap(self.path, dtype=np.uint8, mode="r")
        self.info = header(self.map)
        if self.info["compressed"]:
            raise LasError(f"{self.path}: LAZ-compressed records are not decoded here")
        rl = self.info["point_record_length"]
        n = self.info["point_count"]
        start = self.info["offset_to_points"]
        if start > self.map.size or n * rl > self.map.size - start:
            raise LasError(f"{self.path}: point records exceed the mapped file")
        self.n = int(n)
        self.record_length = int(rl)
        self.records = self.map[start:start + n * rl]

    @property
    def scale(self):
        return self.info["scale"]

    @property
    def offset(self):
        return self.info["offset"]

    def raw_xyz(self):
        """The records' raw X, Y, Z (int32) decoded on the host, for checks."""
        r = np.asarray(self.records).reshape(self.n, self.record_length)
        return tuple(np.ascontiguousarray(r[:, 4 * d:4 * d + 4]).view("<i4").reshape(-1)
                     for d in range(3))


def write_las(path, x, y, z, scale=(0.01, 0.01, 0.01), offset=(0.0, 0.0, 0.0),
              version=(1, 2), point_format=1, extra_bytes=0, fill=None):
    """Writes raw int32 coordinates as a LAS file (ASPRS LAS 1.2/1.4 layout,
    no VLRs): X, Y, Z at the start of each record, the rest of the record
    (`fill`, a uint8 array of the remaining bytes per point, else zeros)."""
    import struct
    x, y, z = (np.asarray(v, dtype=np.int32) for v in (x, y, z))
    n = len(x)
    base_len = {0: 20, 1: 28, 2: 26, 3: 34, 6: 30, 7: 36, 8: 38}[point_format]
    rl = base_len + extra_bytes
    hsize = {(1, 2): 227, (1, 3): 235, (1, 4): 375}[tuple(version)]
    h = bytearray(hsize)
    h[0:4] = b"LASF"
    h[24], h[25] = version
    h[26:26 + 11] = b"gpupdal_b200"[:11]
    struct.pack_into("<HIIBHI", h, 94, hsize, hsize, 0, point_format, rl,
                     n if (point_format < 6 and n < 2 ** 32) else 0)
    struct.pack_into("<3d3d", h, 131, *scale, *offset)
    lo = [min(v.min(), 0) * s + o if n else 0.0 for v, s, o in zip((x, y, z), scale, offset)]
    hi = [max(v.max(), 0) * s + o if n else 0.0 for v, s, o in zip((x, y, z), scale, offset)]
    struct.pack_into("<6d", h, 179, hi[0], lo[0], hi[1], lo[1], hi[2], lo[2])
    if tuple(version) == (1, 4):
        struct.pack_into("<Q", h, 247, n)
    rec = np.zeros((n, rl), dtype=np.uint8)
    if fill is not None:
        rec[:, 12:] = np.asarray(fill, dtype=np.uint8).reshape(n, rl - 12)
    for d, v in enumerate((x, y, z)):
        rec[:, 4 * d:4 * d + 4] = v.astype("<i4").view(np.uint8).reshape(n, 4)
    with open(path, "wb") as f:
        f.write(bytes(h))
        f.write(rec.tobytes())
    return rl
