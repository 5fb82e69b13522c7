"""LAS point data on the CUDA library.

Mirrors crates/spatialrust-io/src/las (read_las / LasReader, reader.rs:21-87;
LasChunkSource, reader.rs:88-190; schema_for_las_header, schema.rs:27-52;
metadata_from_las_header, reader.rs:219-231).  The header is parsed on the
host (ASPRS LAS 1.4 R15, table 3); the point records go to the device as raw
bytes and are decoded there (srcu_las_decode), optionally with an FP64
origin subtracted before the f32 conversion.  Compressed point data
(LAZ / COPC) is not decoded.

encode_las() writes uncompressed LAS bytes from columns: inputs for tests and
benchmarks, not a mirror of the reference's writer.
"""
from __future__ import annotations

import ctypes
import struct
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _native
from .core import (DType, FieldSemantic, InvalidArgument, PointCloud, PointField, StandardSchemas,
                   UnsupportedDType)

# point data record format -> (standard record length, GPS-time offset, RGB offset)
LAS_LAYOUTS = {0: (20, None, None), 1: (28, 20, None), 2: (26, None, 20), 3: (34, 20, 28),
               4: (57, 20, None), 5: (63, 20, 28), 6: (30, 22, None), 7: (36, 22, 30),
               8: (38, 22, 30), 9: (59, 22, None), 10: (67, 22, 30)}


class LasError(InvalidArgument):
    """A malformed or unsupported LAS file."""


@dataclass(frozen=True)
class LasHeader:
    version: tuple
    header_size: int
    offset_to_point_data: int
    point_format: int
    record_length: int
    point_count: int
    scale: tuple
    offset: tuple
    min: tuple
    max: tuple
    compressed: bool

    @property
    def has_gps_time(self) -> bool:
        return LAS_LAYOUTS[self.point_format][1] is not None

    @property
    def has_color(self) -> bool:
        return LAS_LAYOUTS[self.point_format][2] is not None


def parse_header(buf: bytes) -> LasHeader:
    """Public header block fields (LAS 1.0-1.4)."""
    if len(buf) < 227 or buf[:4] != b"LASF":
        raise LasError("not a LAS file (missing LASF signature)")
    major, minor = buf[24], buf[25]
    header_size, = struct.unpack_from("<H", buf, 94)
    offset_to_points, = struct.unpack_from("<I", buf, 96)
    fmt_byte = buf[104]
    record_length, = struct.unpack_from("<H", buf, 105)
    legacy_count, = struct.unpack_from("<I", buf, 107)
    scale = struct.unpack_from("<3d", buf, 131)
    offset = struct.unpack_from("<3d", buf, 155)
    mx_x, mn_x, mx_y, mn_y, mx_z, mn_z = struct.unpack_from("<6d", buf, 179)
    count = legacy_count
    if (major, minor) >= (1, 4) and len(buf) >= 255:
        count64, = struct.unpack_from("<Q", buf, 247)
        count = count64 or legacy_count
    fmt = fmt_byte & 0x3F
    if fmt not in LAS_LAYOUTS:
        raise LasError(f"LAS point data record format {fmt} is not 0-10")
    if record_length < LAS_LAYOUTS[fmt][0]:
        raise LasError(f"record length {record_length} is short for point format {fmt}")
    return LasHeader((major, minor), header_size, offset_to_points, fmt, record_length, count,
                     scale, offset, (mn_x, mn_y, mn_z), (mx_x, mx_y, mx_z), bool(fmt_byte & 0xC0))


def schema_for_las_header(header: LasHeader):
    """schema_for_las_header (schema.rs:27-52)."""
    schema = StandardSchemas.point_xyzi().with_field(
        PointField.scalar("classification", FieldSemantic.Label, DType.U8))
    if header.has_gps_time:
        schema = schema.with_field(PointField.scalar("gps_time", FieldSemantic.TimeOffset, DType.F64))
    if header.has_color:
        for name, sem in (("red", FieldSemantic.ColorR), ("green", FieldSemantic.ColorG),
                          ("blue", FieldSemantic.ColorB)):
            schema = schema.with_field(PointField.scalar(name, sem, DType.U16))
    return schema


def metadata_from_las_header(origin=None) -> dict:
    """metadata_from_las_header (reader.rs:219-231), plus the FP64 origin
    subtracted from the coordinates when one was given."""
    md = {"frame_id": "las", "timestamp": 0, "sensor_origin": None, "unit": "meter"}
    if origin is not None:
        md["origin"] = tuple(float(v) for v in origin)
    return md


def decode_records(records, header: LasHeader, origin=None, device: int = 0) -> dict:
    """Columns of raw point records: a uint8 numpy array (host) or CUDA tensor
    (device, outputs are then CUDA tensors) of n * record_length bytes."""
    if header.compressed:
        raise UnsupportedDType("compressed LAS point data (LAZ / COPC) is not decoded")
    rl = header.record_length
    on_dev = _native._is_device(records)
    nbytes = int(records.numel()) if on_dev else int(np.asarray(records).nbytes)
    if nbytes % rl:
        raise LasError(f"{nbytes} record bytes are not a multiple of the record length {rl}")
    n = nbytes // rl
    keep = []
    if on_dev:
        import torch
        if records.dtype != torch.uint8 or not records.is_contiguous():
            raise InvalidArgument("device records must be a contiguous uint8 CUDA tensor")
        dev = torch.device("cuda", device)

        def alloc(dtype, np_dtype):
            return torch.empty(max(n, 1), dtype=dtype, device=dev)
        f32, u8, f64, u16 = torch.float32, torch.uint8, torch.float64, torch.int16
        rec_addr = records.data_ptr()
    else:
        rec = np.ascontiguousarray(records, np.uint8)
        keep.append(rec)

        def alloc(dtype, np_dtype):
            return np.empty(max(n, 1), np_dtype)
        f32, u8, f64, u16 = (None,) * 4
        rec_addr = rec.ctypes.data
    cols = {"x": alloc(f32, np.float32), "y": alloc(f32, np.float32), "z": alloc(f32, np.float32),
            "intensity": alloc(f32, np.float32), "classification": alloc(u8, np.uint8)}
    if header.has_gps_time:
        cols["gps_time"] = alloc(f64, np.float64)
    if header.has_color:
        for c in ("red", "green", "blue"):
            cols[c] = alloc(u16, np.uint16)
    fmt = _native.SrcuLasFormat(header.point_format, rl, (ctypes.c_double * 3)(*header.scale),
                                (ctypes.c_double * 3)(*header.offset), int(origin is not None), 0,
                                (ctypes.c_double * 3)(*(origin if origin is not None else (0, 0, 0))))
    out = _native.SrcuLasOut(*[_native._addr(cols.get(k)) for k in
                               ("x", "y", "z", "intensity", "classification", "gps_time", "red",
                                "green", "blue")], int(on_dev))
    ctx = _native.shared_context(device)
    ctx._check(ctx._lib.srcu_las_decode(ctx.handle, ctypes.c_void_p(rec_addr), n, int(on_dev),
                                        ctypes.byref(fmt), ctypes.byref(out)))
    # on the device the colour columns are int16 tensors holding the u16 bits
    return {k: v[:n] for k, v in cols.items()}


def _cloud(header: LasHeader, cols: dict, origin) -> PointCloud:
    schema = schema_for_las_header(header)
    host = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in cols.items()}
    for c in ("red", "green", "blue"):
        if c in host:
            host[c] = host[c].view(np.uint16)
    return PointCloud(schema, host, metadata_from_las_header(origin))


def _read_bytes(source) -> bytes:
    if isinstance(source, (bytes, bytearray, memoryview)):
        return bytes(source)
    with open(source, "rb") as f:
        return f.read()


def read_las(source, origin=None, device: int = 0) -> PointCloud:
    """read_las / read_las_file (reader.rs:71-87): a whole LAS file (path or
    bytes) as a PointCloud, decoded on the device."""
    buf = _read_bytes(source)
    h = parse_header(buf)
    start = h.offset_to_point_data
    end = start + h.point_count * h.record_length
    if end > len(buf):
        raise LasError(f"point data ends at byte {end}, the file has {len(buf)}")
    records = np.frombuffer(buf, np.uint8, end - start, start)
    return _cloud(h, decode_records(records, h, origin, device), origin)


class LasReader:
    """LasReader (reader.rs:21-59): header parsed eagerly, points read once."""

    def __init__(self, path, origin=None, device: int = 0):
        self._path = path
        with open(path, "rb") as f:
            self._header = parse_header(f.read(375))
        self._origin = origin
        self._device = device
        self._loaded = False

    @staticmethod
    def open(path, origin=None, device: int = 0) -> "LasReader":
        return LasReader(path, origin, device)

    def header(self) -> LasHeader:
        return self._header

    def schema(self):
        return schema_for_las_header(self._header)

    def read_cloud(self) -> PointCloud:
        if self._loaded:
            raise LasError("LAS reader already consumed")
        self._loaded = True
        return read_las(self._path, self._origin, self._device)


class LasChunkSource:
    """LasChunkSource (reader.rs:88-190): bounded sequential chunks of
    chunk_points points, each decoded on the device."""

    def __init__(self, path, chunk_points: int, origin=None, device: int = 0):
        if chunk_points <= 0:
            raise InvalidArgument("chunk_points must be positive")
        self._f = open(path, "rb")
        self._header = parse_header(self._f.read(375))
        if self._header.compressed:
            raise UnsupportedDType("compressed LAS point data (LAZ / COPC) is not decoded")
        self.schema = schema_for_las_header(self._header)
        self.chunk_points = int(chunk_points)
        self._origin = origin
        self._device = device
        self._next = 0

    def header(self) -> LasHeader:
        return self._header

    def next_chunk(self) -> Optional[PointCloud]:
        h = self._header
        if self._next >= h.point_count:
            self._f.close()
            return None
        count = min(self.chunk_points, h.point_count - self._next)
        self._f.seek(h.offset_to_point_data + self._next * h.record_length)
        data = self._f.read(count * h.record_length)
        if len(data) != count * h.record_length:
            raise LasError("LAS point data is truncated")
        self._next += count
        cols = decode_records(np.frombuffer(data, np.uint8), h, self._origin, self._device)
        return _cloud(h, cols, self._origin)


def encode_las(x, y, z, point_format: int = 1, scale=(0.001, 0.001, 0.001), offset=(0.0, 0.0, 0.0),
               intensity=None, classification=None, gps_time=None, rgb: Sequence = None,
               record_length: Optional[int] = None, version=(1, 4)) -> bytes:
    """Uncompressed LAS bytes (public header + point records, no VLRs): X =
    round((x - offset) / scale) per axis.  For producing inputs."""
    std, gps_off, rgb_off = LAS_LAYOUTS[point_format]
    rl = record_length or std
    if rl < std:
        raise LasError("record length is short for the point format")
    n = len(x)
    w = [np.round((np.asarray(v, np.float64) - o) / s).astype(np.int64)
         for v, o, s in zip((x, y, z), offset, scale)]
    rec = np.zeros((n, rl), np.uint8)
    for a in range(3):
        rec[:, 4 * a:4 * a + 4] = w[a].astype("<i4").view(np.uint8).reshape(n, 4)
    if intensity is not None:
        rec[:, 12:14] = np.asarray(intensity, "<u2").view(np.uint8).reshape(n, 2)
    if classification is not None:
        cls = np.asarray(classification, np.uint8)
        if point_format >= 6:
            rec[:, 16] = cls
        else:
            rec[:, 15] = cls & 0x1F
    if gps_time is not None and gps_off is not None:
        rec[:, gps_off:gps_off + 8] = np.asarray(gps_time, "<f8").view(np.uint8).reshape(n, 8)
    if rgb is not None and rgb_off is not None:
        for c in range(3):
            rec[:, rgb_off + 2 * c:rgb_off + 2 * c + 2] = \
                np.asarray(rgb[c], "<u2").view(np.uint8).reshape(n, 2)
    header_size = 375 if version >= (1, 4) else 227
    hdr = bytearray(header_size)
    hdr[0:4] = b"LASF"
    hdr[24], hdr[25] = version
    struct.pack_into("<H", hdr, 94, header_size)
    struct.pack_into("<I", hdr, 96, header_size)
    hdr[104] = point_format
    struct.pack_into("<H", hdr, 105, rl)
    struct.pack_into("<I", hdr, 107, n if (n < 2 ** 32 and point_format < 6) else 0)
    struct.pack_into("<3d", hdr, 131, *scale)
    struct.pack_into("<3d", hdr, 155, *offset)
    if n:
        world = [np.asarray(v, np.float64) for v in (x, y, z)]
        struct.pack_into("<6d", hdr, 179, world[0].max(), world[0].min(), world[1].max(),
                         world[1].min(), world[2].max(), world[2].min())
    if header_size >= 375:
        struct.pack_into("<Q", hdr, 247, n)
    return bytes(hdr) + rec.tobytes()
