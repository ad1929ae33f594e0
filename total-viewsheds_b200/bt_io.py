"""Binary Terrain (.bt, v1.3) files: the reference's DEM input format.

read_bt restates BinaryTerrain::read (crates/total-viewsheds/src/input.rs:86-175):
the 10-byte "binterr1.3" magic, little-endian header fields, and row-major
i16 or f32 heights starting at byte offset 256.  write_bt produces files that
reader accepts.  scale() restates input.rs:178-185 (Haversine distance of
the top edge / width, with the reference's (top, right) point order: geo's
Point::new takes (x = lon, y = lat), so the reference passes latitude as
longitude and vice versa; kept as is).
"""

import math
import struct

import numpy as np

MAGIC = b"binterr1.3"
HEADER_BYTES = 256
_FIELDS = "<IIHHHHHddddHf"  # width .. vertical_scale, after the magic


class BtError(ValueError):
    pass


def write_bt(path, heights, left=0.0, right=1.0, bottom=0.0, top=1.0, as_float=True,
             horizontal_units=1, utm_zone=0, datum=6326):
    z = np.asarray(heights)
    h, w = z.shape
    data = z.astype("<f4" if as_float else "<i2")
    head = MAGIC + struct.pack(_FIELDS, w, h, 4 if as_float else 2, 1 if as_float else 0,
                               horizontal_units, utm_zone, datum, left, right, bottom, top, 0,
                               1.0)
    with open(path, "wb") as f:
        f.write(head.ljust(HEADER_BYTES, b"\0"))
        f.write(data.tobytes())


def read_bt(path):
    """Returns (header dict, heights as f32 [height, width]).  i16 data is
    converted to f32 as main.rs:51-56 does."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 10 or not raw[:10].startswith(MAGIC):
        raise BtError("Not a Binary Terrain v1.3 file")
    need = 10 + struct.calcsize(_FIELDS)
    if len(raw) < need:
        raise BtError("truncated .bt header")
    (w, h, data_size, is_float, hu, utm, datum, left, right, bottom, top, proj,
     vscale) = struct.unpack_from(_FIELDS, raw, 10)
    header = dict(width=w, height=h, data_size=data_size, is_float=bool(is_float),
                  horizontal_units=hu, utm_zone=utm, datum=datum, left=left, right=right,
                  bottom=bottom, top=top, projection_source=proj, vertical_scale=vscale)
    n = w * h
    if is_float:
        nbytes, dtype = n * 4, "<f4"
    else:
        if data_size != 2:
            raise BtError(f"Unsupported `.bt` field value for data size: {data_size}")
        nbytes, dtype = n * 2, "<i2"
    body = raw[HEADER_BYTES:HEADER_BYTES + nbytes]
    if len(body) < nbytes:
        raise BtError("truncated .bt elevation data")
    z = np.frombuffer(body, dtype).astype(np.float32).reshape(h, w)
    return header, z


def scale(header):
    """input.rs:178-185 with geo 0.30's Haversine (mean earth radius 6371008.8 m)."""
    r = 6371008.8
    # geo::Point::new(x, y): the reference builds (top, right) and (top, left),
    # i.e. x = top, y = right/left; Haversine reads x as longitude.
    lon1, lat1 = math.radians(header["top"]), math.radians(header["right"])
    lon2, lat2 = math.radians(header["top"]), math.radians(header["left"])
    a = (math.sin((lat2 - lat1) / 2) ** 2
         + math.cos(lat1) * math.cos(lat2) * math.sin((lon2 - lon1) / 2) ** 2)
    distance = 2 * r * math.asin(math.sqrt(a))
    return distance / header["width"]
