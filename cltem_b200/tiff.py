"""Minimal float32 TIFF writer/reader with the layout clTEM's fileio::SaveTiff produces
(src/simulation/utilities/fileio.h:43-76): one sample per pixel, 32-bit IEEE float, one strip holding
all rows, no compression, min-is-black, ORIENTATION_BOTLEFT, contiguous planar configuration."""
import struct

import numpy as np

_TAGS = {  # tag: (type, count, value)   type 3 = SHORT, 4 = LONG
    "ImageWidth": 256, "ImageLength": 257, "BitsPerSample": 258, "Compression": 259, "Photometric": 262,
    "StripOffsets": 273, "Orientation": 274, "SamplesPerPixel": 277, "RowsPerStrip": 278,
    "StripByteCounts": 279, "PlanarConfig": 284, "SampleFormat": 339,
}
ORIENTATION_BOTLEFT = 4


def write_tiff(path: str, data: np.ndarray):
    """data: 2-D array (height, width); row r of the array is written as row r of the strip."""
    a = np.ascontiguousarray(np.asarray(data, dtype="<f4"))
    h, w = a.shape
    payload = a.tobytes()
    n_tags = 12
    ifd_offset = 8
    ifd_size = 2 + n_tags * 12 + 4
    data_offset = ifd_offset + ifd_size
    entries = [
        (256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, 32), (259, 3, 1, 1), (262, 3, 1, 1),
        (273, 4, 1, data_offset), (274, 3, 1, ORIENTATION_BOTLEFT), (277, 3, 1, 1), (278, 4, 1, h),
        (279, 4, 1, len(payload)), (284, 3, 1, 1), (339, 3, 1, 3),
    ]
    with open(path, "wb") as f:
        f.write(b"II*\x00" + struct.pack("<I", ifd_offset))
        f.write(struct.pack("<H", n_tags))
        for tag, typ, count, val in entries:
            if typ == 3:
                f.write(struct.pack("<HHIHH", tag, typ, count, val, 0))
            else:
                f.write(struct.pack("<HHII", tag, typ, count, val))
        f.write(struct.pack("<I", 0))
        f.write(payload)


def read_tiff(path: str):
    """Read back a file written by write_tiff (or any single-strip float32 little-endian TIFF):
    returns (array, tags)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:4] != b"II*\x00":
        raise ValueError("not a little-endian TIFF")
    (ifd,) = struct.unpack_from("<I", buf, 4)
    (n,) = struct.unpack_from("<H", buf, ifd)
    tags = {}
    for i in range(n):
        tag, typ, count = struct.unpack_from("<HHI", buf, ifd + 2 + 12 * i)
        if typ == 3:
            (val,) = struct.unpack_from("<H", buf, ifd + 2 + 12 * i + 8)
        else:
            (val,) = struct.unpack_from("<I", buf, ifd + 2 + 12 * i + 8)
        tags[tag] = val
    w, h, off = tags[256], tags[257], tags[273]
    a = np.frombuffer(buf, dtype="<f4", count=w * h, offset=off).reshape(h, w)
    return a, tags
