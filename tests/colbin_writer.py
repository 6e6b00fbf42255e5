"""Writes .colbin v2 files for the ingest tests — TEST INFRASTRUCTURE.

The layout is the reference's on-disk column store (src/infra.h:512-560):
a 48-byte header (magic "TPCHCB01", u32 version 2, u32 column count, u64
row count, u64 source size, i64 source mtime, u64 pad), one 32-byte
descriptor per column (i32 source field index, u8 type, u8 pad, u16 fixed
width, u64 offset, u64 bytes, u64 pad), then each payload at the next
16 KiB boundary."""
import datetime
import struct

import numpy as np

ALIGN = 16384
INT, FLOAT, DATE, CHAR1, CHAR_FIXED = 0, 1, 2, 3, 4


def _up(n: int) -> int:
    return (n + ALIGN - 1) & ~(ALIGN - 1)


def write_colbin(path, columns, rows: int, version: int = 2, magic: bytes = b"TPCHCB01") -> None:
    """`columns`: (source field index, type, numpy array, fixed width)."""
    head = struct.pack("<8sIIQQqQ", magic, version, len(columns), rows, 0, 0, 0)
    assert len(head) == 48
    cursor = _up(48 + 32 * len(columns))
    descs, payloads = [], []
    for idx, dtype, arr, width in columns:
        data = np.ascontiguousarray(arr).tobytes()
        descs.append(struct.pack("<iBBHQQQ", idx, dtype, 0, width, cursor, len(data), 0))
        payloads.append((cursor, data))
        cursor = _up(cursor + len(data))
    with open(path, "wb") as f:
        f.write(head + b"".join(descs))
        for off, data in payloads:
            f.seek(off)
            f.write(data)
        f.truncate(max(cursor, 48 + 32 * len(columns)))


def yyyymmdd(day_numbers: np.ndarray) -> np.ndarray:
    """Days since 1992-01-01 -> YYYYMMDD ints (the reference's date form)."""
    base = datetime.date(1992, 1, 1)
    uniq, inv = np.unique(day_numbers, return_inverse=True)
    conv = np.array([int((base + datetime.timedelta(days=int(d))).strftime("%Y%m%d")) for d in uniq], dtype=np.int32)
    return conv[inv].astype(np.int32)


def fact_as_lineitem(fact) -> list:
    """The synthetic fact table as lineitem-style .colbin columns: quantity
    INT, price / discount / tax FLOAT (currency / fractions), flags CHAR1,
    ship date DATE (YYYYMMDD), at lineitem's field indices."""
    return [
        (4, INT, fact["f_quantity"].astype(np.int32), 0),
        (5, FLOAT, (fact["f_price"] / 100.0).astype(np.float32), 0),
        (6, FLOAT, (fact["f_discount"] / 100.0).astype(np.float32), 0),
        (7, FLOAT, (fact["f_tax"] / 100.0).astype(np.float32), 0),
        (8, CHAR1, fact["f_flag_a"].astype(np.uint8), 0),
        (9, CHAR1, fact["f_flag_b"].astype(np.uint8), 0),
        (10, DATE, yyyymmdd(fact["f_ship_day"]), 0),
    ]
