"""The .colbin v2 reader on the CPU (no GPU): header and directory as the
writer laid them out, 16 KiB-aligned payloads, and the reference's
validity checks (magic, version, payloads inside the file, bytes = rows x
width) reported as errors."""
import struct

import numpy as np
import pytest

from colbin_writer import ALIGN, CHAR1, DATE, FLOAT, INT, write_colbin
from gpudbmetalcodegen_b200 import engine
from gpudbmetalcodegen_b200._lib import GpudbError


def _sample(tmp_path, rows=1000, **kw):
    p = tmp_path / "t.colbin"
    cols = [(4, INT, np.arange(rows, dtype=np.int32), 0),
            (5, FLOAT, np.linspace(0, 1, rows, dtype=np.float32), 0),
            (8, CHAR1, np.full(rows, ord("A"), np.uint8), 0),
            (10, DATE, np.full(rows, 19950617, np.int32), 0)]
    write_colbin(p, cols, rows, **kw)
    return p


def test_inspect_reads_header_and_directory(tmp_path):
    info = engine.colbin_inspect(str(_sample(tmp_path)))
    assert info["rows"] == 1000
    assert [c["index"] for c in info["columns"]] == [4, 5, 8, 10]
    assert [c["dtype"] for c in info["columns"]] == [INT, FLOAT, CHAR1, DATE]
    assert [c["size_bytes"] for c in info["columns"]] == [4000, 4000, 1000, 4000]
    assert all(c["offset"] % ALIGN == 0 for c in info["columns"])


def test_empty_table(tmp_path):
    info = engine.colbin_inspect(str(_sample(tmp_path, rows=0)))
    assert info["rows"] == 0 and all(c["size_bytes"] == 0 for c in info["columns"])


@pytest.mark.parametrize("kw,msg", [({"magic": b"TPCHCB00"}, "bad magic"), ({"version": 1}, "version 1")])
def test_header_is_checked(tmp_path, kw, msg):
    with pytest.raises(GpudbError) as e:
        engine.colbin_inspect(str(_sample(tmp_path, **kw)))
    assert msg in e.value.message


def test_truncated_payload_and_size_mismatch_are_errors(tmp_path):
    p = _sample(tmp_path)
    data = p.read_bytes()
    last = engine.colbin_inspect(str(p))["columns"][-1]
    p.write_bytes(data[:last["offset"] + 100])  # the last payload runs past the end
    with pytest.raises(GpudbError) as e:
        engine.colbin_inspect(str(p))
    assert "beyond the end" in e.value.message
    # a descriptor whose byte count is not rows x width
    d = bytearray(data)
    struct.pack_into("<Q", d, 48 + 16, 3999)
    p.write_bytes(bytes(d))
    with pytest.raises(GpudbError) as e:
        engine.colbin_inspect(str(p))
    assert "not rows x width" in e.value.message
    with pytest.raises(GpudbError):
        engine.colbin_inspect(str(tmp_path / "missing.colbin"))


def test_row_count_that_overflows_rows_times_width_is_rejected(tmp_path):
    # 2^62 int32 rows: rows x 4 wraps to 0 in 64 bits, matching a zero-byte
    # payload unless the reader checks the product before comparing it
    p = tmp_path / "wrap.colbin"
    write_colbin(p, [(4, INT, np.zeros(0, np.int32), 0)], 1 << 62)
    with pytest.raises(GpudbError) as e:
        engine.colbin_inspect(str(p))
    assert "cannot fit" in e.value.message
