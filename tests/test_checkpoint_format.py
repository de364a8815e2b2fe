"""CPU tests of the checkpoint container reader (hprqp_b200/checkpoint.py)
against a file written record by record as include/hprqp.h describes it
(hprqp_set_save_file): the magic, then per record a u16 name length, the
name, a type byte (1 float64, 2 int64, 3 string), a u64 count and the
little-endian payload."""
import struct

import numpy as np
import pytest

from hprqp_b200.checkpoint import read_checkpoint


def rec(name, typ, payload, count):
    b = name.encode()
    return struct.pack("<H", len(b)) + b + bytes([typ]) + struct.pack("<Q", count) + payload


def test_reads_every_record_type(tmp_path):
    x = np.array([1.5, -2.0, 3.25])
    data = (b"HPRQPCK1" + rec("current/x_org", 1, x.astype("<f8").tobytes(), 3)
            + rec("current/iteration", 2, struct.pack("<q", 570), 1)
            + rec("parameters/problem_type", 3, b"QP", 2))
    p = tmp_path / "a.ckpt"
    p.write_bytes(data)
    ck = read_checkpoint(str(p))
    assert np.array_equal(ck["current/x_org"], x)
    assert int(ck["current/iteration"][0]) == 570
    assert ck["parameters/problem_type"] == "QP"


def test_rejects_foreign_and_truncated_files(tmp_path):
    p = tmp_path / "b.ckpt"
    p.write_bytes(b"\x89HDF\r\n\x1a\n")
    with pytest.raises(ValueError):
        read_checkpoint(str(p))
    p.write_bytes(b"HPRQPCK1" + rec("x", 1, b"\x00" * 8, 3))
    with pytest.raises(ValueError):
        read_checkpoint(str(p))
