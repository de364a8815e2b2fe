"""Reader of the library's checkpoint files (params.auto_save): the
datasets of the reference's save_state_to_hdf5! (src/algorithm.jl:183-301)
-- current/..., best/..., parameters/... -- and the resume/... section, in
the container described in include/hprqp.h (hprqp_set_save_file):

    "HPRQPCK1", then per record: u16 name length, name, u8 type
    (1 = float64, 2 = int64, 3 = string), u64 count, little-endian payload.

    ck = read_checkpoint("hprqp_autosave.ckpt")
    x = ck["current/x_org"]; it = int(ck["current/iteration"][0])
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"HPRQPCK1"


def read_checkpoint(path: str) -> dict:
    """{name: numpy array (float64 / int64) or str} of a checkpoint file."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC:
        raise ValueError(f"{path} is not a libhprqp checkpoint")
    out, at = {}, 8
    while at < len(data):
        (ln,) = struct.unpack_from("<H", data, at)
        at += 2
        name = data[at:at + ln].decode()
        at += ln
        typ = data[at]
        at += 1
        (count,) = struct.unpack_from("<Q", data, at)
        at += 8
        if typ == 1:
            out[name] = np.frombuffer(data, dtype="<f8", count=count, offset=at).copy()
            at += 8 * count
        elif typ == 2:
            out[name] = np.frombuffer(data, dtype="<i8", count=count, offset=at).copy()
            at += 8 * count
        elif typ == 3:
            out[name] = data[at:at + count].decode()
            at += count
        else:
            raise ValueError(f"{path}: unknown record type {typ}")
        if at > len(data):
            raise ValueError(f"{path} is truncated")
    return out
