"""The checkpoint byte layout of the reference (crates/trace/src/checkpoint.rs),
read on the host by pfxt_checkpoint_read: the cases of the reference's own
test a_checkpoint_reads_back_as_written_only_under_its_own_key (checkpoint.rs:
250-279), on checkpoints written here byte by byte as Saved::write_to writes
them (checkpoint.rs:82-104)."""
import ctypes as C
import struct

import pytest

from pfx_b200 import abi


def write_to(key: str, size=(3, 2), samples=21, adaptive=False) -> bytes:
    """Saved::write_to of the reference test's `saved(adaptive)` (checkpoint.rs:223-248)."""
    pixels = size[0] * size[1]

    def fill(per, seed):
        return bytes(((n * 7) + seed) & 0xFF for n in range(pixels * per))

    out = b"PFXCKPT1" + struct.pack("<Q", len(key)) + key.encode()
    out += struct.pack("<3I", size[0], size[1], samples)
    out += fill(48, 1) + fill(16, 2) + fill(16, 3) + fill(16, 4)
    if not adaptive:
        out += struct.pack("<I", 0xFFFFFFFF)
    else:
        out += struct.pack("<I", 2) + struct.pack("<IQ", 8, 6) + struct.pack("<IQ", 16, 2) + fill(32, 5)
    return out


def info(key: str, data: bytes):
    lib = abi.load()
    out = abi.CheckpointInfo()
    rc = lib.pfxt_checkpoint_read(key.encode(), data, len(data), C.byref(out))
    return rc, lib.pfxt_last_error().decode(), out


@pytest.mark.parametrize("adaptive", [False, True])
def test_reads_back_only_under_its_own_key(adaptive):
    data = write_to("clip frame 4", adaptive=adaptive)
    rc, _, out = info("clip frame 4", data)
    assert rc == abi.OK
    assert (out.width, out.height, out.samples) == (3, 2, 21)
    assert out.rounds == (2 if adaptive else 0xFFFFFFFF)
    rc, msg, _ = info("clip frame 5", data)
    assert rc == abi.ERR_INVALID and "another render" in msg
    rc, msg, _ = info("clip frame 4", data[:-1])
    assert rc == abi.ERR_INVALID and "cut short" in msg
    rc, msg, _ = info("clip frame 4", data + b"\0")
    assert rc == abi.ERR_INVALID and "past its end" in msg


def test_not_a_checkpoint():
    rc, msg, _ = info("k", b"PNG.....")
    assert rc == abi.ERR_INVALID and "not a pfx checkpoint" in msg
    rc, msg, _ = info("k", b"PFX")
    assert rc == abi.ERR_INVALID and "cut short" in msg
