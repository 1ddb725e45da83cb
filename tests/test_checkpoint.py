"""Density checkpoint files (dss_load_density, host only): a file written in the
documented layout reads back bit for bit, and damaged or mismatched files are
rejected.  The save -> load -> restart round trip after device solves is in
tests/test_gpu_checkpoint.py."""
import struct

import numpy as np
import pytest

from dollarstorescf_b200 import _lib
from dollarstorescf_b200.engine import load_density


def fnv1a(b: bytes) -> int:
    h = 1469598103934665603
    for x in b:
        h ^= x
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def write_file(path, nbf, spins, na, nb, mats, magic=b"DSSDENS1"):
    body = struct.pack("<4i", nbf, spins, na, nb) + b"".join(np.asarray(m, dtype="<f8").tobytes() for m in mats)
    with open(path, "wb") as f:
        f.write(magic + body + struct.pack("<Q", fnv1a(body)))


def test_restricted_and_unrestricted_files_read_back(tmp_path):
    rng = np.random.default_rng(5)
    n = 7
    np_ = n * (n + 1) // 2
    Da = rng.standard_normal(np_)
    write_file(tmp_path / "r.dss", n, 1, 4, 4, [Da])
    a, b, sp, na, nb = load_density(str(tmp_path / "r.dss"), n)
    assert sp == 1 and na == 4 and nb == 4
    assert np.array_equal(a, Da) and np.array_equal(b, Da)
    Db = rng.standard_normal(np_)
    write_file(tmp_path / "u.dss", n, 2, 5, 3, [Da, Db])
    a, b, sp, na, nb = load_density(str(tmp_path / "u.dss"), n)
    assert sp == 2 and na == 5 and nb == 3
    assert np.array_equal(a, Da) and np.array_equal(b, Db)


def test_damaged_or_mismatched_files_are_rejected(tmp_path):
    n = 5
    D = np.arange(n * (n + 1) // 2, dtype=float)
    good = tmp_path / "g.dss"
    write_file(good, n, 1, 2, 2, [D])
    with pytest.raises(_lib.DssError):
        load_density(str(good), n + 1)  # another basis size
    raw = good.read_bytes()
    for name, data in (("trunc", raw[:-9]), ("long", raw + b"\0" * 8),
                       ("flip", raw[:40] + bytes([raw[40] ^ 1]) + raw[41:])):
        p = tmp_path / name
        p.write_bytes(data)
        with pytest.raises(_lib.DssError):
            load_density(str(p), n)
    write_file(tmp_path / "m.dss", n, 1, 2, 2, [D], magic=b"NOTDENS1")
    with pytest.raises(_lib.DssError):
        load_density(str(tmp_path / "m.dss"), n)
    write_file(tmp_path / "s.dss", n, 3, 2, 2, [D, D, D])
    with pytest.raises(_lib.DssError):
        load_density(str(tmp_path / "s.dss"), n)
    with pytest.raises(_lib.DssError):
        load_density(str(tmp_path / "missing.dss"), n)
