"""MSPB v1 snapshots and MSPBPack archives (modules_b200.mspb), host only.

Fixtures are assembled byte by byte from the layout tables of the reference's EXPORT_FORMAT.md / MSPB_PACK.md,
independently of the module's writer, as the reference's own tests/test_mspb_pack.cpp does. Where the reference was
compiled (oracle/_ref), files also cross between this module and the reference's MSPBSnapshot / MSPB_Pack code: each
side reads what the other wrote, and both write the same bytes for the same snapshot."""
import os
import struct

import numpy as np
import pytest

import oracle
from modules_b200 import mspb

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")


def sample(d):
    """A skew cell, arbitrary (non-index) IDs, unequal radii, a declared but empty species."""
    basis = np.eye(d) * 3.0
    basis[d - 1, 0] = 0.75
    if d > 1:
        basis[0, d - 1] = -0.25
    rel = np.array([[0.1, 0.2, 0.3, 0.4][:d], [0.5, -0.25, 1.5, 0.0][:d], [0.999, 0.0, 0.125, 0.5][:d]])
    return mspb.Snapshot.create(basis, rel, species=[0, 2, 2], radii=[0.5, 0.25, 1.25],
                                ids=[7, 2**63 + 5, 0], species_count=4)


def raw(s):
    """The snapshot's bytes from the layout table, field by field."""
    d = s.basis.shape[0]
    out = b"MSPB\r\n\x1a\n" + struct.pack("<I", 1) + struct.pack("<I", d) + struct.pack("<Q", len(s.ids))
    out += struct.pack("<Q", s.species_count) + struct.pack("<I", 3)
    for row in s.basis:
        for x in row:
            out += struct.pack("<d", float(x))
    for i in range(len(s.ids)):
        out += struct.pack("<Q", int(s.ids[i])) + struct.pack("<I", int(s.species[i]))
        for x in s.rel[i]:
            out += struct.pack("<d", float(x))
        out += struct.pack("<d", float(s.radii[i]))
    return out


def same(a, b):
    return (a.species_count == b.species_count and np.array_equal(a.basis, b.basis) and
            np.array_equal(a.ids, b.ids) and np.array_equal(a.species, b.species) and
            np.array_equal(a.rel, b.rel) and np.array_equal(a.radii, b.radii))


@pytest.mark.parametrize("d", [1, 2, 3, 4])
def test_snapshot_layout_and_round_trip(d):
    s = sample(d)
    data = raw(s)
    assert len(data) == 36 + 8 * d * d + 3 * (20 + 8 * d)
    assert s.to_bytes() == data
    assert same(mspb.Snapshot.from_bytes(data), s)


def test_empty_snapshots():
    s = mspb.Snapshot.create(np.eye(2) * 2.0, np.zeros((0, 2)), species_count=0)
    assert mspb.Snapshot.from_bytes(s.to_bytes()).N == 0
    s = mspb.Snapshot.create(np.eye(3), np.zeros((0, 3)), species_count=5)
    back = mspb.Snapshot.from_bytes(s.to_bytes())
    assert back.N == 0 and back.species_count == 5


def patched(data, off, fmt, value):
    b = bytearray(data)
    struct.pack_into(fmt, b, off, value)
    return bytes(b)


def test_reader_rejects_malformed_payloads():
    s = sample(3)
    data = raw(s)
    rec0 = 36 + 8 * 9
    bad = {
        "signature": b"MSPX" + data[4:],
        "version": patched(data, 8, "<I", 2),
        "flags": patched(data, 32, "<I", 1),
        "dimension 0": patched(data, 12, "<I", 0),
        "dimension 5": patched(data, 12, "<I", 5),
        "count": patched(data, 16, "<Q", 4),
        "truncated": data[:-1],
        "trailing": data + b"\0",
        "short header": data[:20],
        "label": patched(data, rec0 + 8, "<I", 4),
        "duplicate id": patched(data, rec0 + (20 + 24), "<Q", 7),
        "radius 0": patched(data, rec0 + 20 + 24 - 8, "<d", 0.0),
        "radius nan": patched(data, rec0 + 20 + 24 - 8, "<d", float("nan")),
        "coordinate inf": patched(data, rec0 + 12, "<d", float("inf")),
        "basis nan": patched(data, 36, "<d", float("nan")),
        "singular basis": patched(patched(patched(data, 36 + 48, "<d", 0.0), 36 + 56, "<d", 0.0), 36 + 64, "<d", 0.0),
    }
    for name, b in bad.items():
        with pytest.raises(mspb.MSPBError):
            mspb.Snapshot.from_bytes(b)
        assert name


def test_writer_rejects_invalid_snapshots():
    s = sample(2)
    for change in (lambda t: setattr(t, "species_count", 2), lambda t: t.ids.__setitem__(1, 7),
                   lambda t: t.radii.__setitem__(0, -1.0), lambda t: t.rel.__setitem__((0, 0), np.nan),
                   lambda t: setattr(t, "basis", np.array([[1.0, 2.0], [2.0, 4.0]]))):
        t = mspb.Snapshot(s.basis.copy(), s.ids.copy(), s.species.copy(), s.rel.copy(), s.radii.copy(),
                          s.species_count)
        change(t)
        with pytest.raises(mspb.MSPBError):
            t.to_bytes()


def test_pack_append_reopen_export_clear(tmp_path):
    prefix = str(tmp_path / "ensemble")
    pack = mspb.Pack(prefix)
    assert len(pack) == 0 and not os.path.exists(prefix + ".MSPBPack")   # a missing archive is empty, not created
    a, b = sample(2), sample(3)
    pack.add(a)
    f = tmp_path / "b.mspb"
    mspb.write(f, b)
    pack.import_file(f)
    archive = b"MSPP\r\n\x1a\n" + struct.pack("<II", 1, 0)
    for s in (a, b):
        archive += struct.pack("<Q", len(raw(s))) + raw(s)
    assert open(prefix + ".MSPBPack", "rb").read() == archive
    again = mspb.Pack(prefix)
    assert len(again) == 2 and same(again.get(0), a) and same(again.get(1), b)
    out = tmp_path / "copy.mspb"
    again.export_file(1, out)
    assert open(out, "rb").read() == raw(b)
    with pytest.raises(FileExistsError):
        again.export_file(0, out)
    with pytest.raises(IndexError):
        again.get(2)
    pack.add(a)                      # another handle appends: `again` is stale
    with pytest.raises(mspb.MSPBError):
        again.get(0)
    again.open(prefix)
    assert len(again) == 3
    again.clear()
    assert len(again) == 0 and open(prefix + ".MSPBPack", "rb").read() == archive[:16]


def test_pack_rejects_malformed_archives(tmp_path):
    prefix = str(tmp_path / "bad")
    good = b"MSPP\r\n\x1a\n" + struct.pack("<II", 1, 0) + struct.pack("<Q", len(raw(sample(2)))) + raw(sample(2))
    for data in (good[:-1], good + b"\0" * 4, b"MSPX" + good[4:], good[:8] + struct.pack("<II", 2, 0) + good[16:],
                 good[:16] + struct.pack("<Q", 35) + good[24:]):
        open(prefix + ".MSPBPack", "wb").write(data)
        with pytest.raises(mspb.MSPBError):
            mspb.Pack(prefix)


@needs_ref
@pytest.mark.parametrize("d", [2, 3])
def test_files_cross_with_the_reference(tmp_path, d):
    s = sample(d)
    ours, theirs = tmp_path / "ours.mspb", tmp_path / "theirs.mspb"
    mspb.write(ours, s)
    r = oracle.ref_mspb_read(ours)                       # the reference reads ours
    assert same(mspb.Snapshot(r["basis"], r["ids"], r["species"], r["rel"], r["radii"], r["species_count"]), s)
    oracle.ref_mspb_write(theirs, s.basis, s.ids, s.species, s.rel, s.radii, s.species_count)
    assert open(theirs, "rb").read() == open(ours, "rb").read()   # both write the same bytes
    assert same(mspb.read(theirs), s)                    # and we read theirs
    bad = tmp_path / "bad.mspb"
    open(bad, "wb").write(raw(s) + b"\0")
    with pytest.raises(oracle.RefMSPBError):
        oracle.ref_mspb_read(bad)                        # the reference also rejects trailing data


@needs_ref
def test_archives_cross_with_the_reference(tmp_path):
    a, b = sample(2), sample(3)
    fa, fb = tmp_path / "a.mspb", tmp_path / "b.mspb"
    mspb.write(fa, a)
    mspb.write(fb, b)
    ref_prefix, our_prefix = str(tmp_path / "theirs"), str(tmp_path / "ours")
    oracle.ref_mspbpack_import(ref_prefix, fa)
    oracle.ref_mspbpack_import(ref_prefix, fb)
    ours = mspb.Pack(our_prefix)
    ours.import_file(fa)
    ours.import_file(fb)
    assert open(ref_prefix + ".MSPBPack", "rb").read() == open(our_prefix + ".MSPBPack", "rb").read()
    assert oracle.ref_mspbpack_count(our_prefix) == 2
    oracle.ref_mspbpack_export(our_prefix, 1, tmp_path / "from_ours.mspb")
    assert same(mspb.read(tmp_path / "from_ours.mspb"), b)
    theirs = mspb.Pack(ref_prefix)
    assert len(theirs) == 2 and same(theirs.get(0), a)
