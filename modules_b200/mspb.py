"""MSPB v1 snapshots and MSPBPack archives: the configuration files of the reference's multi-species optimiser.

The formats are those of apps/CCOptimization/EXPORT_FORMAT.md and MSPB_PACK.md (MultiStealthyPotential::
ExportConfiguration and MSPB_Pack, apps/CCOptimization/MSPB_Pack.cpp:70-288). They carry a cell, particle IDs, species
labels, relative coordinates and radii, which is what `CCMulti.set_snapshot` needs to evaluate a stored configuration
on the GPU, and what a run's results are written back as for the reference's tools. Host code only.

Snapshot (all integers unsigned little-endian, all reals IEEE binary64 little-endian, no padding):
    signature b"MSPB\\r\\n\\x1a\\n", uint32 version = 1, uint32 D, uint64 N, uint64 declared species count,
    uint32 flags = 3 (relative coordinates, Cartesian radii), D x D basis (vector 0's components first), then N
    records of uint64 ID, uint32 species label, D relative coordinates and the radius: 36 + 8 D^2 + N (20 + 8 D) bytes.
Archive <prefix>.MSPBPack: signature b"MSPP\\r\\n\\x1a\\n", uint32 version = 1, uint32 flags = 0, then per snapshot
    a uint64 payload length and the snapshot's bytes.

Readers reject what the reference rejects: other versions or flags, D outside 1..4, a byte count that does not match
N (truncated or trailing data), a singular or non-finite cell, non-finite coordinates, non-positive or non-finite
radii, labels outside the declared species count and repeated IDs.
"""
import os
import struct
from dataclasses import dataclass

import numpy as np

MAGIC = b"MSPB\r\n\x1a\n"
PACK_MAGIC = b"MSPP\r\n\x1a\n"
MAX_DIMENSION = 4   # the reference core's MaxDimension
_HEADER = struct.Struct("<8sIIQQI")   # 36 bytes


class MSPBError(ValueError):
    """A malformed or invalid MSPB snapshot or archive."""


def _record_dtype(d):
    return np.dtype([("id", "<u8"), ("species", "<u4"), ("rel", "<f8", (d,)), ("radius", "<f8")])


def _check_basis(basis):
    """Partial-pivoting elimination, as the reference's MSPBSnapshot::Validate: a zero or non-finite pivot is a
    singular cell."""
    m = np.array(basis, dtype=np.float64)
    d = m.shape[0]
    for k in range(d):
        piv = k + int(np.argmax(np.abs(m[k:, k])))
        if m[piv, k] == 0.0 or not np.isfinite(m[piv, k]):
            raise MSPBError("MSPB: singular basis")
        m[[k, piv]] = m[[piv, k]]
        for r in range(k + 1, d):
            m[r, k + 1:] -= (m[r, k] / m[k, k]) * m[k, k + 1:]


@dataclass
class Snapshot:
    """One configuration: basis (d x d, rows are the cell vectors in Cartesian coordinates), ids (N, uint64), species
    (N, uint32 labels below species_count), rel (N x d relative coordinates), radii (N, Cartesian), species_count
    (declared species, empty ones included)."""
    basis: np.ndarray
    ids: np.ndarray
    species: np.ndarray
    rel: np.ndarray
    radii: np.ndarray
    species_count: int

    @property
    def d(self):
        return int(self.basis.shape[0])

    @property
    def N(self):
        return int(self.ids.shape[0])

    @classmethod
    def create(cls, basis, rel, species=None, radii=None, ids=None, species_count=None):
        """A snapshot from arrays: ids default to 0..N-1, species to 0, radii to 0.5, species_count to the largest
        label + 1."""
        basis = np.ascontiguousarray(basis, dtype=np.float64)
        d = basis.shape[0]
        rel = np.ascontiguousarray(rel, dtype=np.float64).reshape(-1, d)
        n = rel.shape[0]
        ids = np.arange(n, dtype=np.uint64) if ids is None else np.ascontiguousarray(ids, dtype=np.uint64)
        species = np.zeros(n, np.uint32) if species is None else np.ascontiguousarray(species, dtype=np.uint32)
        radii = np.full(n, 0.5) if radii is None else np.ascontiguousarray(radii, dtype=np.float64)
        if species_count is None:
            species_count = int(species.max()) + 1 if n else 0
        s = cls(basis, ids, species, rel, radii, int(species_count))
        s.validate()
        return s

    def validate(self):
        d = self.basis.shape[0] if self.basis.ndim == 2 else 0
        if self.basis.ndim != 2 or self.basis.shape != (d, d) or not 1 <= d <= MAX_DIMENSION:
            raise MSPBError("MSPB: unsupported dimension")
        if not np.all(np.isfinite(self.basis)):
            raise MSPBError("MSPB: nonfinite basis")
        _check_basis(self.basis)
        n = self.ids.shape[0]
        if self.species.shape != (n,) or self.rel.shape != (n, d) or self.radii.shape != (n,):
            raise MSPBError("MSPB: inconsistent particle arrays")
        if n and int(self.species.max()) >= self.species_count:
            raise MSPBError("MSPB: species label outside declared range")
        if np.unique(self.ids).shape[0] != n:
            raise MSPBError("MSPB: duplicate particle ID")
        if not np.all(np.isfinite(self.radii)) or np.any(self.radii <= 0):
            raise MSPBError("MSPB: invalid radius")
        if not np.all(np.isfinite(self.rel)):
            raise MSPBError("MSPB: nonfinite coordinate")
        if not 0 <= self.species_count < 1 << 64:
            raise MSPBError("MSPB: invalid species count")

    def to_bytes(self):
        """The snapshot's MSPB v1 bytes (validated first, as the reference's writer)."""
        self.validate()
        d, n = self.d, self.N
        rec = np.empty(n, _record_dtype(d))
        rec["id"], rec["species"], rec["rel"], rec["radius"] = self.ids, self.species, self.rel, self.radii
        return (_HEADER.pack(MAGIC, 1, d, n, self.species_count, 3) + self.basis.astype("<f8").tobytes() +
                rec.tobytes())

    @classmethod
    def from_bytes(cls, data):
        """Parse exactly one MSPB v1 snapshot (no trailing bytes)."""
        data = bytes(data)
        if len(data) < _HEADER.size:
            raise MSPBError("MSPB: truncated input")
        magic, version, d, n, nspecies, flags = _HEADER.unpack_from(data, 0)
        if magic != MAGIC:
            raise MSPBError("MSPB: invalid signature")
        if version != 1:
            raise MSPBError("MSPB: unsupported snapshot version")
        if flags != 3:
            raise MSPBError("MSPB: unsupported snapshot flags")
        if not 1 <= d <= MAX_DIMENSION:
            raise MSPBError("MSPB: unsupported dimension")
        rest = len(data) - _HEADER.size
        basis_bytes, rec_bytes = 8 * d * d, 20 + 8 * d
        if rest < basis_bytes or (rest - basis_bytes) % rec_bytes or n != (rest - basis_bytes) // rec_bytes:
            raise MSPBError("MSPB: particle count does not match file size")
        basis = np.frombuffer(data, "<f8", d * d, _HEADER.size).reshape(d, d).astype(np.float64)
        rec = np.frombuffer(data, _record_dtype(d), n, _HEADER.size + basis_bytes)
        s = cls(basis, rec["id"].astype(np.uint64), rec["species"].astype(np.uint32), rec["rel"].astype(np.float64),
                rec["radius"].astype(np.float64), int(nspecies))
        s.validate()
        return s


def read(path):
    """Read one .mspb file."""
    with open(path, "rb") as f:
        return Snapshot.from_bytes(f.read())


def write(path, snapshot, overwrite=True):
    """Write one .mspb file (refusing an existing file when overwrite is False)."""
    data = snapshot.to_bytes()
    with open(path, "wb" if overwrite else "xb") as f:
        f.write(data)


class Pack:
    """An MSPBPack archive <prefix>.MSPBPack: append-only, one writer, records read by index. Opening scans the framing
    into an offset index; a record is validated when it is read. A missing file is an empty archive that the first
    append creates. A handle whose file changed size since it last read or wrote refuses to work until reopened."""

    def __init__(self, prefix):
        self.open(prefix)

    def open(self, prefix):
        if not prefix:
            raise ValueError("MSPB_Pack: empty prefix")
        path = prefix + ".MSPBPack"
        entries, size = [], 0
        if os.path.exists(path):
            with open(path, "rb") as f:
                data = f.read()
            size = len(data)
            if size < 16 or data[:8] != PACK_MAGIC:
                raise MSPBError("MSPB: invalid signature")
            version, flags = struct.unpack_from("<II", data, 8)
            if version != 1 or flags != 0:
                raise MSPBError("MSPB: unsupported archive version/flags")
            off = 16
            while off < size:
                if size - off < 8:
                    raise MSPBError("MSPB: incomplete archive frame")
                (length,) = struct.unpack_from("<Q", data, off)
                off += 8
                if length < 36 or length > size - off:
                    raise MSPBError("MSPB: invalid archive frame length")
                entries.append((off, length))
                off += length
        self.filename, self._entries, self._size = path, entries, size

    def __len__(self):
        return len(self._entries)

    def num_config(self):
        return len(self._entries)

    def _check_current(self):
        exists = os.path.exists(self.filename)
        if (not exists and self._size) or (exists and (self._size == 0 or os.path.getsize(self.filename) != self._size)):
            raise MSPBError("MSPB: archive changed; reopen before use")

    def _payload(self, index):
        self._check_current()
        if not 0 <= index < len(self._entries):
            raise IndexError("MSPB_Pack: index out of range")
        off, length = self._entries[index]
        with open(self.filename, "rb") as f:
            f.seek(off)
            data = f.read(length)
        if len(data) != length:
            raise MSPBError("MSPB: truncated input")
        return data

    def get(self, index):
        """Snapshot `index` (zero-based)."""
        return Snapshot.from_bytes(self._payload(index))

    def add(self, snapshot):
        """Append a snapshot (validated first; nothing is written for an invalid one)."""
        self._append(snapshot.to_bytes())

    def _append(self, payload):
        self._check_current()
        base = self._size if self._size else 16
        head = b"" if self._size else PACK_MAGIC + struct.pack("<II", 1, 0)
        try:
            with open(self.filename, "ab") as f:
                f.write(head + struct.pack("<Q", len(payload)) + payload)
        except OSError:
            if self._size:
                os.truncate(self.filename, self._size)
            elif os.path.exists(self.filename):
                os.remove(self.filename)
            raise
        self._entries.append((base + 8, len(payload)))
        self._size = base + 8 + len(payload)

    def import_file(self, path):
        """Append the snapshot of one .mspb file (validated; its bytes are stored as they are)."""
        with open(path, "rb") as f:
            data = f.read()
        Snapshot.from_bytes(data)
        self._append(data)

    def export_file(self, index, path):
        """Write snapshot `index` to a new .mspb file (an existing file is an error); the bytes are the stored ones."""
        s = self.get(index)
        write(path, s, overwrite=False)

    def clear(self):
        """Discard every record, leaving a valid empty archive."""
        self._check_current()
        with open(self.filename, "wb") as f:
            f.write(PACK_MAGIC + struct.pack("<II", 1, 0))
        self._entries, self._size = [], 16
