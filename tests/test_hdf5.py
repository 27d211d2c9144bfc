"""The snapshot file format (spk_h5_write / spk_h5_read, the files of
spk_write_snapshot and spk_read_snapshot) checked byte by byte against the
HDF5 File Format Specification, on CPU.

No HDF5 library is installed here, so this file carries its own reader and
writer of the format, written from the specification independently of the
library's C++ (spooky-git_b200/csrc/spk_hdf5.hpp):
  * every file the library writes is walked field by field -- superblock
    version 0, the root group's symbol-table entry and object header, the
    local heap, the version-1 group B-tree, the symbol-table nodes (names in
    strcmp order, keys bracketing them), each dataset's version-1 object
    header (dataspace, datatype, layout messages) and its raw data;
  * files in the forms that libhdf5 / h5py produce and the library does not
    (a two-level B-tree, symbol-table nodes of K = 4, fill-value, NIL and
    modification-time messages, a continuation chunk, compact storage,
    big-endian and 64-bit integer data) are written here and must be read
    by the library.
The reference's snapshot layout (src/io/hdf5_io.cu:19-111): f8 t_start,
t_save, t_lastsnap, t_lastvar and i4 step of one element, and one f8
dataset of NX*NY*NZ values per field.
"""
import ctypes
import struct

import numpy as np
import pytest

import spooky_b200 as S

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


class H5Dataset(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("type", ctypes.c_int), ("n", ctypes.c_size_t),
                ("data", ctypes.c_void_p)]


def lib():
    L = S.lib()
    L.spk_h5_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(H5Dataset), ctypes.c_int]
    L.spk_h5_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(H5Dataset), ctypes.c_int]
    return L


def h5_write(path, items):
    """items: {name: numpy array (float64 or int32)} through spk_h5_write."""
    keep = []
    arr = (H5Dataset * len(items))()
    for i, (name, a) in enumerate(items.items()):
        a = np.ascontiguousarray(a)
        keep.append(a)
        arr[i] = H5Dataset(name.encode(), 0 if a.dtype == np.float64 else 1, a.size, a.ctypes.data)
    rc = lib().spk_h5_write(str(path).encode(), arr, len(items))
    if rc:
        raise S.SpookyError(rc, lib().spk_last_error(None).decode())


def h5_read(path, spec):
    """spec: {name: (dtype, n)} through spk_h5_read."""
    out = {k: np.zeros(n, dtype=dt) for k, (dt, n) in spec.items()}
    arr = (H5Dataset * len(spec))()
    for i, (name, a) in enumerate(out.items()):
        arr[i] = H5Dataset(name.encode(), 0 if a.dtype == np.float64 else 1, a.size, a.ctypes.data)
    rc = lib().spk_h5_read(str(path).encode(), arr, len(spec))
    if rc:
        raise S.SpookyError(rc, lib().spk_last_error(None).decode())
    return out


# ---- an independent reader that checks the structure as it goes ---------------
class SpecWalk:
    def __init__(self, data):
        self.d = data
        self.log = []

    def u(self, at, n):
        return int.from_bytes(self.d[at:at + n], "little")

    def superblock(self):
        d = self.d
        assert d[:8] == SIG
        assert d[8] == 0, "superblock version 0"
        assert d[9] == 0 and d[10] == 0 and d[11] == 0 and d[12] == 0   # free-space, root entry, reserved, shared
        assert d[13] == 8 and d[14] == 8 and d[15] == 0                 # offsets, lengths, reserved
        self.leaf_k, self.internal_k = self.u(16, 2), self.u(18, 2)
        assert self.leaf_k > 0 and self.internal_k > 0
        assert self.u(20, 4) == 0                                      # consistency flags
        assert self.u(24, 8) == 0                                      # base address
        assert self.u(32, 8) == UNDEF                                  # free-space info
        assert self.u(40, 8) == len(d), "end-of-file address equals the file size"
        assert self.u(48, 8) == UNDEF                                  # driver information block
        # root group symbol table entry
        assert self.u(56, 8) == 0
        self.root_oh = self.u(64, 8)
        assert self.u(72, 4) == 1, "root entry caches its symbol table"
        self.btree, self.heap = self.u(80, 8), self.u(88, 8)

    def object_header(self, at):
        """Messages of a version-1 object header: [(type, flags, data bytes)]."""
        d = self.d
        assert at % 8 == 0
        assert d[at] == 1 and d[at + 1] == 0
        nmsg, refc, size = self.u(at + 2, 2), self.u(at + 4, 4), self.u(at + 8, 4)
        assert refc == 1 and self.u(at + 12, 4) == 0 and size % 8 == 0
        msgs, p = [], at + 16
        while p < at + 16 + size:
            t, n, fl = self.u(p, 2), self.u(p + 2, 2), d[p + 4]
            assert n % 8 == 0 and d[p + 5:p + 8] == b"\0\0\0"
            msgs.append((t, fl, d[p + 8:p + 8 + n]))
            p += 8 + n
        assert p == at + 16 + size and len(msgs) == nmsg
        return msgs

    def walk(self):
        self.superblock()
        (t, _, body), = self.object_header(self.root_oh)
        assert t == 0x0011
        assert struct.unpack("<QQ", body[:16]) == (self.btree, self.heap)
        d = self.d
        h = self.heap
        assert d[h:h + 4] == b"HEAP" and d[h + 4] == 0 and d[h + 5:h + 8] == b"\0\0\0"
        hsize, free, hdata = self.u(h + 8, 8), self.u(h + 16, 8), self.u(h + 24, 8)
        assert free == 1, "no free block: libhdf5's on-disk end of the free list"
        assert d[hdata:hdata + 8] == b"\0" * 8, "the empty name at heap offset 0"
        assert hsize % 8 == 0 and hdata + hsize <= len(d)

        def name(off):
            end = d.index(b"\0", hdata + off)
            return d[hdata + off:end].decode()

        b = self.btree
        assert d[b:b + 4] == b"TREE" and d[b + 4] == 0 and d[b + 5] == 0
        used = self.u(b + 6, 2)
        assert self.u(b + 8, 8) == UNDEF and self.u(b + 16, 8) == UNDEF
        assert 1 <= used <= 2 * self.internal_k
        entries = []
        key = name(self.u(b + 24, 8))
        assert key == ""
        for c in range(used):
            child = self.u(b + 32 + 16 * c, 8)
            right = name(self.u(b + 40 + 16 * c, 8))
            assert d[child:child + 4] == b"SNOD" and d[child + 4] == 1 and d[child + 5] == 0
            n = self.u(child + 6, 2)
            assert 1 <= n <= 2 * self.leaf_k
            names = []
            for e in range(n):
                at = child + 8 + 40 * e
                nm = name(self.u(at, 8))
                assert self.u(at + 16, 4) == 0 and d[at + 24:at + 40] == b"\0" * 16
                names.append(nm)
                entries.append((nm, self.u(at + 8, 8)))
            assert names == sorted(names, key=lambda s: s.encode())
            assert key.encode() < names[0].encode() and names[-1] == right
            key = right
        self.entries = dict(entries)
        assert list(self.entries) == sorted(self.entries, key=lambda s: s.encode())
        return self.entries

    def dataset(self, nm):
        msgs = {t: body for t, _, body in self.object_header(self.entries[nm])}
        assert set(msgs) == {0x0001, 0x0003, 0x0008}
        sp = msgs[0x0001]
        assert sp[0] == 1 and sp[1] == 1 and sp[2] == 0 and sp[3] == 0 and sp[4:8] == b"\0" * 4
        n = struct.unpack("<Q", sp[8:16])[0]
        ty = msgs[0x0003]
        size = struct.unpack("<I", ty[4:8])[0]
        if ty[0] == 0x11:
            assert ty[1:4] == bytes([0x20, 63, 0]) and size == 8
            assert struct.unpack("<HHBBBBI", ty[8:20]) == (0, 64, 52, 11, 0, 52, 1023)
            dt = "<f8"
        else:
            assert ty[0] == 0x10 and ty[1:4] == bytes([0x08, 0, 0]) and size == 4
            assert struct.unpack("<HH", ty[8:12]) == (0, 32)
            dt = "<i4"
        lay = msgs[0x0008]
        assert lay[0] == 3 and lay[1] == 1
        addr, nbytes = struct.unpack("<QQ", lay[2:18])
        assert nbytes == n * size and addr % 8 == 0 and addr + nbytes <= len(self.d)
        return np.frombuffer(self.d[addr:addr + nbytes], dtype=dt)


def snapshot_items(nr=4 * 3 * 2, fields=("vx", "vy", "vz", "bx", "by", "bz"), seed=0):
    rng = np.random.default_rng(seed)
    items = {"t_start": np.array([0.0]), "t_save": np.array([1.25]), "t_lastsnap": np.array([1.2]),
             "t_lastvar": np.array([1.0]), "step": np.array([37], dtype=np.int32)}
    for f in fields:
        items[f] = rng.standard_normal(nr)
    return items


def test_snapshot_file_layout_follows_the_specification(tmp_path):
    path = tmp_path / "snap0003.h5"
    items = snapshot_items()
    h5_write(path, items)
    w = SpecWalk(path.read_bytes())
    ents = w.walk()
    assert sorted(ents) == sorted(items)
    for k, v in items.items():
        got = w.dataset(k)
        assert got.dtype.kind == v.dtype.kind and np.array_equal(got, v)
    back = h5_read(path, {k: (v.dtype, v.size) for k, v in items.items()})
    for k, v in items.items():
        assert np.array_equal(back[k], v)


@pytest.mark.parametrize("nds", [1, 16, 17, 40])
def test_many_datasets_span_symbol_table_nodes(tmp_path, nds):
    path = tmp_path / "many.h5"
    rng = np.random.default_rng(nds)
    items = {f"d{i:03d}_{'x' * (i % 5)}": rng.standard_normal(1 + i) for i in range(nds)}
    h5_write(path, items)
    w = SpecWalk(path.read_bytes())
    assert sorted(w.walk()) == sorted(items)
    for k, v in items.items():
        assert np.array_equal(w.dataset(k), v)
    back = h5_read(path, {k: (np.float64, v.size) for k, v in items.items()})
    assert all(np.array_equal(back[k], v) for k, v in items.items())


def test_reading_converts_types_and_checks_sizes(tmp_path):
    path = tmp_path / "t.h5"
    h5_write(path, {"step": np.array([123456], dtype=np.int32), "x": np.array([1.5, -2.0])})
    assert h5_read(path, {"step": (np.float64, 1)})["step"][0] == 123456.0
    assert h5_read(path, {"x": (np.int32, 2)})["x"].tolist() == [1, -2]
    with pytest.raises(S.SpookyError, match="elements"):
        h5_read(path, {"x": (np.float64, 3)})
    with pytest.raises(S.SpookyError, match="no dataset"):
        h5_read(path, {"y": (np.float64, 2)})
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file" * 8)
    with pytest.raises(S.SpookyError, match="signature"):
        h5_read(bad, {"x": (np.float64, 2)})
    with pytest.raises(S.SpookyError, match="repeated"):
        lib_items = {"a": np.zeros(1)}
        arr = (H5Dataset * 2)(H5Dataset(b"a", 0, 1, lib_items["a"].ctypes.data),
                              H5Dataset(b"a", 0, 1, lib_items["a"].ctypes.data))
        rc = lib().spk_h5_write(str(tmp_path / "r.h5").encode(), arr, 2)
        raise S.SpookyError(rc, lib().spk_last_error(None).decode())


# ---- files in the forms libhdf5 and h5py write ----------------------------------
class SpecWriter:
    """Writes the original format with the variations libhdf5 produces:
    symbol-table nodes of K = 4 under a two-level B-tree, fill-value (0x0005),
    modification-time (0x0012) and NIL messages, a continuation chunk,
    compact storage and big-endian / 64-bit integer data."""

    def __init__(self):
        self.b = bytearray(b"\0" * 96)

    def alloc(self, blob):
        while len(self.b) % 8:
            self.b.append(0)
        at = len(self.b)
        self.b += blob
        return at

    @staticmethod
    def msg(t, body, flags=0):
        body = bytes(body)
        body += b"\0" * (-len(body) % 8)
        return struct.pack("<HHB3x", t, len(body), flags) + body

    def ohdr(self, msgs, extra_chunk=None):
        chunk = b"".join(msgs)
        n = len(msgs)
        if extra_chunk is not None:
            at = self.alloc(b"".join(extra_chunk))
            chunk += self.msg(0x0010, struct.pack("<QQ", at, len(b"".join(extra_chunk))))
            n += 1 + len(extra_chunk)
        return self.alloc(struct.pack("<BBHII4x", 1, 0, n, 1, len(chunk)) + chunk)

    @staticmethod
    def space(n):
        return struct.pack("<BBBB4xQQ", 1, 1, 1, 0, n, n)   # with maximum dims

    @staticmethod
    def f8type(big=False):
        return struct.pack("<BBBBI", 0x11, 0x21 if big else 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)

    @staticmethod
    def i8type():
        return struct.pack("<BBBBI", 0x10, 0x08, 0, 0, 8) + struct.pack("<HH", 0, 64)

    def dataset(self, kind, values):
        fill = self.msg(0x0005, struct.pack("<BBBB", 2, 2, 2, 0))
        mtime = self.msg(0x0012, struct.pack("<B3xI", 1, 1700000000))
        nil = self.msg(0x0000, b"\0" * 8)
        n = len(values)
        if kind == "be_f8":
            data = self.alloc(np.asarray(values, ">f8").tobytes())
            lay = self.msg(0x0008, struct.pack("<BBQQ", 3, 1, data, 8 * n))
            return self.ohdr([self.msg(0x0001, self.space(n)), self.msg(0x0003, self.f8type(True)), fill, lay, mtime])
        if kind == "compact_f8":
            raw = np.asarray(values, "<f8").tobytes()
            lay = self.msg(0x0008, struct.pack("<BBH", 3, 0, len(raw)) + raw)
            return self.ohdr([self.msg(0x0001, self.space(n)), self.msg(0x0003, self.f8type()), fill, lay, nil])
        if kind == "i8_cont":
            data = self.alloc(np.asarray(values, "<i8").tobytes())
            lay = self.msg(0x0008, struct.pack("<BBQQ", 3, 1, data, 8 * n))
            return self.ohdr([self.msg(0x0001, self.space(n)), fill],
                             extra_chunk=[self.msg(0x0003, self.i8type()), lay, mtime])
        raise ValueError(kind)

    def finish(self, items, leaf_k=4, internal_k=16):
        names = sorted(items, key=lambda s: s.encode())
        heap = bytearray(b"\0" * 8)
        off = {}
        for nm in names:
            off[nm] = len(heap)
            heap += nm.encode() + b"\0"
            heap += b"\0" * (-len(heap) % 8)
        ohs = {nm: self.dataset(kind, vals) for nm, (kind, vals) in items.items()}
        hdata = self.alloc(bytes(heap))
        heap_at = self.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), 1, hdata))
        per = 2 * leaf_k
        groups = [names[i:i + per] for i in range(0, len(names), per)]
        snods = []
        for g in groups:
            ents = b"".join(struct.pack("<QQI4x16x", off[nm], ohs[nm], 0) for nm in g)
            snods.append(self.alloc(b"SNOD" + struct.pack("<BBH", 1, 0, len(g)) + ents + b"\0" * (40 * (per - len(g)))))

        def tree(level, children, keys):
            body = b"TREE" + struct.pack("<BBHQQ", 0, level, len(children), UNDEF, UNDEF)
            body += struct.pack("<Q", keys[0])
            for ch, k in zip(children, keys[1:]):
                body += struct.pack("<QQ", ch, k)
            body += b"\0" * (16 * (2 * internal_k - len(children)))
            return self.alloc(body)

        # two leaf-level B-tree nodes under one level-1 root
        half = (len(snods) + 1) // 2
        leaves, lkeys = [], [0]
        for part in (range(0, half), range(half, len(snods))):
            ks = [0 if not leaves else lkeys[-1]] + [off[groups[i][-1]] for i in part]
            leaves.append(tree(0, [snods[i] for i in part], ks))
            lkeys.append(ks[-1])
        root_tree = tree(1, leaves, lkeys)
        root_oh = self.ohdr([self.msg(0x0011, struct.pack("<QQ", root_tree, heap_at))])
        sb = SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", leaf_k, internal_k, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, len(self.b), UNDEF)
        sb += struct.pack("<QQII16x", 0, root_oh, 0, 0)      # no cached symbol table: read the header
        self.b[:96] = sb
        return bytes(self.b)


def test_library_reads_the_forms_libhdf5_writes(tmp_path):
    rng = np.random.default_rng(5)
    items = {}
    for i in range(11):
        items[f"be{i}"] = ("be_f8", rng.standard_normal(3 + i))
    items["t_save"] = ("compact_f8", [2.5])
    items["step"] = ("i8_cont", [-77])
    items["wide"] = ("i8_cont", [1, 2, 3])
    blob = SpecWriter().finish(items)
    path = tmp_path / "h5py_like.h5"
    path.write_bytes(blob)
    spec = {k: (np.float64, len(v)) for k, (_, v) in items.items()}
    got = h5_read(path, spec)
    for k, (_, v) in items.items():
        assert np.array_equal(got[k], np.asarray(v, dtype=np.float64)), k
    assert h5_read(path, {"step": (np.int32, 1)})["step"][0] == -77
