"""HDF5 files of the reference's output and restart layout, without libhdf5.

The reference writes every output file through its storage class (src/headers/storage.h:54-230,
H5Cpp with default properties): one flat root group of 1-D datasets, IEEE F64LE or STD_I32LE,
each with two scalar fixed-length string attributes, "Variable" (the description) and "units".
This module writes and reads exactly that shape, restating the parts of the HDF5 file format
(The HDF Group, "HDF5 File Format Specification", version 0 superblock) that such files use:

  superblock v0 (sizes of offsets and lengths 8, group leaf K 4, internal K 16), whose root
    symbol-table entry caches the root group's B-tree and local heap;
  the root group: an object header v1 holding a symbol-table message, a v1 B-tree of type 0
    (group nodes) whose children are symbol-table nodes ("SNOD", up to 2 x leaf K entries, names
    in strcmp order), and a local heap ("HEAP") holding the link names, 8-byte aligned;
  each dataset: an object header v1 with the messages dataspace (v1, simple, one dimension with
    its maximum), datatype (v1; IEEE double or signed 32-bit integer), fill value (v2), data
    layout (v3, contiguous), modification time (v1) and two attribute messages (v1), in that
    order, as the library writes them; the data follow as one contiguous block.

The reader takes what the library writes for these files (it is checked on files the reference
wrote, tests/golden/h5/): v0 superblocks, symbol-table groups (B-trees of any depth), object
headers v1 with continuation messages, dataspace v1/v2, fixed-point, floating-point and string
datatypes, contiguous and compact layouts, attribute messages v1-v3.
"""
import struct
import time

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
LEAF_K, INTERNAL_K = 4, 16          # the library's defaults (group leaf / internal node K)
SNOD_CAP = 2 * LEAF_K               # entries per symbol-table node
BTREE_CAP = 2 * INTERNAL_K          # children per B-tree node
HEAP_FREE_NULL = 1                  # end of a local heap's free list

# message types
MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL, MSG_LAYOUT = 0x0, 0x1, 0x3, 0x5, 0x8
MSG_ATTRIBUTE, MSG_CONTINUATION, MSG_SYMTAB, MSG_MTIME = 0xC, 0x10, 0x11, 0x12

# datatype messages (v1) of the two numeric types storage.h writes
DT_F64LE = bytes([0x11, 0x20, 0x3F, 0x00]) + struct.pack("<IHHBBBBI", 8, 0, 64, 52, 11, 0, 52, 1023)
DT_I32LE = bytes([0x10, 0x08, 0x00, 0x00]) + struct.pack("<IHH", 4, 0, 32)


class H5FormatError(Exception):
    pass


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _message(mtype, body, flags=0):
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _string_type(n):
    """Fixed-length ASCII string, null-terminated padding (H5T_C_S1 of size n)."""
    return bytes([0x13, 0x00, 0x00, 0x00]) + struct.pack("<I", n)


SCALAR_SPACE = bytes([1, 0, 0, 0, 0, 0, 0, 0])     # dataspace v1, rank 0


def _attribute(name, text):
    """Attribute message v1: a scalar fixed-length string."""
    data = text.encode("ascii")
    if not data:                     # a zero-size string type is not allowed: one null byte
        data = b"\0"
    nm = name.encode("ascii") + b"\0"
    dt = _string_type(len(data))
    head = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(SCALAR_SPACE))
    return _message(MSG_ATTRIBUTE, head + _pad8(nm) + _pad8(dt) + _pad8(SCALAR_SPACE) + data)


class H5Writer:
    """Collects 1-D datasets, then writes the file on close() (storage::append_table /
    append_value)."""

    def __init__(self, path):
        self.path = path
        self.items = {}

    def table(self, name, data, unit, description):
        a = np.asarray(data)
        if a.dtype.kind in "iub":
            a = a.astype("<i4")
        else:
            a = a.astype("<f8")
        self.items[name.lstrip("/")] = (np.ascontiguousarray(a.reshape(-1)), unit, description)

    def value(self, name, v, unit, description):
        is_int = isinstance(v, (int, np.integer)) and not isinstance(v, bool)
        self.table(name, np.array([v], dtype="<i4" if is_int else "<f8"), unit, description)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if exc[0] is None:
            self.close()

    def close(self):
        names = sorted(self.items, key=lambda n: n.encode("ascii"))
        if len(names) > SNOD_CAP * BTREE_CAP:
            raise H5FormatError("more datasets than one B-tree node holds")
        # local heap: the empty name at 0, then every name, 8-byte aligned, then one free block
        heap = bytearray(b"\0" * 8)
        name_off = {}
        for n in names:
            name_off[n] = len(heap)
            heap += _pad8(n.encode("ascii") + b"\0")
        free_off = len(heap)
        heap += struct.pack("<QQ", HEAP_FREE_NULL, 16)
        nsnod = max(1, -(-len(names) // SNOD_CAP))
        snod_size = 8 + SNOD_CAP * 40
        btree_size = 24 + 8 * (2 * INTERNAL_K + 1) + 8 * (2 * INTERNAL_K)
        # addresses: superblock, root object header, B-tree, heap header, heap data, SNODs,
        # then per dataset its object header and its data
        a_root = 96
        a_btree = a_root + 16 + 24
        a_heap = a_btree + btree_size
        a_heapdata = a_heap + 32
        a_snod = a_heapdata + len(heap)
        pos = a_snod + nsnod * snod_size
        now = int(time.time()) & 0xFFFFFFFF
        objects, addr_of = [], {}
        for n in names:
            a, unit, desc = self.items[n]
            msgs = self._dataset_messages(a, unit, desc, now, data_addr=0)
            hdr_size = 16 + len(msgs)
            data_addr = pos + hdr_size
            msgs = self._dataset_messages(a, unit, desc, now, data_addr=data_addr)
            ohdr = struct.pack("<BBHII4x", 1, 0, 7, 1, len(msgs)) + msgs
            addr_of[n] = pos
            objects.append((pos, ohdr, data_addr, a.tobytes()))
            pos = data_addr + len(a.tobytes())
            pos += -pos % 8
        eof = pos
        out = bytearray(eof)
        # superblock v0 with the root group's symbol-table entry (cache type 1: B-tree, heap)
        out[0:8] = SIGNATURE
        out[8:16] = bytes([0, 0, 0, 0, 0, 8, 8, 0])
        out[16:24] = struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
        out[24:56] = struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        out[56:96] = struct.pack("<QQII", 0, a_root, 1, 0) + struct.pack("<QQ", a_btree, a_heap)
        # root object header: one symbol-table message
        root = struct.pack("<BBHII4x", 1, 0, 1, 1, 24) + _message(MSG_SYMTAB,
                                                               struct.pack("<QQ", a_btree, a_heap))
        out[a_root:a_root + len(root)] = root
        # symbol-table nodes and the B-tree over them; key i+1 = the last name of child i
        keys, kids = [0], []
        for k in range(nsnod):
            chunk = names[k * SNOD_CAP:(k + 1) * SNOD_CAP]
            a = a_snod + k * snod_size
            node = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(chunk)))
            for n in chunk:
                node += struct.pack("<QQII", name_off[n], addr_of[n], 0, 0) + b"\0" * 16
            out[a:a + len(node)] = node
            kids.append(a)
            keys.append(name_off[chunk[-1]] if chunk else 0)
        bt = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", len(kids), UNDEF, UNDEF))
        for i, c in enumerate(kids):
            bt += struct.pack("<QQ", keys[i], c)
        bt += struct.pack("<Q", keys[len(kids)])
        out[a_btree:a_btree + len(bt)] = bt
        # local heap header and data
        out[a_heap:a_heap + 32] = b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack(
            "<QQQ", len(heap), free_off, a_heapdata)
        out[a_heapdata:a_heapdata + len(heap)] = heap
        for a, ohdr, data_addr, raw in objects:
            out[a:a + len(ohdr)] = ohdr
            out[data_addr:data_addr + len(raw)] = raw
        with open(self.path, "wb") as f:
            f.write(out)

    @staticmethod
    def _dataset_messages(a, unit, desc, now, data_addr):
        n = a.size
        space = bytes([1, 1, 1, 0, 0, 0, 0, 0]) + struct.pack("<QQ", n, n)
        dtype = DT_I32LE if a.dtype == np.dtype("<i4") else DT_F64LE
        fill = bytes([2, 2, 2, 1, 0, 0, 0, 0])
        layout = bytes([3, 1]) + struct.pack("<QQ", data_addr, a.nbytes)
        mtime = bytes([1, 0, 0, 0]) + struct.pack("<I", now)
        return (_message(MSG_DATASPACE, space) + _message(MSG_DATATYPE, dtype, flags=1)
                + _message(MSG_FILL, fill, flags=1) + _message(MSG_LAYOUT, layout)
                + _message(MSG_MTIME, mtime) + _attribute("Variable", desc)
                + _attribute("units", unit))


# ---------------------------------------------------------------------------------------------
# Reader
# ---------------------------------------------------------------------------------------------
class _File:
    def __init__(self, data):
        self.d = data
        if data[:8] != SIGNATURE:
            raise H5FormatError("not an HDF5 file (signature)")
        if data[8] != 0:
            raise H5FormatError("superblock version %d (only 0 is read)" % data[8])
        if data[13] != 8 or data[14] != 8:
            raise H5FormatError("sizes of offsets/lengths other than 8")
        self.root_ohdr = self.u("Q", 56 + 8)

    def u(self, fmt, off):
        v = struct.unpack_from("<" + fmt, self.d, off)
        return v[0] if len(v) == 1 else v

    def cstr(self, off):
        e = self.d.index(b"\0", off)
        return self.d[off:e].decode("ascii")

    def messages(self, addr):
        """(type, body) of every message of the object header v1 at addr, continuations followed."""
        if self.d[addr] != 1:
            raise H5FormatError("object header version %d (only 1 is read)" % self.d[addr])
        nmsgs, _, size = self.u("HII", addr + 2)
        chunks, out = [(addr + 16, size)], []
        while chunks and len(out) < nmsgs:
            p, size = chunks.pop(0)
            end = p + size
            while p + 8 <= end and len(out) < nmsgs:
                mtype, msize, _ = self.u("HHB", p)
                body = self.d[p + 8:p + 8 + msize]
                if mtype == MSG_CONTINUATION:
                    chunks.append(struct.unpack_from("<QQ", body))
                out.append((mtype, body))
                p += 8 + msize
        return out

    def group_entries(self, btree, heap):
        """{name: object header address} of a symbol-table group."""
        if self.d[heap:heap + 4] != b"HEAP":
            raise H5FormatError("bad local heap")
        heap_data = self.u("Q", heap + 24)
        out = {}

        def walk(node):
            if self.d[node:node + 4] != b"TREE" or self.d[node + 4] != 0:
                raise H5FormatError("bad group B-tree node")
            level, used = self.d[node + 5], self.u("H", node + 6)
            p = node + 24
            for _ in range(used):
                child = self.u("Q", p + 8)
                if level > 0:
                    walk(child)
                else:
                    if self.d[child:child + 4] != b"SNOD":
                        raise H5FormatError("bad symbol-table node")
                    nsym = self.u("H", child + 6)
                    for i in range(nsym):
                        e = child + 8 + 40 * i
                        lno, oh = self.u("QQ", e)
                        out[self.cstr(heap_data + lno)] = oh
                p += 16

        walk(btree)
        return out

    def dtype(self, b):
        cls, ver = b[0] & 0x0F, b[0] >> 4
        size = struct.unpack_from("<I", b, 4)[0]
        if cls == 0:
            order = ">" if b[1] & 1 else "<"
            return np.dtype("%s%s%d" % (order, "i" if b[1] & 8 else "u", size))
        if cls == 1:
            order = ">" if b[1] & 1 else "<"
            return np.dtype("%sf%d" % (order, size))
        if cls == 3:
            return np.dtype("S%d" % size)
        raise H5FormatError("datatype class %d not read" % cls)

    @staticmethod
    def space(b):
        ver, rank, flags = b[0], b[1], b[2]
        if ver == 1:
            return struct.unpack_from("<%dQ" % rank, b, 8) if rank else ()
        if ver == 2:
            if b[3] == 0 or rank == 0:       # scalar (type 0) or rank 0
                return ()
            return struct.unpack_from("<%dQ" % rank, b, 4)
        raise H5FormatError("dataspace version %d" % ver)

    def attribute(self, b):
        ver = b[0]
        if ver == 1:
            nsz, tsz, ssz = struct.unpack_from("<HHH", b, 2)
            p = 8
            name = b[p:p + nsz].split(b"\0")[0].decode("ascii")
            p += nsz + (-nsz % 8)
            dt = self.dtype(b[p:p + tsz])
            p += tsz + (-tsz % 8)
            shape = self.space(b[p:p + ssz])
            p += ssz + (-ssz % 8)
        elif ver in (2, 3):
            nsz, tsz, ssz = struct.unpack_from("<HHH", b, 2)
            p = 8 + (1 if ver == 3 else 0)
            name = b[p:p + nsz].split(b"\0")[0].decode("ascii")
            p += nsz
            dt = self.dtype(b[p:p + tsz])
            p += tsz
            shape = self.space(b[p:p + ssz])
            p += ssz
        else:
            raise H5FormatError("attribute version %d" % ver)
        n = int(np.prod(shape)) if shape else 1
        raw = bytes(b[p:p + n * dt.itemsize])
        val = np.frombuffer(raw, dtype=dt, count=n)
        if dt.kind == "S":
            return name, val[0].split(b"\0")[0].decode("ascii")
        return name, val if shape else val[0]

    def dataset(self, addr):
        shape, dt, data, attrs = None, None, None, {}
        for mtype, b in self.messages(addr):
            if mtype == MSG_DATASPACE:
                shape = self.space(b)
            elif mtype == MSG_DATATYPE:
                dt = self.dtype(b)
            elif mtype == MSG_LAYOUT:
                if b[0] != 3:
                    raise H5FormatError("layout version %d" % b[0])
                if b[1] == 1:                            # contiguous
                    a, size = struct.unpack_from("<QQ", b, 2)
                    data = (a, size)
                elif b[1] == 0:                          # compact
                    size = struct.unpack_from("<H", b, 2)[0]
                    data = bytes(b[4:4 + size])
                else:
                    raise H5FormatError("chunked layout not read")
            elif mtype == MSG_ATTRIBUTE:
                k, v = self.attribute(b)
                attrs[k] = v
        if shape is None or dt is None or data is None:
            raise H5FormatError("object is not a dataset")
        n = int(np.prod(shape)) if shape else 1
        if isinstance(data, tuple):
            a, size = data
            raw = self.d[a:a + n * dt.itemsize] if a != UNDEF else b"\0" * (n * dt.itemsize)
        else:
            raw = data
        arr = np.frombuffer(bytes(raw), dtype=dt, count=n).reshape(shape)
        return arr.astype(dt.newbyteorder("=")), attrs


def read(path):
    """{name: (array, {"Variable": ..., "units": ...})} of every dataset in the root group."""
    with open(path, "rb") as f:
        F = _File(f.read())
    btree = heap = None
    for mtype, b in F.messages(F.root_ohdr):
        if mtype == MSG_SYMTAB:
            btree, heap = struct.unpack_from("<QQ", b)
    if btree is None:
        raise H5FormatError("root group without a symbol table (new-style groups are not read)")
    return {n: F.dataset(a) for n, a in F.group_entries(btree, heap).items()}


def structure(path):
    """For each dataset, the sequence of its object header's message types and the datatype
    message: the layout a writer must match."""
    with open(path, "rb") as f:
        F = _File(f.read())
    btree = heap = None
    for mtype, b in F.messages(F.root_ohdr):
        if mtype == MSG_SYMTAB:
            btree, heap = struct.unpack_from("<QQ", b)
    out = {}
    for n, a in F.group_entries(btree, heap).items():
        msgs = [(t, bytes(b)) for t, b in F.messages(a) if t != MSG_NIL]
        out[n] = ([t for t, _ in msgs], [b[:20] for t, b in msgs if t == MSG_DATATYPE][0])
    return out
