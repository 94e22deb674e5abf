"""A reader for the subset of the HDF5 file format that dmplex_b200.vtkhdf writes (superblock
version 0, version-1 object headers, symbol-table groups, contiguous datasets, version-1
attributes), written from the HDF5 file-format specification to check the writer's files
without an HDF5 library. It asserts the invariants a reader of the format relies on: the
signatures and versions, 8-byte alignment, the end-of-file address, message sizes, sorted
symbol-table entries with B-tree keys naming the last entry of each child, and whole
B-tree / symbol-table nodes inside the file (a library reads them at full size)."""
import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class Reader:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.b = f.read()
        b = self.b
        assert b[:8] == SIG
        v_sb, v_fs, v_root, _, v_shared, so, sl, _ = b[8:16]
        assert (v_sb, v_fs, v_root, v_shared, so, sl) == (0, 0, 0, 0, 8, 8)
        self.leaf_k, self.node_k, flags = struct.unpack_from("<HHI", b, 16)
        assert flags == 0 and self.leaf_k > 0 and self.node_k > 0
        base, free, eof, driver = struct.unpack_from("<QQQQ", b, 24)
        assert base == 0 and free == UNDEF and driver == UNDEF and eof == len(b)
        name, header, cache = struct.unpack_from("<QQI", b, 56)
        btree, heap = struct.unpack_from("<QQ", b, 80)
        assert name == 0 and cache == 1
        self.root = self.read_object(header, expect_cache=(btree, heap))

    def read_object(self, addr, expect_cache=None):
        b = self.b
        assert addr % 8 == 0
        version, _, nmsgs, refs, size = struct.unpack_from("<BBHII", b, addr)
        assert version == 1 and refs >= 1 and addr + 16 + size <= len(b)
        p, end = addr + 16, addr + 16 + size
        msgs = []
        while p < end:
            mtype, msize, mflags = struct.unpack_from("<HHB", b, p)
            assert msize % 8 == 0 and p + 8 + msize <= end
            msgs.append((mtype, b[p + 8:p + 8 + msize]))
            p += 8 + msize
        assert p == end and len(msgs) == nmsgs
        kinds = {t for t, _ in msgs}
        attrs = dict(self.attribute(m) for t, m in msgs if t == 0x000C)
        if 0x0011 in kinds:
            (stab,) = [m for t, m in msgs if t == 0x0011]
            btree, heap = struct.unpack_from("<QQ", stab)
            if expect_cache is not None:
                assert expect_cache == (btree, heap)
            return ("group", self.group(btree, heap), attrs)
        assert {0x0001, 0x0003, 0x0008} <= kinds
        (space,) = [m for t, m in msgs if t == 0x0001]
        (dtype_msg,) = [m for t, m in msgs if t == 0x0003]
        (layout,) = [m for t, m in msgs if t == 0x0008]
        for t, m in msgs:
            if t == 0x0005:
                assert m[0] == 2  # fill value message version 2
        shape = self.dataspace(space)
        dt = self.datatype(dtype_msg)
        lv, lclass, daddr, dsize = struct.unpack_from("<BBQQ", layout)
        assert lv == 3 and lclass == 1
        n = int(np.prod(shape)) * dt.itemsize
        assert dsize == n
        if n == 0:
            assert daddr == UNDEF
            return ("dataset", np.zeros(shape, dt), attrs)
        assert daddr + n <= len(b)
        return ("dataset", np.frombuffer(b, dt, int(np.prod(shape)), daddr).reshape(shape).copy(), attrs)

    @staticmethod
    def dataspace(m):
        version, rank, flags = m[0], m[1], m[2]
        assert version == 1 and flags == 0
        return tuple(struct.unpack_from("<Q", m, 8 + 8 * i)[0] for i in range(rank))

    @staticmethod
    def datatype(m):
        cv = m[0]
        version, cls = cv >> 4, cv & 15
        bits = m[1:4]
        (size,) = struct.unpack_from("<I", m, 4)
        assert version == 1
        if cls == 0:
            assert bits[0] & 1 == 0  # little endian
            offset, precision = struct.unpack_from("<HH", m, 8)
            assert offset == 0 and precision == 8 * size
            return np.dtype(("<i" if bits[0] & 8 else "<u") + str(size))
        if cls == 1:
            assert bits[0] == 0x20 and bits[1] == 8 * size - 1
            offset, precision, eloc, esize, mloc, msize, bias = struct.unpack_from("<HHBBBBI", m, 8)
            assert (offset, precision, mloc) == (0, 8 * size, 0)
            assert (eloc, esize, msize, bias) == {8: (52, 11, 52, 1023), 4: (23, 8, 23, 127)}[size]
            return np.dtype("<f" + str(size))
        if cls == 3:
            assert bits[0] & 15 in (0, 1) and bits[0] >> 4 == 0  # null terminated/padded, ASCII
            return np.dtype("S" + str(size))
        raise AssertionError(f"datatype class {cls}")

    def attribute(self, m):
        version, _, nsize, dsize, ssize = struct.unpack_from("<BBHHH", m)
        assert version == 1
        p = 8
        name = m[p:p + nsize]
        assert name.endswith(b"\0")
        p += -(-nsize // 8) * 8
        dt = self.datatype(m[p:p + dsize])
        p += -(-dsize // 8) * 8
        shape = self.dataspace(m[p:p + ssize])
        p += -(-ssize // 8) * 8
        n = int(np.prod(shape))
        value = np.frombuffer(m, dt, n, p).reshape(shape).copy()
        return name[:-1].decode(), value

    def heap(self, addr):
        b = self.b
        assert b[addr:addr + 4] == b"HEAP" and b[addr + 4] == 0
        size, free, data = struct.unpack_from("<QQQ", b, addr + 8)
        assert free == 1 or free < size  # 1: no free block
        assert data + size <= len(b) and size % 8 == 0
        return b[data:data + size]

    def group(self, btree, heap_addr):
        b = self.b
        heap = self.heap(heap_addr)

        def name_at(off):
            return heap[off:heap.index(b"\0", off)].decode()
        assert b[btree:btree + 4] == b"TREE"
        ntype, level, used = struct.unpack_from("<BBH", b, btree + 4)
        left, right = struct.unpack_from("<QQ", b, btree + 8)
        assert ntype == 0 and level == 0 and left == UNDEF and right == UNDEF
        two_k = 2 * self.node_k
        assert used <= two_k and btree + 24 + (two_k + 1) * 8 + two_k * 8 <= len(b)
        p = btree + 24
        keys, children = [struct.unpack_from("<Q", b, p)[0]], []
        p += 8
        for _ in range(used):
            child, key = struct.unpack_from("<QQ", b, p)
            children.append(child)
            keys.append(key)
            p += 16
        assert name_at(keys[0]) == ""
        members, names = {}, []
        snod_size = 8 + 2 * self.leaf_k * 40
        for i, child in enumerate(children):
            assert b[child:child + 4] == b"SNOD" and b[child + 4] == 1
            (nsym,) = struct.unpack_from("<H", b, child + 6)
            assert 1 <= nsym <= 2 * self.leaf_k and child + snod_size <= len(b)
            last = None
            for j in range(nsym):
                off, header, cache = struct.unpack_from("<QQI", b, child + 8 + 40 * j)
                name = name_at(off)
                cache_addrs = struct.unpack_from("<QQ", b, child + 8 + 40 * j + 24) if cache == 1 else None
                members[name] = self.read_object(header, expect_cache=cache_addrs)
                names.append(name)
                last = off
            assert keys[i + 1] == last  # key after child i: its last name
        assert names == sorted(names, key=lambda s: s.encode())
        return members


def read_hdf5(path):
    """(members, attributes) of the root group; a member is ('group', members, attrs) or
    ('dataset', array, attrs)."""
    r = Reader(path)
    return r.root[1], r.root[2]
