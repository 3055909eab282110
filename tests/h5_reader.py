"""A reader of the HDF5 subset the library's dump writer produces (test
infrastructure): superblock version 0, version 1 object headers, groups as
symbol tables (version 1 B-tree, local heap, symbol-table nodes), contiguous
datasets of little-endian fixed-point and IEEE floating-point elements.
Written from the published file-format description; it checks every
signature, version and size field it reads, so a file that strays from that
description fails here.

read(path) -> {"name": ndarray or nested dict}.
"""
import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


def _u(b, o, n):
    return int.from_bytes(b[o:o + n], "little")


class _File:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.b = f.read()
        b = self.b
        assert b[:8] == b"\x89HDF\r\n\x1a\n", "signature"
        assert b[8] == 0, "superblock version"
        assert b[13] == 8 and b[14] == 8, "sizes of offsets and lengths"
        self.leaf_k = _u(b, 16, 2)
        self.internal_k = _u(b, 18, 2)
        assert _u(b, 24, 8) == 0, "base address"
        eof = _u(b, 40, 8)
        assert eof == len(b), ("end of file address", eof, len(b))
        self.root_header = _u(b, 64, 8)

    def header(self, addr):
        """Messages (type, data) of a version 1 object header."""
        b = self.b
        assert b[addr] == 1, "object header version"
        nmsg = _u(b, addr + 2, 2)
        size = _u(b, addr + 8, 4)
        o, end, out = addr + 16, addr + 16 + size, []
        for _ in range(nmsg):
            t, s = _u(b, o, 2), _u(b, o + 2, 2)
            assert s % 8 == 0, "message size"
            out.append((t, b[o + 8:o + 8 + s]))
            o += 8 + s
        assert o == end, "object header size"
        return out

    def heap_name(self, heap, off):
        b = self.b
        assert b[heap:heap + 4] == b"HEAP" and b[heap + 4] == 0, "local heap"
        size = _u(b, heap + 8, 8)
        free = _u(b, heap + 16, 8)
        data = _u(b, heap + 24, 8)
        assert free == 1 or free < size, "heap free list"
        assert off < size
        s = b[data + off:data + size]
        return s[:s.index(b"\0")].decode()

    def group(self, addr):
        msgs = self.header(addr)
        sym = [d for t, d in msgs if t == 0x11]
        assert len(sym) == 1, "symbol table message"
        btree, heap = _u(sym[0], 0, 8), _u(sym[0], 8, 8)
        b = self.b
        assert b[btree:btree + 4] == b"TREE" and b[btree + 4] == 0 and b[btree + 5] == 0, "leaf group B-tree"
        used = _u(b, btree + 6, 2)
        out = {}
        prev = None
        for k in range(used):
            child = _u(b, btree + 24 + 8 + 16 * k, 8)
            assert b[child:child + 4] == b"SNOD" and b[child + 4] == 1, "symbol table node"
            nsym = _u(b, child + 6, 2)
            assert nsym <= 2 * self.leaf_k
            for e in range(nsym):
                o = child + 8 + 40 * e
                name = self.heap_name(heap, _u(b, o, 8))
                assert prev is None or name > prev, "entries sorted by name"
                prev = name
                hdr = _u(b, o + 8, 8)
                kinds = [t for t, _ in self.header(hdr)]
                out[name] = self.group(hdr) if 0x11 in kinds else self.dataset(hdr)
        return out

    def dataset(self, addr):
        msgs = dict(self.header(addr))
        sp, ty, lay = msgs[0x01], msgs[0x03], msgs[0x08]
        assert 0x05 in msgs, "fill value message"
        assert sp[0] == 1, "dataspace version"
        rank = sp[1]
        dims = [_u(sp, 8 + 8 * i, 8) for i in range(rank)]
        cls, ver = ty[0] & 0x0F, ty[0] >> 4
        assert ver == 1
        size = _u(ty, 4, 4)
        if cls == 0:
            assert ty[1] & 1 == 0, "little endian"
            dt = np.dtype(("<i" if ty[1] & 8 else "<u") + str(size))
            assert _u(ty, 10, 2) == 8 * size, "precision"
        elif cls == 1:
            assert ty[1] & 1 == 0 and (ty[1] >> 4) & 3 == 2, "little endian, implied msb"
            assert ty[2] == 8 * size - 1, "sign bit"
            assert _u(ty, 10, 2) == 8 * size
            expect = (23, 8, 0, 23, 127) if size == 4 else (52, 11, 0, 52, 1023)
            got = (ty[12], ty[13], ty[14], ty[15], _u(ty, 16, 4))
            assert got == expect, ("IEEE layout", got)
            dt = np.dtype("<f" + str(size))
        else:
            raise AssertionError(f"datatype class {cls}")
        assert lay[0] == 3 and lay[1] == 1, "contiguous layout, version 3"
        daddr, nbytes = _u(lay, 2, 8), _u(lay, 10, 8)
        n = int(np.prod(dims)) if dims else 1
        assert nbytes == n * dt.itemsize, "layout size"
        return np.frombuffer(self.b, dtype=dt, count=n, offset=daddr).reshape(dims).copy()


def read(path):
    f = _File(path)
    return f.group(f.root_header)

