"""A small, independent walker of the HDF5 structures the checkpoint files use, for the tests:
it lists the root group's datasets with their raw object-header messages, so that a file the
library writes can be compared message by message with one the HDF5 library wrote (the
reference's fixtures).  It follows the HDF5 file format specification for a version-0
superblock, symbol-table groups (v1 B-tree, SNOD, local heap) and version-1 object headers;
it shares no code with channel_passive_b200/csrc/h5io.cpp."""
from __future__ import annotations

import struct

UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Walk:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        assert self.b[:8] == b"\x89HDF\r\n\x1a\n", "HDF5 signature"
        assert self.b[8] == 0, "superblock version 0"
        self.leaf_k, self.node_k = struct.unpack_from("<HH", self.b, 16)
        self.eof = self._q(40)
        self.root = self._q(64)
        self.root_msgs = self.messages(self.root)
        stab = [m for m in self.root_msgs if m[0] == 0x11]
        assert len(stab) == 1
        self.btree, self.heap = struct.unpack_from("<QQ", stab[0][2])
        assert self.b[self.heap:self.heap + 4] == b"HEAP"
        self.heap_size, self.heap_free, self.heap_data = struct.unpack_from("<QQQ", self.b, self.heap + 8)
        self.links = {}
        self.btree_keys = []
        self._walk(self.btree)

    def _q(self, o):
        return struct.unpack_from("<Q", self.b, o)[0]

    def _name(self, off):
        s = self.heap_data + off
        return self.b[s:self.b.index(b"\0", s)].decode()

    def messages(self, addr):
        """[(type, flags, body bytes)] of a version-1 object header, continuations followed."""
        assert self.b[addr] == 1, "object header version 1"
        nmsg, _, size = struct.unpack_from("<HII", self.b, addr + 2)
        blocks, out = [(addr + 16, size)], []
        while blocks and len(out) < nmsg:
            p, n = blocks.pop(0)
            end = p + n
            while p + 8 <= end and len(out) < nmsg:
                t, s, fl = struct.unpack_from("<HHB", self.b, p)
                body = self.b[p + 8:p + 8 + s]
                if t == 0x10:
                    blocks.append(struct.unpack_from("<QQ", body))
                out.append((t, fl, body))
                p += 8 + s
        return out

    def _walk(self, node):
        assert self.b[node:node + 4] == b"TREE" and self.b[node + 4] == 0
        level, used = self.b[node + 5], struct.unpack_from("<H", self.b, node + 6)[0]
        keys = [self._q(node + 24 + 16 * i) for i in range(used + 1)]
        kids = [self._q(node + 32 + 16 * i) for i in range(used)]
        self.btree_keys.append([self._name(k) for k in keys])
        for c in kids:
            if level:
                self._walk(c)
                continue
            assert self.b[c:c + 4] == b"SNOD" and self.b[c + 4] == 1
            n = struct.unpack_from("<H", self.b, c + 6)[0]
            assert n <= 2 * self.leaf_k
            for i in range(n):
                e = c + 8 + 40 * i
                self.links[self._name(self._q(e))] = self._q(e + 8)

    def dataset(self, name):
        """{type: (flags, body)} of a dataset's messages (the last of each type)."""
        return {t: (fl, body) for t, fl, body in self.messages(self.links[name])}

    def data(self, name):
        m = self.dataset(name)
        lay = m[0x08][1]
        assert lay[0] == 3 and lay[1] == 1, "contiguous layout, version 3"
        addr, size = struct.unpack_from("<QQ", lay, 2)
        return self.b[addr:addr + size]
