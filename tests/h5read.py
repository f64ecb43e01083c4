"""TEST INFRASTRUCTURE: an independent reader of the HDF5 files the snapshot writer produces, written
from the public HDF5 File Format Specification for the tests (the product's reader is C++, in
nse2d-channel-gpu_b200/host/h5lite.cpp). It reads superblock version 0, the root group as a
symbol-table group (version-1 B-tree of type 0, symbol table nodes, local heap), version-1 object
headers with continuation messages, and the dataspace, datatype, layout (version 3) and attribute
(version 1) messages; every structure it walks is also recorded in `structures` so that tests can
check the layout byte by byte.
"""
import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(Exception):
    pass


class Dataset:
    def __init__(self, name, dims, dtype, address, size, messages):
        self.name, self.dims, self.dtype, self.address, self.size, self.messages = \
            name, dims, dtype, address, size, messages


class H5File:
    def __init__(self, path):
        self.buf = open(path, "rb").read()
        self.structures = {}
        b = self.buf
        if b[:8] != SIG:
            raise H5Error("no HDF5 signature at offset 0")
        sb = dict(version=b[8], freespace_version=b[9], root_entry_version=b[10], shared_header_version=b[12],
                  sizeof_offsets=b[13], sizeof_lengths=b[14], leaf_k=self.u(16, 2), internal_k=self.u(18, 2),
                  flags=self.u(20, 4))
        if sb["version"] != 0 or sb["sizeof_offsets"] != 8 or sb["sizeof_lengths"] != 8:
            raise H5Error(f"unsupported superblock {sb}")
        sb.update(base=self.u(24), freespace=self.u(32), eof=self.u(40), driver=self.u(48))
        ste = self.symbol_table_entry(56)
        sb["root"] = ste
        self.structures["superblock"] = sb
        root_msgs = self.object_header(ste["header"])
        self.structures["root_header_messages"] = root_msgs
        sym = [m for m in root_msgs if m["type"] == 0x11]
        if not sym:
            raise H5Error("root group has no symbol table message")
        btree, heap = struct.unpack_from("<QQ", sym[0]["data"])
        if ste["cache_type"] == 1 and (ste["scratch"][0], ste["scratch"][1]) != (btree, heap):
            raise H5Error("root entry scratch pad disagrees with the symbol table message")
        self.heap = self.local_heap(heap)
        self.links = {}
        self.btree(btree)
        self.attrs = {}
        for m in root_msgs:
            if m["type"] == 0x0C:
                name, value, dt = self.attribute(m["data"])
                self.attrs[name] = value
                self.structures.setdefault("attr_types", {})[name] = dt

    def u(self, off, n=8):
        return int.from_bytes(self.buf[off:off + n], "little")

    def symbol_table_entry(self, off):
        return dict(name_offset=self.u(off), header=self.u(off + 8), cache_type=self.u(off + 16, 4),
                    scratch=(self.u(off + 24), self.u(off + 32)))

    def local_heap(self, off):
        b = self.buf
        if b[off:off + 4] != b"HEAP":
            raise H5Error("bad local heap signature")
        h = dict(version=b[off + 4], data_size=self.u(off + 8), free_list=self.u(off + 16), data=self.u(off + 24))
        self.structures["local_heap"] = h
        return h

    def heap_name(self, offset):
        start = self.heap["data"] + offset
        end = self.buf.index(b"\0", start)
        return self.buf[start:end].decode()

    def btree(self, off, depth=0):
        b = self.buf
        if b[off:off + 4] == b"TREE":
            node = dict(type=b[off + 4], level=b[off + 5], entries=self.u(off + 6, 2), left=self.u(off + 8),
                        right=self.u(off + 16))
            keys, children = [], []
            p = off + 24
            for k in range(node["entries"]):
                keys.append(self.u(p))
                children.append(self.u(p + 8))
                p += 16
            keys.append(self.u(p))
            node.update(keys=keys, children=children)
            self.structures.setdefault("btree_nodes", []).append(node)
            if node["type"] != 0:
                raise H5Error("not a group B-tree")
            for c in children:
                self.btree(c, depth + 1)
        elif b[off:off + 4] == b"SNOD":
            n = self.u(off + 6, 2)
            node = dict(version=b[off + 4], symbols=n, entries=[])
            for k in range(n):
                e = self.symbol_table_entry(off + 8 + 40 * k)
                e["name"] = self.heap_name(e["name_offset"])
                node["entries"].append(e)
                self.links[e["name"]] = e["header"]
            self.structures.setdefault("symbol_nodes", []).append(node)
        else:
            raise H5Error(f"bad group node at {off}")

    def object_header(self, off):
        b = self.buf
        if b[off] != 1:
            raise H5Error(f"object header version {b[off]} (expected 1)")
        nmsg, refcount, size = self.u(off + 2, 2), self.u(off + 4, 4), self.u(off + 8, 4)
        chunks = [(off + 16, size)]
        msgs = []
        while chunks:
            start, length = chunks.pop(0)
            p = start
            while p + 8 <= start + length:
                t, n, fl = self.u(p, 2), self.u(p + 2, 2), b[p + 4]
                if n % 8:
                    raise H5Error("version-1 header message not 8-byte aligned")
                data = b[p + 8:p + 8 + n]
                if t == 0x10:
                    chunks.append(struct.unpack_from("<QQ", data))
                msgs.append(dict(type=t, size=n, flags=fl, data=data))
                p += 8 + n
            if p != start + length:
                raise H5Error("messages do not fill the header chunk")
        if len(msgs) != nmsg:
            raise H5Error(f"header says {nmsg} messages, found {len(msgs)}")
        return msgs

    @staticmethod
    def datatype(d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = struct.unpack_from("<I", d, 4)[0]
        order = ">" if bits & 1 else "<"
        if cls == 1:
            if size not in (4, 8):
                raise H5Error("float size")
            return dict(cls="float", version=ver, size=size, np=np.dtype(order + ("f8" if size == 8 else "f4")),
                        sign_bit=(bits >> 8) & 0xFF, props=struct.unpack_from("<HHBBBBI", d, 8))
        if cls == 0:
            signed = bool(bits & 8)
            return dict(cls="int", version=ver, size=size, signed=signed,
                        np=np.dtype(order + ("i" if signed else "u") + str(size)), props=struct.unpack_from("<HH", d, 8))
        raise H5Error(f"datatype class {cls}")

    @staticmethod
    def dataspace(d):
        ver, rank, flags = d[0], d[1], d[2]
        if ver != 1:
            raise H5Error("dataspace version")
        dims = [struct.unpack_from("<Q", d, 8 + 8 * k)[0] for k in range(rank)]
        return dict(version=ver, rank=rank, flags=flags, dims=dims)

    def attribute(self, d):
        if d[0] != 1:
            raise H5Error("attribute message version")
        nlen, tlen, slen = struct.unpack_from("<HHH", d, 2)
        pad = lambda n: (n + 7) & ~7          # noqa: E731
        p = 8
        name = d[p:p + nlen].split(b"\0")[0].decode()
        p += pad(nlen)
        dt = self.datatype(d[p:p + tlen])
        p += pad(tlen)
        ds = self.dataspace(d[p:p + slen])
        p += pad(slen)
        count = int(np.prod(ds["dims"])) if ds["rank"] else 1
        val = np.frombuffer(d[p:p + count * dt["size"]], dtype=dt["np"])
        return name, (val[0].item() if ds["rank"] == 0 else val), dict(dt, space=ds)

    def dataset(self, name):
        msgs = self.object_header(self.links[name])
        by = {m["type"]: m for m in msgs}
        for t in (0x01, 0x03, 0x08):
            if t not in by:
                raise H5Error(f"dataset {name} lacks message {t:#x}")
        space = self.dataspace(by[0x01]["data"])
        dt = self.datatype(by[0x03]["data"])
        lay = by[0x08]["data"]
        if lay[0] != 3 or lay[1] != 1:
            raise H5Error("layout is not version-3 contiguous")
        addr, size = struct.unpack_from("<QQ", lay, 2)
        return Dataset(name, space["dims"], dt, addr, size, msgs)

    def read(self, name):
        ds = self.dataset(name)
        n = int(np.prod(ds.dims))
        if ds.size != n * ds.dtype["size"] or ds.address + ds.size > len(self.buf):
            raise H5Error("data does not fit")
        return np.frombuffer(self.buf[ds.address:ds.address + ds.size], dtype=ds.dtype["np"]).reshape(ds.dims)
