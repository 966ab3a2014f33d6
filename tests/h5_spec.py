"""A second, independent HDF5 reader (and a small writer) in numpy, written
from the published HDF5 file format specification, used by the tests to
check the library's P123 files.  Test infrastructure only.

Reader scope: superblock versions 0/1, version-1 object headers (with
continuation blocks), symbol-table groups (v1 B-trees, SNOD nodes, local
heaps), dataspace messages v1/v2, datatypes fixed-point / IEEE float /
fixed string / compound (v1-v3), layout message v3 (compact, contiguous,
chunked with a v1 B-tree index, no filters) and attribute messages v1.

Writer scope: the same structures, contiguous or chunked rank-1 datasets,
attributes optionally in object-header continuation blocks, used to produce
files laid out like the HDF5 library's H5TBmake_table (chunked tables with
unlimited maximum size) that the library reader must also accept.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


def _pad8(n):
    return (n + 7) // 8 * 8


class H5Error(Exception):
    pass


# --------------------------------------------------------------------------
# reader
# --------------------------------------------------------------------------
class _Buf:
    def __init__(self, b, pos=0):
        self.b = b
        self.pos = pos

    def take(self, n):
        if self.pos + n > len(self.b):
            raise H5Error("truncated structure")
        out = self.b[self.pos:self.pos + n]
        self.pos += n
        return out

    def u(self, n):
        return int.from_bytes(self.take(n), "little")

    def cstring(self):
        end = self.b.index(b"\0", self.pos)
        s = self.b[self.pos:end].decode()
        self.pos = end + 1
        return s


def _dtype(buf):
    """Decodes a datatype message; returns a dict with 'np' (numpy dtype)."""
    cv = buf.u(1)
    version, cls = cv >> 4, cv & 0x0F
    bits = buf.take(3)
    size = buf.u(4)
    if cls == 0:
        order = ">" if bits[0] & 1 else "<"
        signed = bool(bits[0] & 0x08)
        buf.take(4)
        return {"class": "int", "size": size, "signed": signed, "np": np.dtype(f"{order}{'i' if signed else 'u'}{size}")}
    if cls == 1:
        order = ">" if bits[0] & 1 else "<"
        props = buf.take(12)
        _, prec, eloc, esize, mloc, msize, bias = struct.unpack("<HHBBBBI", props)
        if (size, prec, eloc, esize, mloc, msize, bias) != (8, 64, 52, 11, 0, 52, 1023):
            raise H5Error("only IEEE binary64 floats are handled")
        return {"class": "float", "size": size, "np": np.dtype(f"{order}f8")}
    if cls == 3:
        return {"class": "string", "size": size, "pad": bits[0] & 0x0F, "np": np.dtype(f"S{size}")}
    if cls == 6:
        nmemb = bits[0] | (bits[1] << 8)
        names, offsets, types = [], [], []
        for _ in range(nmemb):
            start = buf.pos
            names.append(buf.cstring())
            if version < 3:
                buf.pos = start + _pad8(buf.pos - start)
                offsets.append(buf.u(4))
                if version == 1:
                    buf.take(1 + 3 + 4 + 4 + 16)
            else:
                nb = 1
                while nb < 4 and (1 << (8 * nb)) <= size:
                    nb += 1
                offsets.append(buf.u(nb))
            types.append(_dtype(buf))
        npdt = np.dtype({"names": names, "formats": [t["np"] for t in types], "offsets": offsets, "itemsize": size})
        return {"class": "compound", "size": size, "names": names, "offsets": offsets, "types": types, "np": npdt}
    raise H5Error(f"datatype class {cls} not handled")


def _dataspace(buf):
    version = buf.u(1)
    rank = buf.u(1)
    flags = buf.u(1)
    buf.take(5 if version == 1 else 1)
    dims = [buf.u(8) for _ in range(rank)]
    maxdims = [buf.u(8) for _ in range(rank)] if flags & 1 else None
    return {"version": version, "dims": dims, "maxdims": maxdims, "scalar": rank == 0}


class File:
    """Parses a whole file; `datasets` maps root link names to dicts with
    'dims', 'type', 'layout', 'attrs' and 'data' (numpy array)."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self.raw = fh.read()
        b = self.raw
        if b[:8] != SIGNATURE:
            raise H5Error("no HDF5 signature at offset 0")
        sb = _Buf(b, 8)
        self.superblock_version = sb.u(1)
        if self.superblock_version > 1:
            raise H5Error("superblock version > 1")
        sb.u(1), sb.u(1), sb.u(1), sb.u(1)
        if sb.u(1) != 8 or sb.u(1) != 8:
            raise H5Error("offset/length sizes other than 8")
        sb.u(1)
        self.leaf_k, self.internal_k = sb.u(2), sb.u(2)
        sb.u(4)
        if self.superblock_version == 1:
            sb.u(4)
        self.base, self.freespace, self.eof, self.driver = sb.u(8), sb.u(8), sb.u(8), sb.u(8)
        self.root_name_off, self.root_oh = sb.u(8), sb.u(8)
        self.root_cache_type = sb.u(4)
        sb.u(4)
        self.root_scratch = (sb.u(8), sb.u(8))
        self.links = self._group(self.root_oh)
        self.datasets = {name: self._dataset(addr) for name, addr in self.links.items()}

    # -- object headers
    def _messages(self, addr):
        pre = _Buf(self.raw, addr)
        if pre.u(1) != 1:
            raise H5Error("object header version other than 1")
        pre.u(1)
        nmsg = pre.u(2)
        pre.u(4)
        size = pre.u(4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            if start % 8:
                raise H5Error("object header messages not 8-byte aligned")
            m = _Buf(self.raw, start)
            while m.pos + 8 <= start + length and len(out) < nmsg:
                mtype, msize, flags = m.u(2), m.u(2), m.u(1)
                m.take(3)
                if msize % 8:
                    raise H5Error("message size not a multiple of 8")
                body = m.take(msize)
                out.append((mtype, flags, body))
                if mtype == 0x10:
                    c = _Buf(body)
                    blocks.append((c.u(8), c.u(8)))
        return [x for x in out if x[0] not in (0x00, 0x10)]

    # -- groups
    def _group(self, oh):
        for mtype, _, body in self._messages(oh):
            if mtype == 0x11:
                c = _Buf(body)
                tree, heap = c.u(8), c.u(8)
                names = self._heap(heap)
                links = {}
                self._tree(tree, names, links)
                return links
        raise H5Error("group without a symbol table message")

    def _heap(self, addr):
        h = _Buf(self.raw, addr)
        if h.take(4) != b"HEAP" or h.u(1) != 0:
            raise H5Error("bad local heap")
        h.take(3)
        size, free, data = h.u(8), h.u(8), h.u(8)
        if free != 1 and free >= size:
            raise H5Error("bad local heap free list")
        seg = self.raw[data:data + size]
        if len(seg) != size or seg[:1] != b"\0":
            raise H5Error("local heap data segment must start with the empty name")
        return seg

    def _tree(self, addr, names, links):
        t = _Buf(self.raw, addr)
        if t.take(4) != b"TREE" or t.u(1) != 0:
            raise H5Error("bad group B-tree node")
        level, entries = t.u(1), t.u(2)
        t.u(8), t.u(8)
        keys, kids = [], []
        for _ in range(entries):
            keys.append(t.u(8))
            kids.append(t.u(8))
        keys.append(t.u(8))
        for i, kid in enumerate(kids):
            if level:
                self._tree(kid, names, links)
            else:
                child = self._snod(kid, names)
                # keys bound the child's names: (key[i], key[i+1]]
                last = names[keys[i + 1]:names.index(b"\0", keys[i + 1])].decode()
                if max(child) != last:
                    raise H5Error("B-tree key does not name the node's last link")
                links.update(child)

    def _snod(self, addr, names):
        s = _Buf(self.raw, addr)
        if s.take(4) != b"SNOD" or s.u(1) != 1:
            raise H5Error("bad symbol table node")
        s.u(1)
        n = s.u(2)
        if n > 2 * self.leaf_k:
            raise H5Error("symbol table node over capacity")
        out, prev = {}, None
        for _ in range(n):
            off, oh, cache = s.u(8), s.u(8), s.u(4)
            s.take(4 + 16)
            name = names[off:names.index(b"\0", off)].decode()
            if prev is not None and not prev < name:
                raise H5Error("symbol table entries not sorted by name")
            prev = name
            out[name] = oh
        return out

    # -- datasets
    def _dataset(self, oh):
        ds = {"attrs": {}}
        for mtype, flags, body in self._messages(oh):
            b = _Buf(body)
            if mtype == 0x01:
                ds["space"] = _dataspace(b)
                ds["dims"] = ds["space"]["dims"]
            elif mtype == 0x03:
                ds["type"] = _dtype(b)
            elif mtype == 0x05:
                ds["fill"] = bytes(body[:4])
            elif mtype == 0x08:
                if b.u(1) != 3:
                    raise H5Error("layout message version other than 3")
                cls = b.u(1)
                if cls == 0:
                    n = b.u(2)
                    ds["layout"] = {"class": "compact", "data": b.take(n)}
                elif cls == 1:
                    ds["layout"] = {"class": "contiguous", "addr": b.u(8), "size": b.u(8)}
                elif cls == 2:
                    nd = b.u(1)
                    addr = b.u(8)
                    ds["layout"] = {"class": "chunked", "addr": addr, "chunk": [b.u(4) for _ in range(nd)]}
            elif mtype == 0x0B:
                raise H5Error("filter pipelines not handled")
            elif mtype == 0x0C:
                name, value = self._attribute(b)
                ds["attrs"][name] = value
        for k in ("space", "type", "layout"):
            if k not in ds:
                raise H5Error(f"dataset without a {k} message")
        ds["data"] = self._data(ds)
        return ds

    def _attribute(self, b):
        if b.u(1) != 1:
            raise H5Error("attribute message version other than 1")
        b.u(1)
        nlen, tlen, slen = b.u(2), b.u(2), b.u(2)
        name = b.take(_pad8(nlen))[:nlen - 1].decode()
        tb = _Buf(b.take(_pad8(tlen)))
        t = _dtype(tb)
        sp = _dataspace(_Buf(b.take(_pad8(slen))))
        n = int(np.prod(sp["dims"])) if sp["dims"] else 1
        raw = b.take(n * t["size"])
        if t["class"] == "string":
            return name, raw.split(b"\0", 1)[0].decode()
        return name, np.frombuffer(raw, dtype=t["np"])

    def _data(self, ds):
        t, dims, lay = ds["type"], ds["dims"], ds["layout"]
        n = int(np.prod(dims)) if dims else 1
        nbytes = n * t["size"]
        if lay["class"] == "compact":
            raw = lay["data"][:nbytes]
        elif lay["class"] == "contiguous":
            if lay["addr"] == UNDEF:
                raw = bytes(nbytes)
            else:
                if lay["size"] != nbytes:
                    raise H5Error("contiguous storage size differs from the extent")
                raw = self.raw[lay["addr"]:lay["addr"] + nbytes]
                if lay["addr"] + nbytes > self.eof:
                    raise H5Error("data beyond the end-of-file address")
        else:
            out = bytearray(nbytes)
            if lay["addr"] != UNDEF:
                self._chunks(lay["addr"], lay["chunk"], t["size"], dims, out)
            raw = bytes(out)
        if len(raw) != nbytes:
            raise H5Error("short data")
        return np.frombuffer(raw, dtype=t["np"]).reshape(dims if dims else ())

    def _chunks(self, addr, chunk, esize, dims, out):
        t = _Buf(self.raw, addr)
        if t.take(4) != b"TREE" or t.u(1) != 1:
            raise H5Error("bad chunk B-tree node")
        level, entries = t.u(1), t.u(2)
        t.u(8), t.u(8)
        nd = len(chunk)
        for _ in range(entries):
            csize, mask = t.u(4), t.u(4)
            offs = [t.u(8) for _ in range(nd)]
            kid = t.u(8)
            if level:
                self._chunks(kid, chunk, esize, dims, out)
                continue
            if mask:
                raise H5Error("filtered chunk")
            lo = offs[0]
            cnt = min(chunk[0], dims[0] - lo)
            if cnt > 0:
                out[lo * esize:(lo + cnt) * esize] = self.raw[kid:kid + cnt * esize]


# --------------------------------------------------------------------------
# writer (test files only)
# --------------------------------------------------------------------------
def _le(n, v):
    return int(v).to_bytes(n, "little")


def _name8(s):
    b = s.encode() + b"\0"
    return b + bytes(_pad8(len(b)) - len(b))


def dt_int(size=4, signed=True):
    return bytes([0x10, 0x08 if signed else 0, 0, 0]) + _le(4, size) + _le(2, 0) + _le(2, 8 * size)


def dt_f64():
    return bytes([0x11, 0x20, 63, 0]) + _le(4, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)


def dt_str(n):
    return bytes([0x13, 0, 0, 0]) + _le(4, n)


def dt_compound(size, members):
    out = bytes([0x16, len(members) & 0xFF, len(members) >> 8, 0]) + _le(4, size)
    for name, off, t in members:
        out += _name8(name) + _le(4, off) + bytes(1 + 3 + 4 + 4 + 16) + t
    return out


def _space(n, unlimited=False, scalar=False):
    if scalar:
        return bytes([1, 0, 0, 0]) + bytes(4)
    out = bytes([1, 1, 1 if unlimited else 0, 0]) + bytes(4) + _le(8, n)
    return out + (_le(8, UNDEF) if unlimited else b"")


def _msg(mtype, body, flags=0):
    return _le(2, mtype) + _le(2, _pad8(len(body))) + bytes([flags, 0, 0, 0]) + body + bytes(_pad8(len(body)) - len(body))


def _header(msgs, extra=0):
    """Version-1 object header; extra = messages kept in continuation blocks."""
    body = b"".join(msgs)
    return bytes([1, 0]) + _le(2, len(msgs) + extra) + _le(4, 1) + _le(4, len(body)) + bytes(4) + body


def _attr(name, value):
    t, s = dt_str(len(value) + 1), _space(0, scalar=True)
    return (bytes([1, 0]) + _le(2, len(name) + 1) + _le(2, len(t)) + _le(2, len(s)) + _name8(name) +
            t + bytes(_pad8(len(t)) - len(t)) + s + bytes(_pad8(len(s)) - len(s)) + value.encode() + b"\0")


def write(path, datasets, leaf_k=4):
    """datasets: list of dicts {name, type (bytes), n, data (bytes), chunk (int or None), attrs (list of pairs),
    split (bool: attributes in an object-header continuation block)}.  Rank-1 datasets only.  Links go into
    as many symbol-table nodes as leaf_k needs."""
    ds = sorted(datasets, key=lambda d: d["name"])
    heap = bytearray(8)
    name_off = []
    for d in ds:
        name_off.append(len(heap))
        heap += _name8(d["name"])
    cap = 2 * leaf_k
    groups = [ds[i:i + cap] for i in range(0, len(ds), cap)]
    internal_k = 16
    tree_size = 24 + (2 * internal_k + 1) * 8 + 2 * internal_k * 8
    snod_size = 8 + cap * 40

    def headers(addrs, conts=None):
        out, tails = [], []
        for i, (d, a) in enumerate(zip(ds, addrs)):
            esize = len(d["data"]) // max(d["n"], 1) if d["n"] else 0
            msgs = [_msg(0x01, _space(d["n"], unlimited=d.get("chunk") is not None)), _msg(0x03, d["type"], 1),
                    _msg(0x05, bytes([2, 2, 2, 0]), 1)]
            if d.get("chunk") is None:
                msgs.append(_msg(0x08, bytes([3, 1]) + _le(8, a[0] if d["data"] else UNDEF) + _le(8, len(d["data"]))))
            else:
                tsize = d["type_size"]
                msgs.append(_msg(0x08, bytes([3, 2, 2]) + _le(8, a[1]) + _le(4, d["chunk"]) + _le(4, tsize)))
            for k, v in d.get("attrs", []):
                msgs.append(_msg(0x0C, _attr(k, v)))
            if d.get("split") and len(msgs) > 4:
                tail = b"".join(msgs[4:])
                head = msgs[:4] + [_msg(0x10, _le(8, conts[i] if conts else 0) + _le(8, len(tail)))]
                out.append(_header(head, extra=len(msgs) - 4))
                tails.append(tail)
            else:
                out.append(_header(msgs))
                tails.append(b"")
        return out, tails

    a_root = 96
    root = _header([_msg(0x11, bytes(16))])
    a_heap = a_root + len(root)
    a_heapdata = a_heap + 32
    a_tree = a_heapdata + len(heap)
    a_snods = [a_tree + tree_size + i * snod_size for i in range(len(groups))]
    a = a_snods[-1] + snod_size
    probe, tails = headers([(0, 0)] * len(ds))
    a_oh = []
    for h in probe:
        a_oh.append(a)
        a += len(h)
    conts = []
    for t in tails:
        conts.append(a if t else 0)
        a += len(t)
    # data: contiguous blocks; chunked = one B-tree node then the chunks
    layout_addrs, blobs = [], []
    for d in ds:
        if d.get("chunk") is None:
            layout_addrs.append((a, 0))
            blobs.append((a, d["data"]))
            a += _pad8(len(d["data"]))
        else:
            c, tsize, n = d["chunk"], d["type_size"], d["n"]
            nchunks = (n + c - 1) // c
            tree_at = a
            node_size = 24 + nchunks * (8 + 16 + 8) + (8 + 16)
            a += _pad8(node_size)
            chunk_addrs = []
            for i in range(nchunks):
                chunk_addrs.append(a)
                piece = d["data"][i * c * tsize:(i + 1) * c * tsize]
                piece = piece + bytes(c * tsize - len(piece))
                blobs.append((a, piece))
                a += _pad8(len(piece))
            node = b"TREE" + bytes([1, 0]) + _le(2, nchunks) + _le(8, UNDEF) + _le(8, UNDEF)
            for i in range(nchunks):
                node += _le(4, c * tsize) + _le(4, 0) + _le(8, i * c) + _le(8, 0) + _le(8, chunk_addrs[i])
            node += _le(4, 0) + _le(4, 0) + _le(8, nchunks * c) + _le(8, 0)
            blobs.append((tree_at, node))
            layout_addrs.append((0, tree_at))
    eof = a
    hdrs, tails = headers(layout_addrs, conts)
    img = bytearray(eof)
    sb = (SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + _le(2, leaf_k) + _le(2, internal_k) + _le(4, 0) +
          _le(8, 0) + _le(8, UNDEF) + _le(8, eof) + _le(8, UNDEF) +
          _le(8, 0) + _le(8, a_root) + _le(4, 1) + _le(4, 0) + _le(8, a_tree) + _le(8, a_heap))
    img[0:len(sb)] = sb
    root = _header([_msg(0x11, _le(8, a_tree) + _le(8, a_heap))])
    img[a_root:a_root + len(root)] = root
    hh = b"HEAP" + bytes(4) + _le(8, len(heap)) + _le(8, 1) + _le(8, a_heapdata)
    img[a_heap:a_heap + 32] = hh
    img[a_heapdata:a_heapdata + len(heap)] = heap
    node = b"TREE" + bytes([0, 0]) + _le(2, len(groups)) + _le(8, UNDEF) + _le(8, UNDEF) + _le(8, 0)
    pos = 0
    for gi, g in enumerate(groups):
        pos += len(g)
        node += _le(8, a_snods[gi]) + _le(8, name_off[pos - 1])
    img[a_tree:a_tree + len(node)] = node
    pos = 0
    for gi, g in enumerate(groups):
        sn = b"SNOD" + bytes([1, 0]) + _le(2, len(g))
        for d in g:
            sn += _le(8, name_off[pos]) + _le(8, a_oh[pos]) + bytes(24)
            pos += 1
        img[a_snods[gi]:a_snods[gi] + len(sn)] = sn
    for h, at in zip(hdrs, a_oh):
        img[at:at + len(h)] = h
    for t, at in zip(tails, conts):
        if t:
            img[at:at + len(t)] = t
    for at, blob in blobs:
        img[at:at + len(blob)] = blob
    with open(path, "wb") as fh:
        fh.write(bytes(img))
