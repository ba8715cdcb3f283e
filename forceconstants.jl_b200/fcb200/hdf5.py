"""A small HDF5 writer and reader for the force-constant files of
``save_second_order`` / ``save_third_order`` (``fmt="JLD2"``).

The reference writes its default output with JLD2's ``jldsave`` (src/io.jl:32,
63): one HDF5 file whose root group holds ``F2``/``F3`` (the Float64 array),
``N_atoms`` and ``dimension`` (Int64) and ``unit`` (a string).  No HDF5
library is available to this package, so this module writes that file
itself, following the published HDF5 file-format specification, in the
structures JLD2 itself uses:

* superblock version 2 at offset 0 (48 bytes, Jenkins lookup3 checksum);
* the root group as a version-2 object header ("OHDR") holding a Link Info
  message, a Group Info message and one hard-link message per entry (compact
  "new-style" group storage);
* each entry a dataset with a version-2 object header: dataspace (version 2;
  scalar for the integers and the string, simple with the array's dimensions
  otherwise), datatype (IEEE little-endian float, signed little-endian
  integer, or a null-terminated UTF-8 fixed-length string), fill value
  (version 3) and a contiguous data layout (version 3);
* array data stored contiguously in Julia's column-major order, so the
  HDF5 dimensions are the Julia dimensions reversed — what JLD2 and HDF5.jl
  write for a Julia array and reverse again on reading.

The reader handles these structures and the older ones the HDF5 library
writes by default (superblock version 0, version-1 object headers,
symbol-table groups with a version-1 B-tree, symbol-table nodes and a local
heap; dataspace version 1, data layout versions 1-5), contiguous and compact
datasets of integers, floats, fixed-length strings and JLD2's variable-length
strings (global heap).  It is tested against
a file written by the HDF5 library (and against the checksum's published test
vectors); JLD2 and h5py are not available here, so files written by this
module have been read back only by this reader.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
_M32 = 0xFFFFFFFF


# ---------------------------------------------------------------------------
# Jenkins lookup3 "hashlittle" (Bob Jenkins, 2006, public domain), the
# checksum of every version-2 HDF5 metadata structure (initial value 0).

def _rot(x: int, k: int) -> int:
    return ((x << k) | (x >> (32 - k))) & _M32


def lookup3(data: bytes, initval: int = 0) -> int:
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & _M32
    i = 0
    while n - i > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & _M32
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & _M32
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & _M32
        # mix(a, b, c)
        a = (a - c) & _M32; a ^= _rot(c, 4); c = (c + b) & _M32
        b = (b - a) & _M32; b ^= _rot(a, 6); a = (a + c) & _M32
        c = (c - b) & _M32; c ^= _rot(b, 8); b = (b + a) & _M32
        a = (a - c) & _M32; a ^= _rot(c, 16); c = (c + b) & _M32
        b = (b - a) & _M32; b ^= _rot(a, 19); a = (a + c) & _M32
        c = (c - b) & _M32; c ^= _rot(b, 4); b = (b + a) & _M32
        i += 12
    rest = data[i:]
    if not rest:
        return c
    tail = rest + b"\x00" * (12 - len(rest))
    a = (a + int.from_bytes(tail[0:4], "little")) & _M32
    b = (b + int.from_bytes(tail[4:8], "little")) & _M32
    c = (c + int.from_bytes(tail[8:12], "little")) & _M32
    # final(a, b, c)
    c ^= b; c = (c - _rot(b, 14)) & _M32
    a ^= c; a = (a - _rot(c, 11)) & _M32
    b ^= a; b = (b - _rot(a, 25)) & _M32
    c ^= b; c = (c - _rot(b, 16)) & _M32
    a ^= c; a = (a - _rot(c, 4)) & _M32
    b ^= a; b = (b - _rot(a, 14)) & _M32
    c ^= b; c = (c - _rot(b, 24)) & _M32
    return c


# ---------------------------------------------------------------------------
# Writer

def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    return struct.pack("<BHB", mtype, len(body), flags) + body


def _object_header(messages: list[bytes]) -> bytes:
    """Version-2 object header: no times, no attribute phase values, the
    chunk-0 size in 4 bytes (flags bits 0-1 = 2), then the checksum."""
    body = b"".join(messages)
    head = b"OHDR" + struct.pack("<BBI", 2, 0x02, len(body))
    blob = head + body
    return blob + struct.pack("<I", lookup3(blob))


def _dataspace(dims: tuple[int, ...]) -> bytes:
    if not dims:
        return struct.pack("<BBBB", 2, 0, 0, 0)                  # scalar
    return struct.pack("<BBBB", 2, len(dims), 0, 1) + b"".join(struct.pack("<Q", d) for d in dims)


def _datatype(kind: str, size: int) -> bytes:
    if kind == "f":
        if size == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            bits = bytes([0x20, 63, 0])
        else:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            bits = bytes([0x20, 31, 0])
        return bytes([0x11]) + bits + struct.pack("<I", size) + props
    if kind == "i":
        return bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", size) + struct.pack("<HH", 0, 8 * size)
    if kind == "s":                                                # null-terminated, UTF-8
        return bytes([0x13, 0x10, 0, 0]) + struct.pack("<I", size)
    raise ValueError(kind)


def _fill_value() -> bytes:
    # version 3; allocation time late (2), write time "if set" (2), no value
    return bytes([3, 0x02 | (0x02 << 2)])


def _layout_contiguous(addr: int, size: int) -> bytes:
    return struct.pack("<BBQQ", 3, 1, addr, size)


def _encode(value):
    """(kind, element size, HDF5 dims, payload) of a value; the payload is
    bytes, or for an array a C-contiguous view whose memory is the array in
    Julia's column-major order (written without a copy)."""
    if isinstance(value, str):
        raw = value.encode("utf-8") + b"\x00"
        return "s", len(raw), (), raw
    if isinstance(value, (bool, np.bool_)):
        raise TypeError("booleans are not written")
    if isinstance(value, (int, np.integer)):
        return "i", 8, (), struct.pack("<q", int(value))
    a = np.asarray(value)
    if a.dtype.kind == "f" and a.dtype.itemsize in (4, 8):
        dt = np.dtype("<f8") if a.dtype.itemsize == 8 else np.dtype("<f4")
        kind = "f"
    elif a.dtype.kind in "iu":
        dt, kind = np.dtype("<i8"), "i"
    else:
        raise TypeError(f"cannot write dtype {a.dtype}")
    if a.ndim == 0:
        return kind, dt.itemsize, (), a.astype(dt).tobytes()
    # Julia column-major order; HDF5 lists the slowest dimension first
    view = np.asfortranarray(a, dtype=dt).T
    return kind, dt.itemsize, view.shape, view


def _nbytes(payload) -> int:
    return payload.nbytes if isinstance(payload, np.ndarray) else len(payload)


def write(path: str, items: dict) -> None:
    """Writes ``items`` (name -> str, int, or numpy array in Julia's
    column-major sense) as datasets of the root group of a new HDF5 file."""
    names = list(items)
    for nm in names:
        if not nm or "/" in nm or len(nm.encode("utf-8")) > 255:
            raise ValueError(f"invalid dataset name {nm!r}")
    if len(set(names)) != len(names):
        raise ValueError("duplicate dataset names")
    enc = [_encode(items[nm]) for nm in names]

    def align(x: int) -> int:
        return (x + 7) // 8 * 8

    def dataset_header(k, sz, dims, payload, addr):
        return _object_header([
            _message(1, _dataspace(dims)), _message(3, _datatype(k, sz), 1),
            _message(5, _fill_value(), 1), _message(8, _layout_contiguous(addr, _nbytes(payload)))])

    # layout: superblock, root group header, dataset headers, then the data
    link_msgs_len = sum(4 + 3 + len(nm.encode("utf-8")) + 8 for nm in names)
    root_size = 4 + 6 + (4 + 18) + (4 + 2) + link_msgs_len + 4
    root_addr = 48
    pos = align(root_addr + root_size)
    ds_addr = []
    for e in enc:
        ds_addr.append(pos)
        pos = align(pos + len(dataset_header(*e, 0)))
    data_addr = []
    for e in enc:
        data_addr.append(pos)
        pos = align(pos + _nbytes(e[3]))
    eof = pos

    link_info = struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF)
    group_info = struct.pack("<BB", 0, 0)
    msgs = [_message(2, link_info), _message(10, group_info)]
    for nm, a in zip(names, ds_addr):
        b = nm.encode("utf-8")
        msgs.append(_message(6, struct.pack("<BBB", 1, 0x00, len(b)) + b + struct.pack("<Q", a)))
    root = _object_header(msgs)
    assert len(root) == root_size
    sb = SIGNATURE + struct.pack("<BBBB", 2, 8, 8, 0) + struct.pack("<QQQQ", 0, UNDEF, eof, root_addr)
    with open(path, "wb") as f:
        f.write(sb + struct.pack("<I", lookup3(sb)))
        f.seek(root_addr)
        f.write(root)
        for e, a, d in zip(enc, ds_addr, data_addr):
            f.seek(a)
            f.write(dataset_header(*e, d))
        for e, d in zip(enc, data_addr):
            f.seek(d)
            f.write(e[3].data if isinstance(e[3], np.ndarray) else e[3])
        f.truncate(eof)


# ---------------------------------------------------------------------------
# Reader

class FormatError(ValueError):
    pass


class _File:
    def __init__(self, data: bytes):
        self.d = data
        for off in (0, 512, 1024, 2048, 4096, 8192):
            if data[off:off + 8] == SIGNATURE:
                self.sb = off
                break
        else:
            raise FormatError("no HDF5 superblock signature")
        d, s = data, self.sb
        ver = d[s + 8]
        if ver in (0, 1):
            self.so, self.sl = d[s + 13], d[s + 14]
            if (self.so, self.sl) != (8, 8):
                raise FormatError("only 8-byte offsets and lengths are read")
            p = s + 24 + (4 if ver == 1 else 0)
            self.base = self.q(p)
            root_entry = p + 4 * 8                      # after base, free-space, EOF, driver addresses
            self.root = self.q(root_entry + 8)
        elif ver in (2, 3):
            self.so, self.sl = d[s + 9], d[s + 10]
            if (self.so, self.sl) != (8, 8):
                raise FormatError("only 8-byte offsets and lengths are read")
            if lookup3(d[s:s + 44]) != struct.unpack_from("<I", d, s + 44)[0]:
                raise FormatError("superblock checksum mismatch")
            self.base = self.q(s + 12)
            self.root = self.q(s + 36)
        else:
            raise FormatError(f"superblock version {ver}")

    def q(self, p: int) -> int:
        return struct.unpack_from("<Q", self.d, p)[0]

    def at(self, addr: int) -> int:
        """File position of a (base-relative) address."""
        return self.base + addr

    # -- object headers ------------------------------------------------------
    def messages(self, addr: int) -> list[tuple[int, bytes]]:
        d = self.d
        p = self.at(addr)
        out = []
        if d[p:p + 4] == b"OHDR":
            flags = d[p + 5]
            q = p + 6
            if flags & 0x20:
                q += 16
            if flags & 0x10:
                q += 4
            w = 1 << (flags & 3)
            size = int.from_bytes(d[q:q + w], "little")
            q += w
            chunks = [(p, q, q + size)]
            while chunks:
                start, q, end = chunks.pop(0)
                if lookup3(d[start:end]) != struct.unpack_from("<I", d, end)[0]:
                    raise FormatError("object header checksum mismatch")
                while q + 4 <= end:
                    mtype, msize, _mflags = struct.unpack_from("<BHB", d, q)
                    q += 4 + (2 if flags & 0x04 else 0)
                    body = d[q:q + msize]
                    q += msize
                    if mtype == 0x10:                     # continuation
                        caddr, clen = struct.unpack_from("<QQ", body, 0)
                        cp = self.at(caddr)
                        if d[cp:cp + 4] != b"OCHK":
                            raise FormatError("bad continuation chunk")
                        chunks.append((cp, cp + 4, cp + clen - 4))
                    elif mtype != 0:
                        out.append((mtype, body))
            return out
        if d[p] != 1:
            raise FormatError(f"object header version {d[p]}")
        nmsg, _refs, size = struct.unpack_from("<HII", d, p + 2)
        chunks = [(p + 16, p + 16 + size)]
        count = 0
        while chunks and count < nmsg:
            q, end = chunks.pop(0)
            while q + 8 <= end and count < nmsg:
                mtype, msize, _mflags = struct.unpack_from("<HHB", d, q)
                body = d[q + 8:q + 8 + msize]
                q += 8 + msize
                count += 1
                if mtype == 0x10:
                    caddr, clen = struct.unpack_from("<QQ", body, 0)
                    chunks.append((self.at(caddr), self.at(caddr) + clen))
                elif mtype != 0:
                    out.append((mtype, body))
        return out

    # -- groups --------------------------------------------------------------
    def links(self, addr: int) -> dict[str, int]:
        msgs = self.messages(addr)
        found = {}
        for mtype, body in msgs:
            if mtype == 0x06:
                name, target = self._link(body)
                if target is not None:
                    found[name] = target
            elif mtype == 0x02:
                if struct.unpack_from("<Q", body, 2 + (8 if body[1] & 1 else 0))[0] != UNDEF:
                    raise FormatError("dense link storage (fractal heap) is not read")
            elif mtype == 0x11:
                btree, heap = struct.unpack_from("<QQ", body, 0)
                found.update(self._symbol_table(btree, heap))
        return found

    @staticmethod
    def _link(body: bytes):
        flags = body[1]
        p = 2
        ltype = 0
        if flags & 0x08:
            ltype = body[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        w = 1 << (flags & 3)
        ln = int.from_bytes(body[p:p + w], "little")
        p += w
        name = body[p:p + ln].decode("utf-8")
        p += ln
        if ltype != 0:
            return name, None                             # soft / external links are skipped
        return name, struct.unpack_from("<Q", body, p)[0]

    def _heap_name(self, heap: int, off: int) -> str:
        d = self.d
        h = self.at(heap)
        if d[h:h + 4] != b"HEAP":
            raise FormatError("bad local heap")
        data = self.at(self.q(h + 24))
        end = d.index(b"\x00", data + off)
        return d[data + off:end].decode("utf-8")

    def _symbol_table(self, btree: int, heap: int) -> dict[str, int]:
        d = self.d
        out = {}
        stack = [btree]
        while stack:
            p = self.at(stack.pop())
            if d[p:p + 4] == b"TREE":
                ntype, used = d[p + 4], struct.unpack_from("<H", d, p + 6)[0]
                if ntype != 0:
                    raise FormatError("not a group B-tree")
                q = p + 24 + 8                            # past the siblings and key 0
                children = [self.q(q + 16 * c) for c in range(used)]
                stack.extend(reversed(children))          # visited in key (name) order
            elif d[p:p + 4] == b"SNOD":
                nsym = struct.unpack_from("<H", d, p + 6)[0]
                q = p + 8
                for _ in range(nsym):
                    name_off, oh = struct.unpack_from("<QQ", d, q)
                    out[self._heap_name(heap, name_off)] = oh
                    q += 40
            else:
                raise FormatError("bad group node")
        return out

    # -- datasets ------------------------------------------------------------
    def dataset(self, addr: int):
        space = dtype = layout = None
        for mtype, body in self.messages(addr):
            if mtype == 0x01:
                space = self._dataspace(body)
            elif mtype == 0x03:
                dtype = self._datatype(body)
            elif mtype == 0x08:
                layout = body
        if space is None or dtype is None or layout is None:
            raise FormatError("not a dataset")
        count = int(np.prod(space)) if space else 1
        raw = self._data(layout, count * dtype[1])
        kind, size, np_dt = dtype
        if kind in ("s", "vs"):
            if kind == "s":
                vals = [raw[i * size:(i + 1) * size].split(b"\x00", 1)[0].rstrip(b" ").decode("utf-8")
                        for i in range(count)]
            else:
                vals = [self._vlen(raw[i * size:(i + 1) * size]).decode("utf-8") for i in range(count)]
            return vals[0] if not space else np.array(vals, dtype=object).reshape(tuple(reversed(space)), order="F")
        arr = np.frombuffer(raw, dtype=np_dt, count=count)
        if not space:
            return arr[0].item()
        return arr.reshape(tuple(reversed(space)), order="F")

    @staticmethod
    def _dataspace(body: bytes) -> tuple[int, ...]:
        ver, rank = body[0], body[1]
        if ver == 1:
            p = 8
        elif ver == 2:
            if body[3] == 2:
                raise FormatError("null dataspace")
            p = 4
        else:
            raise FormatError(f"dataspace version {ver}")
        return tuple(struct.unpack_from("<Q", body, p + 8 * i)[0] for i in range(rank))

    @staticmethod
    def _datatype(body: bytes):
        cls = body[0] & 0x0F
        bits = body[1] | (body[2] << 8) | (body[3] << 16)
        size = struct.unpack_from("<I", body, 4)[0]
        order = ">" if bits & 1 else "<"
        if cls == 0:
            return "i", size, np.dtype(f"{order}{'i' if bits & 0x08 else 'u'}{size}")
        if cls == 1:
            if size not in (4, 8):
                raise FormatError(f"{size}-byte floats are not read")
            return "f", size, np.dtype(f"{order}f{size}")
        if cls == 3:
            return "s", size, None
        if cls == 9 and (bits & 0x0F) == 1:   # variable-length string (JLD2's String)
            return "vs", 16, None
        raise FormatError(f"datatype class {cls} is not read")

    def _vlen(self, elem: bytes) -> bytes:
        """A variable-length element: its length, then the global heap
        collection's address and the object's index in it."""
        length, coll, index = struct.unpack_from("<IQI", elem, 0)
        if length == 0:
            return b""
        d = self.d
        p = self.at(coll)
        if d[p:p + 4] != b"GCOL":
            raise FormatError("bad global heap collection")
        end = p + struct.unpack_from("<Q", d, p + 8)[0]
        q = p + 16
        while q + 16 <= end:
            idx, _refs, _res, size = struct.unpack_from("<HHIQ", d, q)
            if idx == 0:
                break
            if idx == index:
                return d[q + 16:q + 16 + min(length, size)]
            q += 16 + (size + 7) // 8 * 8
        raise FormatError("global heap object not found")

    def _data(self, body: bytes, nbytes: int) -> bytes:
        ver = body[0]
        if ver in (1, 2):
            ndims, cls = body[1], body[2]
            if cls == 1:
                addr = struct.unpack_from("<Q", body, 8)[0]
                p = self.at(addr)
                return self.d[p:p + nbytes]
            if cls == 0:
                p = 8 + 4 * ndims
                size = struct.unpack_from("<I", body, p)[0]
                return body[p + 4:p + 4 + min(size, nbytes)]
            raise FormatError("chunked layout is not read")
        if ver in (3, 4, 5):                      # compact and contiguous are alike in 3-5
            cls = body[1]
            if cls == 0:
                size = struct.unpack_from("<H", body, 2)[0]
                return body[4:4 + min(size, nbytes)]
            if cls == 1:
                addr = struct.unpack_from("<Q", body, 2)[0]
                if addr == UNDEF:
                    return b"\x00" * nbytes
                p = self.at(addr)
                return self.d[p:p + nbytes]
            raise FormatError("chunked layout is not read")
        raise FormatError(f"data layout version {ver}")


def read(path: str) -> dict:
    """Every dataset of the root group: name -> str, int, float or numpy
    array (Julia's column-major shape: the HDF5 dimensions reversed)."""
    with open(path, "rb") as f:
        data = f.read()
    h = _File(data)
    return {name: h.dataset(addr) for name, addr in h.links(h.root).items()}
