"""A small read-only HDF5 reader for files in h5py's default ("earliest") format: the reference's
bundled ``.h5`` coils and its ``.h5`` field results load where h5py is not installed.
``read_dataset`` reads one dataset of the root group; ``read_tree`` reads the whole file (groups,
their attributes, numeric datasets).

Written from the HDF5 File Format Specification (version 0 superblock), covering what such files
use: a version-0 superblock with 8-byte offsets and lengths; groups as symbol tables (version-1
B-tree of group nodes, symbol-table nodes, local heap); version-1 object headers with continuation
blocks; the dataspace, datatype, data layout (version 3: compact, contiguous, chunked), filter
pipeline (deflate, shuffle) and attribute messages; raw-data-chunk B-trees; numeric data
(little- or big-endian integers and IEEE floats) and fixed- or variable-length strings (the latter
through global-heap collections). Anything else raises ``ValueError`` naming what is missing.
"""

from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

_SIGNATURE = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class _File:
    def __init__(self, data: bytes) -> None:
        self.d = data

    def u(self, fmt: str, off: int):
        return struct.unpack_from("<" + fmt, self.d, off)

    def sig(self, off: int, s: bytes) -> None:
        if self.d[off:off + len(s)] != s:
            raise ValueError(f"HDF5: expected {s!r} at offset {off}")

    # --- groups -----------------------------------------------------------------------------

    def local_heap_name(self, heap: int, offset: int) -> str:
        self.sig(heap, b"HEAP")
        data_addr = self.u("Q", heap + 24)[0]
        start = data_addr + offset
        end = self.d.index(b"\x00", start)
        return self.d[start:end].decode()

    def group_entries(self, btree: int, heap: int, _seen: set[int] | None = None) -> dict[str, int]:
        """name -> object header address over a version-1 B-tree of group nodes. A node reached a
        second time (a cycle in a malformed file) raises ValueError."""
        seen = set() if _seen is None else _seen
        if btree in seen:
            raise ValueError(f"HDF5: group B-tree node at {btree} is reached twice")
        seen.add(btree)
        out: dict[str, int] = {}
        self.sig(btree, b"TREE")
        node_type, level, used = self.d[btree + 4], self.d[btree + 5], self.u("H", btree + 6)[0]
        if node_type != 0:
            raise ValueError("HDF5: a group B-tree must hold group nodes")
        q = btree + 24 + 8  # past the header and key 0
        for _ in range(used):
            child = self.u("Q", q)[0]
            q += 16  # child address, then the next key
            if level > 0:
                out.update(self.group_entries(child, heap, seen))
                continue
            self.sig(child, b"SNOD")
            n_sym = self.u("H", child + 6)[0]
            for i in range(n_sym):
                e = child + 8 + 40 * i
                name_off, header = self.u("QQ", e)
                out[self.local_heap_name(heap, name_off)] = header
        return out

    # --- object headers ---------------------------------------------------------------------

    def messages(self, header: int) -> list[tuple[int, int, int]]:
        """(type, offset of its data, size) of every message of a version-1 object header."""
        if self.d[header] != 1:
            raise ValueError("HDF5: only version-1 object headers are handled")
        n_msg, _refs, size = self.u("HII", header + 2)
        blocks = [(header + 16, size)]
        out = []
        while blocks and len(out) < n_msg:
            start, length = blocks.pop(0)
            q = start
            while q + 8 <= start + length and len(out) < n_msg:
                mtype, msize = self.u("HH", q)
                if mtype == 0x10:  # continuation: another block of messages
                    blocks.append(self.u("QQ", q + 8))
                out.append((mtype, q + 8, msize))
                q += 8 + msize
        return out

    def dataspace(self, off: int) -> tuple[int, ...]:
        version, ndim, flags = self.d[off], self.d[off + 1], self.d[off + 2]
        if version == 1:
            dims_at = off + 8
        elif version == 2:
            dims_at = off + 4
            if self.d[off + 3] == 0:  # scalar
                return ()
        else:
            raise ValueError(f"HDF5: dataspace message version {version}")
        return tuple(self.u(f"{ndim}Q", dims_at)) if ndim else ()

    def datatype(self, off: int) -> dict:
        cv = self.d[off]
        cls = cv & 0x0F
        bits = self.d[off + 1] | (self.d[off + 2] << 8) | (self.d[off + 3] << 16)
        size = self.u("I", off + 4)[0]
        order = ">" if bits & 1 else "<"
        if cls == 0:
            return {"kind": "num", "dtype": np.dtype(f"{order}{'i' if bits & 8 else 'u'}{size}"), "size": size}
        if cls == 1:
            return {"kind": "num", "dtype": np.dtype(f"{order}f{size}"), "size": size}
        if cls == 3:
            return {"kind": "fstr", "size": size}
        if cls == 9:
            if bits & 0x0F != 1:
                raise ValueError("HDF5: variable-length sequences other than strings")
            return {"kind": "vstr", "size": size}
        raise ValueError(f"HDF5: datatype class {cls}")

    def global_heap_object(self, collection: int, index: int) -> bytes:
        self.sig(collection, b"GCOL")
        total = self.u("Q", collection + 8)[0]
        q, end = collection + 16, collection + total
        while q + 16 <= end:
            idx, _refs, _res, osize = self.u("HHIQ", q)
            if idx == 0:
                break
            if idx == index:
                return self.d[q + 16:q + 16 + osize]
            q += 16 + ((osize + 7) // 8) * 8
        raise ValueError("HDF5: global heap object not found")

    def values(self, dtype: dict, shape: tuple[int, ...], off: int):
        n = int(np.prod(shape)) if shape else 1
        if dtype["kind"] == "num":
            a = np.frombuffer(self.d, dtype=dtype["dtype"], count=n, offset=off)
            a = a.astype(dtype["dtype"].newbyteorder("="))
            return a.reshape(shape) if shape else a[0].item()
        if dtype["kind"] == "fstr":
            s = [self.d[off + i * dtype["size"]:off + (i + 1) * dtype["size"]].split(b"\x00")[0].decode()
                 for i in range(n)]
        else:
            s = []
            for i in range(n):
                _length, coll, index = self.u("IQI", off + 16 * i)
                s.append(self.global_heap_object(coll, index).decode())
        return s if shape else s[0]

    def attribute(self, off: int) -> tuple[str, object]:
        version = self.d[off]
        name_size, type_size, space_size = self.u("HHH", off + 2)
        if version == 1:
            pad = lambda x: (x + 7) // 8 * 8  # noqa: E731
            q = off + 8
        elif version in (2, 3):
            pad = lambda x: x  # noqa: E731
            q = off + 8 + (1 if version == 3 else 0)
        else:
            raise ValueError(f"HDF5: attribute message version {version}")
        name = self.d[q:q + name_size].split(b"\x00")[0].decode()
        q += pad(name_size)
        dtype = self.datatype(q)
        q += pad(type_size)
        shape = self.dataspace(q)
        q += pad(space_size)
        return name, self.values(dtype, shape, q)

    def chunk_index(self, btree: int, ndim: int) -> list[tuple[tuple[int, ...], int, int, int]]:
        """(offset, filter mask, size, address) of every chunk of a raw-data-chunk B-tree."""
        self.sig(btree, b"TREE")
        node_type, level, used = self.d[btree + 4], self.d[btree + 5], self.u("H", btree + 6)[0]
        if node_type != 1:
            raise ValueError("HDF5: a chunk B-tree must hold raw-data chunks")
        key = 8 + 8 * (ndim + 1)
        out = []
        q = btree + 24
        for _ in range(used):
            size, mask = self.u("II", q)
            offs = self.u(f"{ndim}Q", q + 8)
            child = self.u("Q", q + key)[0]
            if level > 0:
                out += self.chunk_index(child, ndim)
            else:
                out.append((offs, mask, size, child))
            q += key + 8
        return out

    def dataset(self, header: int) -> tuple[np.ndarray, dict]:
        shape = dtype = layout = None
        filters: list[int] = []
        attrs: dict = {}
        for mtype, off, _size in self.messages(header):
            if mtype == 0x01:
                shape = self.dataspace(off)
            elif mtype == 0x03:
                dtype = self.datatype(off)
            elif mtype == 0x08:
                layout = off
            elif mtype == 0x0B:
                filters = self.filter_ids(off)
            elif mtype == 0x0C:
                k, v = self.attribute(off)
                attrs[k] = v
        if shape is None or dtype is None or layout is None or dtype["kind"] != "num":
            raise ValueError("HDF5: not a numeric dataset")
        return self.read_layout(layout, shape, dtype["dtype"], filters), attrs

    def filter_ids(self, off: int) -> list[int]:
        version, n = self.d[off], self.d[off + 1]
        q = off + (8 if version == 1 else 2)
        ids = []
        for _ in range(n):
            fid = self.u("H", q)[0]
            if version == 1 or fid >= 256:
                name_len, _flags, n_val = self.u("HHH", q + 2)
                q += 8 + ((name_len + 7) // 8 * 8 if version == 1 else name_len)
            else:
                _flags, n_val = self.u("HH", q + 2)
                q += 6
            q += 4 * n_val + (4 if version == 1 and n_val % 2 else 0)
            ids.append(fid)
        return ids

    def read_layout(self, off: int, shape: tuple[int, ...], dt: np.dtype, filters: list[int]) -> np.ndarray:
        version, cls = self.d[off], self.d[off + 1]
        if version != 3:
            raise ValueError(f"HDF5: data layout message version {version}")
        n = int(np.prod(shape))
        if cls == 0:  # compact
            size = self.u("H", off + 2)[0]
            raw = self.d[off + 4:off + 4 + size]
            return np.frombuffer(raw, dtype=dt, count=n).astype(dt.newbyteorder("=")).reshape(shape)
        if cls == 1:  # contiguous
            addr = self.u("Q", off + 2)[0]
            if n == 0 or addr == _UNDEF:  # no storage allocated: empty, or never written (fill value 0)
                return np.zeros(shape, dtype=dt.newbyteorder("="))
            return np.frombuffer(self.d, dtype=dt, count=n, offset=addr).astype(dt.newbyteorder("=")).reshape(shape)
        if cls != 2:
            raise ValueError(f"HDF5: layout class {cls}")
        ndim = self.d[off + 2] - 1  # the last chunk dimension is the element size
        btree = self.u("Q", off + 3)[0]
        cdims = self.u(f"{ndim}I", off + 11)
        out = np.zeros(shape, dtype=dt.newbyteorder("="))
        if btree == _UNDEF:
            return out
        for offs, mask, size, addr in self.chunk_index(btree, ndim):
            raw = self.d[addr:addr + size]
            for i, fid in reversed(list(enumerate(filters))):
                if mask & (1 << i):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:  # shuffle: bytes grouped by position within the element
                    raw = np.frombuffer(raw, np.uint8).reshape(dt.itemsize, -1).T.tobytes()
                else:
                    raise ValueError(f"HDF5: filter {fid}")
            chunk = np.frombuffer(raw, dtype=dt).astype(dt.newbyteorder("=")).reshape(cdims)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
            out[sl] = chunk[tuple(slice(0, x.stop - x.start) for x in sl)]
        return out


    def group(self, header: int, depth: int = 0, _seen: set[int] | None = None) -> dict:
        """A group's attributes, datasets (array, attributes) and subgroups, read recursively. A group
        whose object header comes round again (links forming a cycle) raises ValueError."""
        if depth > 32:
            raise ValueError("HDF5: groups nested deeper than 32 levels")
        seen = set() if _seen is None else _seen
        if header in seen:
            raise ValueError(f"HDF5: the group object header at {header} is reached twice (a cycle)")
        seen.add(header)
        table, attrs = None, {}
        for mtype, off, _size in self.messages(header):
            if mtype == 0x11:
                table = self.u("QQ", off)
            elif mtype == 0x0C:
                k, v = self.attribute(off)
                attrs[k] = v
        if table is None:
            raise ValueError("HDF5: a group object header without a symbol table message")
        out = {"attrs": attrs, "datasets": {}, "groups": {}}
        for name, child in self.group_entries(*table).items():
            if any(mtype == 0x11 for mtype, _, _ in self.messages(child)):
                out["groups"][name] = self.group(child, depth + 1, seen)
            else:
                out["datasets"][name] = self.dataset(child)
        return out


def _open(path: str | Path) -> _File:
    f = _File(Path(path).read_bytes())
    f.sig(0, _SIGNATURE)
    if f.d[8] != 0:
        raise ValueError(f"HDF5: superblock version {f.d[8]} (only version 0 is handled)")
    if f.d[13] != 8 or f.d[14] != 8:
        raise ValueError("HDF5: only 8-byte offsets and lengths are handled")
    return f


def is_hdf5(path: str | Path) -> bool:
    with open(path, "rb") as fh:
        return fh.read(len(_SIGNATURE)) == _SIGNATURE


def _malformed(fn):
    """Reads past the end of the file, zlib errors, runaway recursion and the reader's own
    structural errors surface as ValueError naming the file."""
    import functools

    @functools.wraps(fn)
    def wrapper(path, *args):
        try:
            return fn(path, *args)
        except (struct.error, IndexError, zlib.error, RecursionError) as exc:
            raise ValueError(f"HDF5: {path} is truncated or malformed ({exc})") from exc
        except ValueError as exc:
            if str(path) in str(exc):
                raise
            raise ValueError(f"HDF5: {path} is malformed ({exc})") from exc

    return wrapper


@_malformed
def read_dataset(path: str | Path, name: str) -> tuple[np.ndarray, dict]:
    """The dataset ``name`` of the root group of an HDF5 file and its attributes."""
    f = _open(path)
    root_cache = f.u("I", 56 + 16)[0]
    if root_cache != 1:
        raise ValueError("HDF5: the root group has no cached symbol table")
    btree, heap = f.u("QQ", 56 + 24)
    entries = f.group_entries(btree, heap)
    if name not in entries:
        raise KeyError(f"{path}: no dataset {name!r} in the root group (has {sorted(entries)})")
    return f.dataset(entries[name])


@_malformed
def read_tree(path: str | Path) -> dict:
    """The whole file from the root group: ``{"attrs": {...}, "datasets": {name: (array, attrs)},
    "groups": {name: <the same for the subgroup>}}``."""
    f = _open(path)
    return f.group(f.u("Q", 56 + 8)[0])


# --- writing -------------------------------------------------------------------------------------
#
# The writer produces the same structures the reader handles and h5py's default ("earliest")
# format uses, as the bundled coil files show them: a version-0 superblock (8-byte offsets and
# lengths, group leaf K 4, internal K 16); each group an object header holding a symbol-table
# message and its attributes, with a one-node version-1 B-tree (allocated at full size), symbol
# table nodes of up to 8 entries, names sorted, and a local heap; each dataset an object header with
# dataspace (version 1), datatype, fill value (version 2) and contiguous layout (version 3)
# messages and its attributes; strings as variable-length UTF-8 strings in one global heap
# collection, as h5py writes Python strings. Numeric data is written little-endian.

_GROUP_LEAF_K = 4
_GROUP_INTERNAL_K = 16
_BTREE_NODE_BYTES = 24 + (2 * _GROUP_INTERNAL_K + 1) * 8 + 2 * _GROUP_INTERNAL_K * 8
_SNOD_BYTES = 8 + 2 * _GROUP_LEAF_K * 40
_VLEN_STR_TYPE = bytes.fromhex("1901010010000000") + bytes.fromhex("100000000100000000000800")


def _pad8(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 8)


def _dtype_message(dt: np.dtype) -> bytes:
    dt = np.dtype(dt).newbyteorder("<") if np.dtype(dt).byteorder == ">" else np.dtype(dt)
    size = dt.itemsize
    if dt.kind == "f":
        if size == 8:
            bits, exp_loc, exp_size, mant_size, bias = 0x3F20, 52, 11, 52, 1023
        elif size == 4:
            bits, exp_loc, exp_size, mant_size, bias = 0x1F20, 23, 8, 23, 127
        else:
            raise ValueError(f"HDF5 writer: float of {size} bytes")
        return struct.pack("<B3sI", 0x11, bits.to_bytes(3, "little"), size) + struct.pack(
            "<HHBBBBI", 0, 8 * size, exp_loc, exp_size, 0, mant_size, bias)
    if dt.kind in "iu" or dt.kind == "b":
        signed = 0x08 if dt.kind == "i" else 0x00
        return struct.pack("<B3sI", 0x10, bytes([signed, 0, 0]), size) + struct.pack("<HH", 0, 8 * size)
    raise ValueError(f"HDF5 writer: dtype {dt}")


def _dataspace_message(shape: tuple[int, ...]) -> bytes:
    return struct.pack("<BBBBI", 1, len(shape), 0, 0, 0) + b"".join(struct.pack("<Q", int(n)) for n in shape)


class _Writer:
    def __init__(self) -> None:
        self.buf = bytearray(96)  # the superblock goes first, written last
        self.strings: list[bytes] = []
        self.gcol_at: int | None = None
        self.pending_vlen: list[tuple[int, int]] = []  # (where a heap ID's address goes, string index)

    def alloc(self, data: bytes) -> int:
        at = len(self.buf)
        self.buf += _pad8(bytes(data))
        return at

    def vlen_string(self, s: str) -> bytes:
        """The 16-byte on-disk reference to a global-heap string (address patched at the end)."""
        b = s.encode()
        self.strings.append(b)
        return struct.pack("<IQI", len(b), 0, len(self.strings))

    def attribute_message(self, name: str, value) -> bytes:
        nm = name.encode() + b"\x00"
        vlen_slots = []
        if isinstance(value, str):
            dtm, space = _VLEN_STR_TYPE, _dataspace_message(())
            data = self.vlen_string(value)
            vlen_slots.append(4)
        elif isinstance(value, (list, tuple)) and value and all(isinstance(v, str) for v in value):
            dtm, space = _VLEN_STR_TYPE, _dataspace_message((len(value),))
            parts = []
            for i, v in enumerate(value):
                parts.append(self.vlen_string(v))
                vlen_slots.append(16 * i + 4)
            data = b"".join(parts)
        else:
            a = np.asarray(value)
            if a.dtype == bool:
                a = a.astype(np.int8)
            if a.dtype.kind not in "iuf":
                raise ValueError(f"HDF5 writer: attribute {name!r} of type {a.dtype}")
            a = a.astype(a.dtype.newbyteorder("<"))
            dtm, space, data = _dtype_message(a.dtype), _dataspace_message(a.shape), a.tobytes()
        head = struct.pack("<BBHHH", 1, 0, len(nm), len(dtm), len(space))
        body = head + _pad8(nm) + _pad8(dtm) + _pad8(space)
        data_at = len(body)
        msg = _pad8(body + data)
        return msg, [data_at + s for s in vlen_slots]

    def object_header(self, messages: list[tuple[int, bytes, int]], vlen_fixups: list[list[int]]) -> int:
        """messages: (type, data, flags); vlen_fixups[i]: offsets in message i's data that hold a
        global-heap collection address. Returns the header's address."""
        block = bytearray()
        fix_at = []
        for (mtype, data, flags), fixes in zip(messages, vlen_fixups):
            data = _pad8(data)
            start = len(block) + 8
            block += struct.pack("<HHB3x", mtype, len(data), flags) + data
            fix_at += [start + f for f in fixes]
        prefix = struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(block))
        at = self.alloc(prefix + bytes(block))
        self.pending_vlen += [(at + 16 + f, 0) for f in fix_at]
        return at

    def dataset(self, arr: np.ndarray, attrs: dict) -> int:
        a = np.ascontiguousarray(arr)
        if a.dtype == bool:
            a = a.astype(np.int8)
        a = a.astype(a.dtype.newbyteorder("<"))
        raw_at = self.alloc(a.tobytes()) if a.nbytes else _UNDEF
        msgs = [(0x01, _dataspace_message(a.shape), 0), (0x03, _dtype_message(a.dtype), 1),
                (0x05, bytes([2, 2, 2, 0]), 1),
                (0x08, struct.pack("<BBQQ", 3, 1, raw_at, a.nbytes), 0)]
        fixes: list[list[int]] = [[], [], [], []]
        for k, v in attrs.items():
            m, f = self.attribute_message(k, v)
            msgs.append((0x0C, m, 0))
            fixes.append(f)
        return self.object_header(msgs, fixes)

    def group(self, tree: dict) -> tuple[int, int, int]:
        """Writes a group and everything under it; returns (header, B-tree, local heap) addresses."""
        children: dict[str, tuple[int, bool, tuple[int, int]]] = {}
        for name, item in tree.get("datasets", {}).items():
            arr, attrs = item if isinstance(item, tuple) else (item, {})
            children[name] = (self.dataset(arr, attrs), False, (0, 0))
        for name, sub in tree.get("groups", {}).items():
            hdr, bt, hp = self.group(sub)
            children[name] = (hdr, True, (bt, hp))
        names = sorted(children, key=lambda s: s.encode())
        if len(names) > 2 * _GROUP_LEAF_K * 2 * _GROUP_INTERNAL_K:
            raise ValueError("HDF5 writer: more than 256 members in one group")
        # Local heap: "" at 0, then the names, each null-terminated and padded to 8 bytes.
        heap_data = bytearray(8)
        offset = {}
        for n in names:
            offset[n] = len(heap_data)
            heap_data += _pad8(n.encode() + b"\x00")
        # Symbol table nodes of up to 2 * leaf K entries each.
        snods, keys = [], [0]
        for s in range(0, len(names), 2 * _GROUP_LEAF_K):
            part = names[s:s + 2 * _GROUP_LEAF_K]
            node = bytearray(b"SNOD" + struct.pack("<BBH", 1, 0, len(part)))
            for n in part:
                hdr, is_group, (bt, hp) = children[n]
                node += struct.pack("<QQII", offset[n], hdr, 1 if is_group else 0, 0)
                node += struct.pack("<QQ", bt, hp) if is_group else bytes(16)
            node += bytes(_SNOD_BYTES - len(node))
            snods.append(self.alloc(bytes(node)))
            keys.append(offset[part[-1]])
        btree = bytearray(b"TREE" + struct.pack("<BBHQQ", 0, 0, len(snods), _UNDEF, _UNDEF))
        for i, child in enumerate(snods):
            btree += struct.pack("<QQ", keys[i], child)
        btree += struct.pack("<Q", keys[len(snods)])
        btree += bytes(_BTREE_NODE_BYTES - len(btree))
        bt_at = self.alloc(bytes(btree))
        heap_at = len(self.buf)
        self.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), _UNDEF, heap_at + 32))
        self.alloc(bytes(heap_data))
        msgs = [(0x11, struct.pack("<QQ", bt_at, heap_at), 0)]
        fixes: list[list[int]] = [[]]
        for k, v in tree.get("attrs", {}).items():
            m, f = self.attribute_message(k, v)
            msgs.append((0x0C, m, 0))
            fixes.append(f)
        return self.object_header(msgs, fixes), bt_at, heap_at

    def finish(self, root: tuple[int, int, int]) -> bytes:
        if self.strings:
            objs = bytearray()
            for i, b in enumerate(self.strings, start=1):
                objs += struct.pack("<HHIQ", i, 0, 0, len(b)) + _pad8(b)
            size = max(4096, 16 + len(objs) + 16)
            gcol = bytearray(b"GCOL" + struct.pack("<B3xQ", 1, size)) + objs
            free = size - len(gcol)
            gcol += struct.pack("<HHIQ", 0, 0, 0, free) + bytes(free - 16)
            self.gcol_at = self.alloc(bytes(gcol))
            for where, _ in self.pending_vlen:
                struct.pack_into("<Q", self.buf, where, self.gcol_at)
        hdr, bt, hp = root
        sb = bytearray(_SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]))
        sb += struct.pack("<HHI", _GROUP_LEAF_K, _GROUP_INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, _UNDEF, len(self.buf), _UNDEF)
        sb += struct.pack("<QQII", 0, hdr, 1, 0) + struct.pack("<QQ", bt, hp)
        self.buf[0:96] = sb
        return bytes(self.buf)


def write_tree(path: str | Path, tree: dict) -> None:
    """Writes ``tree`` -- ``{"attrs": {...}, "datasets": {name: array or (array, attrs)},
    "groups": {name: <the same>}}``, the form ``read_tree`` returns -- as an HDF5 file. Attribute
    values may be str (stored as variable-length UTF-8 strings), lists of str, or numbers and
    numeric arrays; datasets are numeric arrays (stored contiguous, uncompressed)."""
    w = _Writer()
    root = w.group(tree)
    Path(path).write_bytes(w.finish(root))
