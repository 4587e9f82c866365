"""Reader of the JLD2 (HDF5-based) files gtdgl writes: its checkpoints (``save_state``, gtdgl/src/io.jl:131-154,
written with ``compress=true``) and the golden files of its test suite.

Only what those files use is implemented: superblock v2/v3, object
headers v2 (with continuation chunks), contiguous / compact / chunked(deflate) layouts, the datatype
classes fixed-point, float, string, compound, reference and variable-length, committed (shared)
datatypes, and the global heap for variable-length strings.  JLD2 conventions on top of HDF5:

* addresses are relative to the superblock's base address (the 512-byte JLD2 header);
* a Julia array of size (n1, n2, n3) is stored with HDF5 dims (n3, n2, n1), so the raw bytes are the
  column-major Julia array (``order="F"`` with the reversed HDF5 dims);
* ``Dict{String,Any}`` is a ``JLD2.SerializedDict`` whose ``kvvec`` is a vector of ``Pair{String,Any}``
  (a vlen string and an object reference to the value).

`juliatdgl_b200.checkpoint.load` reads a reference checkpoint with it, and `tests/golden/make_fixtures.py` turns
the reference's golden data into numpy fixtures.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np


class _Dtype:
    def __init__(self, cls, size, **kw):
        self.cls = cls
        self.size = size
        self.__dict__.update(kw)

    def __repr__(self):
        return f"_Dtype(cls={self.cls}, size={self.size})"


class JLD2File:
    def __init__(self, path):
        with open(path, "rb") as fh:
            self.buf = fh.read()
        sb = self.buf.find(b"\x89HDF\r\n\x1a\n")
        if sb < 0:
            raise ValueError("not an HDF5/JLD2 file")
        ver = self.buf[sb + 8]
        if ver not in (2, 3):
            raise ValueError(f"superblock version {ver} not supported")
        so, sl = self.buf[sb + 9], self.buf[sb + 10]
        assert so == 8 and sl == 8
        self.base, _ext, _eof, self.root = struct.unpack_from("<4Q", self.buf, sb + 12)
        self._gheap = {}

    # ---------------------------------------------------------------- object headers
    def _abs(self, addr):
        return self.base + addr

    def _messages(self, addr):
        b = self.buf
        p = self._abs(addr)
        if b[p:p + 4] != b"OHDR":
            raise ValueError(f"expected OHDR at {addr:#x}")
        flags = b[p + 5]
        q = p + 6
        if flags & 0x20:
            q += 16
        if flags & 0x10:
            q += 4
        nsz = 1 << (flags & 3)
        size = int.from_bytes(b[q:q + nsz], "little")
        q += nsz
        chunks = [(q, q + size)]
        msgs = []
        while chunks:
            start, end = chunks.pop(0)
            r = start
            while r + 4 <= end:
                mtype = b[r]
                msize = struct.unpack_from("<H", b, r + 1)[0]
                mflags = b[r + 3]
                r += 4
                if flags & 0x04:
                    r += 2
                data = b[r:r + msize]
                r += msize
                if mtype == 0x10:
                    off, ln = struct.unpack_from("<2Q", data, 0)
                    cp = self._abs(off)
                    assert b[cp:cp + 4] == b"OCHK"
                    chunks.append((cp + 4, cp + ln - 4))
                else:
                    msgs.append((mtype, mflags, data))
        return msgs

    # ---------------------------------------------------------------- datatypes
    def _datatype(self, data, off=0):
        """Parse a datatype description at data[off:]; return (dtype, bytes consumed)."""
        cv = data[off]
        cls, ver = cv & 0x0F, cv >> 4
        bits = data[off + 1] | (data[off + 2] << 8) | (data[off + 3] << 16)
        size = struct.unpack_from("<I", data, off + 4)[0]
        p = off + 8
        if cls == 0:  # fixed point
            signed = bool(bits & 0x08)
            p += 4
            return _Dtype(0, size, signed=signed), p - off
        if cls == 4:  # bitfield (JLD2 writes Bool as one)
            p += 4
            return _Dtype(0, size, signed=False), p - off
        if cls == 1:  # float
            p += 12
            return _Dtype(1, size), p - off
        if cls == 3:  # fixed string
            return _Dtype(3, size), p - off
        if cls == 5:  # opaque
            tag_end = data.index(b"\x00", p)
            p = tag_end + 1
            p += (-(p - off - 8)) % 8
            return _Dtype(5, size), p - off
        if cls == 6:  # compound
            nmem = bits & 0xFFFF
            members = []
            for _ in range(nmem):
                e = data.index(b"\x00", p)
                name = data[p:e].decode()
                if ver < 3:
                    p = e + 1
                    p += (-(p - off - 8)) % 8 if ver == 1 else (-(p - (off + 8))) % 8
                    moff = struct.unpack_from("<I", data, p)[0]
                    p += 4
                    if ver == 1:
                        p += 1 + 3 + 4 + 4 + 16
                else:
                    p = e + 1
                    nb = max(1, (size.bit_length() + 7) // 8)
                    moff = int.from_bytes(data[p:p + nb], "little")
                    p += nb
                mt, used = self._datatype(data, p)
                p += used
                members.append((name, moff, mt))
            return _Dtype(6, size, members=members), p - off
        if cls == 7:  # reference
            return _Dtype(7, size), p - off
        if cls == 9:  # variable length
            base, used = self._datatype(data, p)
            p += used
            return _Dtype(9, size, vtype=bits & 0x0F, base=base), p - off
        if cls == 10:  # array
            nd = data[p]
            p += 4 if ver < 3 else 1
            dims = struct.unpack_from(f"<{nd}I", data, p)
            p += 4 * nd
            if ver < 3:
                p += 4 * nd
            base, used = self._datatype(data, p)
            p += used
            return _Dtype(10, size, dims=dims, base=base), p - off
        raise NotImplementedError(f"datatype class {cls}")

    def _shared_or_inline_dtype(self, mflags, data):
        if mflags & 0x02:  # shared message: a committed datatype
            ver, typ = data[0], data[1]
            addr = struct.unpack_from("<Q", data, 2)[0]
            for mt, mf, md in self._messages(addr):
                if mt == 0x03:
                    dt, _ = self._datatype(md)
                    dt.committed = addr
                    return dt
            raise ValueError("committed datatype without a datatype message")
        dt, _ = self._datatype(data)
        dt.committed = None
        return dt

    def _attrs_of(self, addr):
        out = {}
        for mt, mf, md in self._messages(addr):
            if mt == 0x0C:
                name, val = self._attribute(md)
                out[name] = val
        return out

    def _attribute(self, md):
        ver = md[0]
        flags = md[1]
        nlen, dlen, slen = struct.unpack_from("<3H", md, 2)
        p = 8
        if ver >= 3:
            p += 1
        name = md[p:p + nlen].split(b"\x00")[0].decode()
        p += nlen if ver >= 2 else nlen + (-nlen) % 8
        dtdata = md[p:p + dlen]
        p += dlen if ver >= 2 else dlen + (-dlen) % 8
        if flags & 0x01:
            dt = self._shared_or_inline_dtype(0x02, dtdata)
        else:
            dt, _ = self._datatype(dtdata)
        sdata = md[p:p + slen]
        p += slen if ver >= 2 else slen + (-slen) % 8
        dims = self._dataspace(sdata)
        n = int(np.prod(dims)) if dims else 1
        raw = md[p:p + n * dt.size]
        try:
            val = self._decode(dt, raw, dims)
        except NotImplementedError:
            val = None
        return name, val

    # ---------------------------------------------------------------- dataspace / layout
    @staticmethod
    def _dataspace(data):
        ver, nd, flags = data[0], data[1], data[2]
        if ver == 1:
            p = 8
        else:
            typ = data[3]
            p = 4
            if typ == 0:
                return ()
            if typ == 2:
                return None
        dims = struct.unpack_from(f"<{nd}Q", data, p)
        return tuple(dims)

    def _gheap_obj(self, addr, idx):
        if addr not in self._gheap:
            b = self.buf
            p = self._abs(addr)
            assert b[p:p + 4] == b"GCOL", "global heap expected"
            csize = struct.unpack_from("<Q", b, p + 8)[0]
            end = p + csize
            q = p + 16
            objs = {}
            while q + 16 <= end:
                hi, _rc = struct.unpack_from("<HH", b, q)
                osz = struct.unpack_from("<Q", b, q + 8)[0]
                if hi == 0:
                    break
                objs[hi] = b[q + 16:q + 16 + osz]
                q += 16 + osz + (-osz) % 8
            self._gheap[addr] = objs
        return self._gheap[addr][idx]

    def _decode(self, dt, raw, dims):
        n = int(np.prod(dims)) if dims else 1
        shape = tuple(reversed(dims)) if dims else ()
        if dt.cls == 1:
            arr = np.frombuffer(raw, dtype=f"<f{dt.size}", count=n)
            return arr.reshape(shape, order="F").copy() if dims else float(arr[0])
        if dt.cls == 0:
            arr = np.frombuffer(raw, dtype=("<i" if dt.signed else "<u") + str(dt.size), count=n)
            if dt.size == 1 and not dt.signed:
                arr = arr.astype(bool)
            return arr.reshape(shape, order="F").copy() if dims else arr[0].item()
        if dt.cls == 3:
            s = raw[:dt.size].split(b"\x00")[0].decode()
            return s
        if dt.cls == 6:
            names = [m[0] for m in dt.members]
            if len(dt.members) == 2 and all(m[2].cls == 1 and m[2].size == 8 for m in dt.members):
                arr = np.frombuffer(raw, dtype="<f8", count=2 * n).reshape(n, 2)
                c = arr[:, 0] + 1j * arr[:, 1]
                return c.reshape(shape, order="F").copy() if dims else complex(c[0])
            recs = []
            for e in range(n):
                rec = {}
                for name, moff, mt in dt.members:
                    rec[name] = self._decode(mt, raw[e * dt.size + moff:e * dt.size + moff + mt.size], ())
                recs.append(rec)
            if names == ["kvvec"] and n == 1:
                return recs[0]["kvvec"]
            if names == ["first", "second"]:
                return [(r["first"], r["second"]) for r in recs] if dims else (recs[0]["first"], recs[0]["second"])
            return recs if dims else recs[0]
        if dt.cls == 7:
            refs = np.frombuffer(raw, dtype="<u8", count=n)
            vals = [self.read_object(int(r)) if r != 0 else None for r in refs]
            if not dims:
                return vals[0]
            return vals
        if dt.cls == 9:
            out = []
            for e in range(n):
                ln, haddr, hidx = struct.unpack_from("<IQI", raw, e * 16)
                obj = self._gheap_obj(haddr, hidx) if haddr else b""
                if dt.vtype == 1:
                    out.append(obj[:ln].decode())
                else:
                    out.append(self._decode(dt.base, obj[:ln * dt.base.size], (ln,)))
            return out if dims else out[0]
        raise NotImplementedError(f"decode class {dt.cls}")

    # ---------------------------------------------------------------- datasets / groups
    def read_object(self, addr):
        msgs = self._messages(addr)
        dt = dims = layout = None
        filters = []
        links = {}
        for mt, mf, md in msgs:
            if mt == 0x03:
                dt = self._shared_or_inline_dtype(mf, md)
            elif mt == 0x01:
                dims = self._dataspace(md)
            elif mt == 0x08:
                layout = md
            elif mt == 0x0B:
                filters = self._filters(md)
            elif mt == 0x06:
                name, target = self._link(md)
                links[name] = target
        if dt is None:  # a group
            return {k: self.read_object(v) for k, v in links.items()}
        raw = self._layout_data(layout, dt, dims, filters)
        if dims is None:
            return None
        kvvec = dt.cls == 6 and [m[0] for m in dt.members] == ["kvvec"]
        val = self._decode(dt, raw, dims)
        if kvvec:
            return dict(val)
        return val

    def _filters(self, md):
        ver, nf = md[0], md[1]
        p = 8 if ver == 1 else 2
        out = []
        for _ in range(nf):
            fid = struct.unpack_from("<H", md, p)[0]
            if ver == 1 or fid >= 256:
                nlen = struct.unpack_from("<H", md, p + 2)[0]
                nvals = struct.unpack_from("<H", md, p + 6)[0]
                p += 8 + nlen + (-nlen) % 8 if ver == 1 else 8 + nlen
            else:
                nvals = struct.unpack_from("<H", md, p + 4)[0]
                p += 6
            p += 4 * nvals
            if ver == 1 and nvals % 2:
                p += 4
            out.append(fid)
        return out

    def _layout_data(self, md, dt, dims, filters):
        ver, cls = md[0], md[1]
        n = int(np.prod(dims)) if dims else 1
        nbytes = n * dt.size
        if cls == 0:
            sz = struct.unpack_from("<H", md, 2)[0]
            return md[4:4 + sz]
        if cls == 1:
            addr, sz = struct.unpack_from("<2Q", md, 2)
            if addr == 0xFFFFFFFFFFFFFFFF:
                return b"\x00" * nbytes
            p = self._abs(addr)
            return self.buf[p:p + sz]
        if cls == 2:
            return self._chunked(md, dt, dims, filters)
        raise NotImplementedError(f"layout class {cls}")

    def _chunked(self, md, dt, dims, filters):
        ver = md[0]
        if ver == 4:
            flags = md[2]
            nd = md[3]
            enc = md[4]
            cdims = [int.from_bytes(md[5 + i * enc:5 + (i + 1) * enc], "little") for i in range(nd)]
            p = 5 + nd * enc
            itype = md[p]
            p += 1
            if itype == 1:  # single chunk
                if filters:
                    fsize = struct.unpack_from("<Q", md, p)[0]
                    p += 8 + 4
                    addr = struct.unpack_from("<Q", md, p)[0]
                    raw = self.buf[self._abs(addr):self._abs(addr) + fsize]
                else:
                    addr = struct.unpack_from("<Q", md, p)[0]
                    n = int(np.prod(dims)) * dt.size
                    raw = self.buf[self._abs(addr):self._abs(addr) + n]
                if 1 in filters:
                    raw = zlib.decompress(raw)
                return raw
            raise NotImplementedError(f"chunk index type {itype}")
        raise NotImplementedError(f"chunked layout version {ver}")

    @staticmethod
    def _link(md):
        flags = md[1]
        p = 2
        ltype = 0
        if flags & 0x08:
            ltype = md[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        nb = 1 << (flags & 3)
        nlen = int.from_bytes(md[p:p + nb], "little")
        p += nb
        name = md[p:p + nlen].decode()
        p += nlen
        if ltype != 0:
            return name, None
        return name, struct.unpack_from("<Q", md, p)[0]

    def load(self):
        """Every top-level name of the file (as JLD2.load does), without the committed types."""
        out = {}
        for mt, mf, md in self._messages(self.root):
            if mt == 0x06:
                name, target = self._link(md)
                if name.startswith("_") or target is None:
                    continue
                out[name] = self.read_object(target)
        return out


def load(path):
    return JLD2File(path).load()
