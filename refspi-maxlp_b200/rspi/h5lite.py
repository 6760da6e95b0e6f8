"""Minimal HDF5 reader/writer for the reference's photons and output files.

h5py and libhdf5 are not available on this platform, so this module
implements, from the public HDF5 file-format specification, the subset that
the reference's files use (make_data.py:228-276, emc.py:231-239), i.e. what
h5py writes with its default settings:

* superblock version 0, 8-byte offsets and lengths;
* the root group as a symbol table (v1 B-tree of symbol-table nodes plus a
  local heap of names); version-1 object headers with continuation blocks;
* datasets with a simple dataspace and contiguous (or compact) layout;
* datatypes: little/big-endian integers (1, 2, 4, 8 bytes), IEEE
  float32/float64, compound types (complex numbers are written as h5py
  does: a compound of float64 members ``r`` and ``i``) and variable-length
  sequences of a fixed type (vlen int32 lists, stored in global heap
  collections).

``read_datasets(path)`` returns ``{name: ndarray}`` for the root group's
datasets (vlen datasets as ``name@flat`` + ``name@lens`` arrays, the layout
``photonfile`` uses); ``write_datasets(path, data)`` writes a file with the
same subset.  Attributes and nested groups are skipped when reading.
"""
import struct

import numpy as np

SIGNATURE = b'\x89HDF\r\n\x1a\n'
UNDEF = 0xffffffffffffffff

# ---------------------------------------------------------------------------
# reading
# ---------------------------------------------------------------------------


class H5FormatError(ValueError):
    pass


class _Reader:
    def __init__(self, buf):
        self.b = buf
        if buf[:8] != SIGNATURE:
            raise H5FormatError('not an HDF5 file (signature)')
        ver = buf[8]
        if ver not in (0, 1):
            raise H5FormatError('superblock version %d is not supported' % ver)
        if buf[13] != 8 or buf[14] != 8:
            raise H5FormatError('only 8-byte offsets and lengths are supported')
        pos = 24 if ver == 0 else 28
        self.base = self._u64(pos)
        pos += 32                              # base, free-space, eof, driver
        # root group symbol table entry
        self.root_header = self._u64(pos + 8)
        cache = struct.unpack_from('<I', buf, pos + 16)[0]
        self.root_scratch = (self._u64(pos + 24), self._u64(pos + 32)) if cache == 1 else None
        self._gheap = {}

    def _u64(self, off):
        return struct.unpack_from('<Q', self.b, off)[0]

    def addr(self, a):
        return self.base + a

    # -- object headers ----------------------------------------------------
    def messages(self, header_addr):
        """[(type, flags, bytes)] of a version-1 object header, following
        continuation messages."""
        off = self.addr(header_addr)
        if self.b[off] != 1:
            raise H5FormatError('object header version %d is not supported' % self.b[off])
        nmsg = struct.unpack_from('<H', self.b, off + 2)[0]
        size = struct.unpack_from('<I', self.b, off + 8)[0]
        blocks = [(off + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(out) < nmsg:
                mtype, msize, mflags = struct.unpack_from('<HHB', self.b, p)
                body = self.b[p + 8:p + 8 + msize]
                out.append((mtype, mflags, body))
                if mtype == 0x0010:            # continuation
                    caddr, clen = struct.unpack_from('<QQ', body, 0)
                    blocks.append((self.addr(caddr), clen))
                p += 8 + msize
        return out

    # -- groups ------------------------------------------------------------
    def group_entries(self, btree_addr, heap_addr):
        heap = self.addr(heap_addr)
        if self.b[heap:heap + 4] != b'HEAP':
            raise H5FormatError('bad local heap signature')
        data_addr = self._u64(heap + 24)
        names = self.addr(data_addr)
        entries = []
        self._walk_btree(btree_addr, names, entries)
        return entries

    def _walk_btree(self, node_addr, names, entries):
        off = self.addr(node_addr)
        if self.b[off:off + 4] != b'TREE':
            raise H5FormatError('bad B-tree signature')
        level = self.b[off + 5]
        used = struct.unpack_from('<H', self.b, off + 6)[0]
        p = off + 24 + 8                        # skip key 0
        for _ in range(used):
            child = self._u64(p)
            p += 16                             # child, next key
            if level > 0:
                self._walk_btree(child, names, entries)
            else:
                self._read_snod(child, names, entries)

    def _read_snod(self, addr, names, entries):
        off = self.addr(addr)
        if self.b[off:off + 4] != b'SNOD':
            raise H5FormatError('bad symbol table node signature')
        nsym = struct.unpack_from('<H', self.b, off + 6)[0]
        p = off + 8
        for _ in range(nsym):
            name_off, hdr = struct.unpack_from('<QQ', self.b, p)
            n0 = names + name_off
            n1 = self.b.index(b'\0', n0)
            entries.append((self.b[n0:n1].decode(), hdr))
            p += 40

    # -- datatypes -----------------------------------------------------------
    def datatype(self, body, pos=0):
        """Parse a datatype message; returns (descriptor, size, next pos)."""
        cv = body[pos]
        cls, ver = cv & 0x0f, cv >> 4
        bits = body[pos + 1] | (body[pos + 2] << 8) | (body[pos + 3] << 16)
        size = struct.unpack_from('<I', body, pos + 4)[0]
        p = pos + 8
        if cls == 0:                            # fixed point
            endian = '>' if bits & 1 else '<'
            signed = bool(bits & 8)
            return ('int', np.dtype('%s%s%d' % (endian, 'i' if signed else 'u', size))), size, p + 4
        if cls == 1:                            # floating point
            endian = '>' if bits & 1 else '<'
            if size not in (2, 4, 8):
                raise H5FormatError('float of %d bytes' % size)
            return ('float', np.dtype('%sf%d' % (endian, size))), size, p + 12
        if cls == 6:                            # compound
            nmem = bits & 0xffff
            members = []
            for _ in range(nmem):
                n1 = body.index(b'\0', p)
                name = body[p:n1].decode()
                if ver < 3:
                    p = p + ((n1 - p) // 8 + 1) * 8
                else:
                    p = n1 + 1
                if ver == 1:
                    moff = struct.unpack_from('<I', body, p)[0]
                    p += 4 + 1 + 3 + 4 + 4 + 16
                elif ver == 2:
                    moff = struct.unpack_from('<I', body, p)[0]
                    p += 4
                else:
                    nb = max(1, (size.bit_length() + 7) // 8)
                    moff = int.from_bytes(body[p:p + nb], 'little')
                    p += nb
                mdesc, msize, p = self.datatype(body, p)
                members.append((name, moff, mdesc))
            return ('compound', members), size, p
        if cls == 9:                            # variable length
            kind = bits & 0x3
            base, bsize, p2 = self.datatype(body, p)
            if kind != 0:
                raise H5FormatError('variable-length strings are not supported')
            return ('vlen', base), size, p2
        raise H5FormatError('datatype class %d is not supported' % cls)

    @staticmethod
    def numpy_dtype(desc):
        kind = desc[0]
        if kind in ('int', 'float'):
            return desc[1]
        if kind == 'compound':
            names = [m[0] for m in desc[1]]
            if names == ['r', 'i'] and all(m[2][0] == 'float' for m in desc[1]):
                f = desc[1][0][2][1]
                return np.dtype('c%d' % (2 * f.itemsize)).newbyteorder(f.byteorder)
            return np.dtype({'names': names, 'formats': [_Reader.numpy_dtype(m[2]) for m in desc[1]],
                             'offsets': [m[1] for m in desc[1]]})
        raise H5FormatError('no NumPy type for %s' % kind)

    # -- datasets --------------------------------------------------------------
    def dataset(self, header_addr):
        shape, desc, layout = None, None, None
        for mtype, _, body in self.messages(header_addr):
            if mtype == 0x0001:                 # dataspace
                ver, ndim, flags = body[0], body[1], body[2]
                p = 8 if ver == 1 else 4
                shape = tuple(struct.unpack_from('<%dQ' % ndim, body, p)) if ndim else ()
            elif mtype == 0x0003:
                desc, esize, _ = self.datatype(body, 0)
            elif mtype == 0x0008:               # layout
                ver = body[0]
                if ver < 3:
                    raise H5FormatError('layout message version %d is not supported' % ver)
                cls = body[1]
                if cls == 1:
                    addr, size = struct.unpack_from('<QQ', body, 2)
                    layout = ('contiguous', addr, size)
                elif cls == 0:
                    size = struct.unpack_from('<H', body, 2)[0]
                    layout = ('compact', body[4:4 + size])
                else:
                    raise H5FormatError('chunked datasets are not supported')
        if shape is None or desc is None or layout is None:
            return None
        n = int(np.prod(shape)) if shape else 1
        if layout[0] == 'contiguous':
            raw = b'' if layout[1] == UNDEF else self.b[self.addr(layout[1]):self.addr(layout[1]) + n * esize]
        else:
            raw = bytes(layout[1])
        if len(raw) < n * esize:                # never written: fill with zeros
            raw = raw + b'\0' * (n * esize - len(raw))
        if desc[0] == 'vlen':
            base = self.numpy_dtype(desc[1])
            lens = np.empty(n, dtype=np.int64)
            parts = []
            for i in range(n):
                ln, caddr, idx = struct.unpack_from('<IQI', raw, 16 * i)
                lens[i] = ln
                parts.append(np.frombuffer(self._gheap_object(caddr, idx), dtype=base, count=ln)
                             if ln else np.zeros(0, base))
            flat = np.concatenate(parts) if parts else np.zeros(0, base)
            return ('vlen', flat.astype(base.newbyteorder('=')), lens)
        dt = self.numpy_dtype(desc)
        arr = np.frombuffer(raw, dtype=dt, count=n).reshape(shape)
        return ('plain', arr.astype(dt.newbyteorder('=')))

    def _gheap_object(self, caddr, idx):
        if caddr not in self._gheap:
            off = self.addr(caddr)
            if self.b[off:off + 4] != b'GCOL':
                raise H5FormatError('bad global heap signature')
            csize = self._u64(off + 8)
            objs = {}
            p = off + 16
            while p + 16 <= off + csize:
                oidx, _, _, osize = struct.unpack_from('<HHIQ', self.b, p)
                if oidx == 0:
                    break
                objs[oidx] = self.b[p + 16:p + 16 + osize]
                p += 16 + ((osize + 7) // 8) * 8
            self._gheap[caddr] = objs
        return self._gheap[caddr][idx]

    def root_datasets(self):
        scratch = self.root_scratch
        if scratch is None:
            for mtype, _, body in self.messages(self.root_header):
                if mtype == 0x0011:
                    scratch = struct.unpack_from('<QQ', body, 0)
        if scratch is None:
            raise H5FormatError('root group is not a symbol-table group')
        out = {}
        for name, hdr in self.group_entries(*scratch):
            ds = self.dataset(hdr)
            if ds is None:
                continue                        # a subgroup or another object
            if ds[0] == 'vlen':
                out[name + '@flat'] = ds[1]
                out[name + '@lens'] = ds[2]
            else:
                out[name] = ds[1]
        return out


def read_datasets(path):
    """{name: array} of the root group's datasets (see the module docstring)."""
    with open(path, 'rb') as f:
        return _Reader(f.read()).root_datasets()


# ---------------------------------------------------------------------------
# writing
# ---------------------------------------------------------------------------

def _pad8(b):
    return b + b'\0' * ((-len(b)) % 8)


def _dt_fixed(dtype):
    dt = np.dtype(dtype)
    bits = (1 if dt.byteorder == '>' else 0) | (8 if dt.kind == 'i' else 0)
    return struct.pack('<BBBBI', 0x10 | 0, bits, 0, 0, dt.itemsize) + \
        struct.pack('<HH', 0, 8 * dt.itemsize)


def _dt_float(dtype):
    dt = np.dtype(dtype)
    if dt.itemsize == 8:
        bits, props = 0x20 | (63 << 8), struct.pack('<HHBBBBI', 0, 64, 52, 11, 0, 52, 1023)
    elif dt.itemsize == 4:
        bits, props = 0x20 | (31 << 8), struct.pack('<HHBBBBI', 0, 32, 23, 8, 0, 23, 127)
    else:
        raise ValueError('float%d is not supported' % (8 * dt.itemsize))
    bits |= 1 if dt.byteorder == '>' else 0
    return struct.pack('<BBBBI', 0x10 | 1, bits & 0xff, (bits >> 8) & 0xff, 0, dt.itemsize) + props


def _dt(dtype):
    dt = np.dtype(dtype)
    if dt.kind in 'iu':
        return _dt_fixed(dt)
    if dt.kind == 'f':
        return _dt_float(dt)
    if dt.kind == 'c':
        f = np.dtype('f%d' % (dt.itemsize // 2))
        mem = b''
        for name, off in (('r', 0), ('i', f.itemsize)):
            mem += _pad8(name.encode() + b'\0') + struct.pack('<IB3xI4x16x', off, 0, 0) + _dt_float(f)
        return struct.pack('<BBBBI', 0x10 | 6, 2, 0, 0, dt.itemsize) + mem
    raise ValueError('dtype %s is not supported' % dt)


def _dt_vlen(base):
    return struct.pack('<BBBBI', 0x10 | 9, 0, 0, 0, 16) + _dt(base)


def _msg(mtype, body, flags=0):
    body = _pad8(body)
    return struct.pack('<HHB3x', mtype, len(body), flags) + body


def _dataspace(shape):
    return struct.pack('<BBB5x', 1, len(shape), 0) + b''.join(struct.pack('<Q', s) for s in shape)


def _fill_value():
    # version 2: allocation time late, fill time never, no value defined
    return struct.pack('<BBBB', 2, 2, 2, 0)


def _object_header(messages):
    body = b''.join(messages)
    return struct.pack('<BBHII4x', 1, 0, len(messages), 1, len(body)) + body


class _Writer:
    def __init__(self):
        self.buf = bytearray(b'\0' * 96)        # superblock, filled last

    def alloc(self, data, align=8):
        pad = (-len(self.buf)) % align
        self.buf += b'\0' * pad
        addr = len(self.buf)
        self.buf += data
        return addr

    def global_heap(self, objects):
        """Global heap collections holding the objects in order (at most
        65,535 per collection: the object index is 16 bits); returns each
        object's (collection address, index)."""
        refs = []
        for c0 in range(0, len(objects), 65535):
            chunk = objects[c0:c0 + 65535]
            parts = []
            for i, o in enumerate(chunk, start=1):
                parts.append(struct.pack('<HHIQ', i, 1, 0, len(o)))
                parts.append(_pad8(o))
            body = b''.join(parts)
            size = max(16 + len(body) + 16, 4096)
            free = size - 16 - len(body)
            data = b''.join([b'GCOL', struct.pack('<B3xQ', 1, size), body,
                             struct.pack('<HHIQ', 0, 0, 0, free)])
            data += b'\0' * (size - len(data))
            addr = self.alloc(data)
            refs.extend((addr, i) for i in range(1, len(chunk) + 1))
        return refs

    def dataset(self, arr):
        if isinstance(arr, tuple) and arr[0] == 'vlen':
            _, flat, lens = arr
            flat = np.ascontiguousarray(flat)
            base = flat.dtype
            bounds = np.concatenate([[0], np.cumsum(lens)])
            objs = [flat[bounds[i]:bounds[i + 1]].tobytes() for i in range(len(lens))]
            refs = iter(self.global_heap([o for o in objs if o]))
            parts = []
            for i, o in enumerate(objs):
                if o:
                    gaddr, k = next(refs)
                    parts.append(struct.pack('<IQI', int(lens[i]), gaddr, k))
                else:
                    parts.append(struct.pack('<IQI', 0, 0, 0))
            raw = b''.join(parts)
            shape = (len(lens),)
            dtmsg = _dt_vlen(base)
        else:
            arr = np.ascontiguousarray(arr)
            if arr.dtype == np.bool_:
                arr = arr.astype('u1')
            raw = arr.tobytes()
            shape = arr.shape
            dtmsg = _dt(arr.dtype)
        daddr = self.alloc(raw) if raw else UNDEF
        layout = struct.pack('<BBQQ', 3, 1, daddr, len(raw))
        msgs = [_msg(0x0001, _dataspace(shape)), _msg(0x0003, dtmsg, 1),
                _msg(0x0005, _fill_value(), 1), _msg(0x0008, layout)]
        return self.alloc(_object_header(msgs))


def write_datasets(path, data):
    """Write {name: array} as root-group datasets; a value ('vlen', flat,
    lens) becomes a variable-length dataset."""
    w = _Writer()
    names = sorted(data)
    headers = {n: w.dataset(data[n]) for n in names}
    # local heap of names (offset 0 is the empty string)
    heap_data = b'\0' * 8
    name_off = {}
    for n in names:
        name_off[n] = len(heap_data)
        heap_data += _pad8(n.encode() + b'\0')
    heap_data += b'\0' * 16                         # room for a free block
    data_addr = w.alloc(heap_data)
    free_off = len(heap_data) - 16
    heap_data_free = struct.pack('<QQ', 1, 16)       # next free (1 = none), size
    w.buf[data_addr + free_off:data_addr + free_off + 16] = heap_data_free
    heap_addr = w.alloc(b'HEAP' + struct.pack('<B3xQQQ', 0, len(heap_data), free_off, data_addr))
    # symbol table nodes of at most 8 entries, names in order
    snods, keys = [], []
    for i in range(0, max(1, len(names)), 8):
        chunk = names[i:i + 8]
        body = b'SNOD' + struct.pack('<BBH', 1, 0, len(chunk))
        for n in chunk:
            body += struct.pack('<QQII16x', name_off[n], headers[n], 0, 0)
        body += b'\0' * (40 * (8 - len(chunk)))
        snods.append(w.alloc(body))
        keys.append(name_off[chunk[-1]] if chunk else 0)
    btree = b'TREE' + struct.pack('<BBHQQ', 0, 0, len(snods), UNDEF, UNDEF)
    btree += struct.pack('<Q', 0)
    for addr, key in zip(snods, keys):
        btree += struct.pack('<QQ', addr, key)
    btree += b'\0' * (16 * (32 - len(snods)))
    btree_addr = w.alloc(btree)
    root = w.alloc(_object_header([_msg(0x0011, struct.pack('<QQ', btree_addr, heap_addr))]))
    eof = len(w.buf)
    sb = SIGNATURE + struct.pack('<BBBBBBBBHHI', 0, 0, 0, 0, 0, 8, 8, 0, 4, 16, 0)
    sb += struct.pack('<QQQQ', 0, UNDEF, eof, UNDEF)
    sb += struct.pack('<QQII', 0, root, 1, 0) + struct.pack('<QQ', btree_addr, heap_addr)
    w.buf[:len(sb)] = sb
    with open(path, 'wb') as f:
        f.write(bytes(w.buf))


def write_photons(path, data):
    """Photons file in the reference layout (make_data.py:245-251)."""
    out = {}
    lens = {'place_ones': data['ones'], 'place_multi': data['multi'],
            'count_multi': data['multi']}
    for key, val in data.items():
        if key in lens:
            out[key] = ('vlen', np.asarray(val, dtype='<i4'), np.asarray(lens[key]))
        else:
            out[key] = np.asarray(val)
    write_datasets(path, out)
    return path
