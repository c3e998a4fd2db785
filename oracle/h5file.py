"""h5file.py -- CPU restatement of the reference's field checkpoint file
uvwp_NNNN.h5 and an independent reader of it.

TEST INFRASTRUCTURE ONLY: the checker of the library's HDF5 writer and
reader (ductgpu_save_4fields_fou_hdf5_dev / ductgpu_read_*); only tests/
use it.

What the file holds follows the reference's calls: save_4fields_fou_hdf5
(src/readwrite_hdf5.f90:276-386) creates u, v, w, p with h5dump_parallel
(:650-722) as H5T_IEEE_F64BE datasets of Fortran shape (2, my, mz, mx1+1)
-- HDF5 (C-order) shape (mx1+1, mz, my, 2) -- and writeheader_hdf5
(:851-920) adds nparams, numerop, mgalx, my, mz, mx1 (H5T_STD_I32LE) and
alp, aspect, time, fnu, cfl, dtfixed, cmassflow, SLIP-VELOCITY, DIVERGENCE
(H5T_IEEE_F64LE), each of shape (1), through h5write_simple_int / _double
(:922-968).

How the bytes are laid out follows the published HDF5 File Format
Specification (superblock version 0; version 1 object headers with the
dataspace (0x0001), datatype (0x0003), fill value (0x0005), layout
(0x0008), symbol table (0x0011) and continuation (0x0010) messages; the
version 1 B-tree of a symbol-table group, its symbol table nodes and local
heap), in the form libhdf5 gives such a file with its default format bounds.

Parity unpinned: there is no HDF5 library and no file written by the
reference in this image, so neither the writer restated here nor the
library's can be read back by libhdf5 here.  The checks are: the library's
file equals write_4fields() byte for byte, and read() -- written from the
specification separately from both writers, with libhdf5's own consistency
rules (message alignment, message counts, the local heap's free-list end
marker, the end-of-file address) -- decodes it to the fields and scalars.
"""
import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
HEAP_FREE_NULL = 1          # libhdf5's end of a local heap free list
LEAF_K, NODE_K = 4, 16      # group K values of the superblock
SNOD_BYTES = 8 + 2 * LEAF_K * 40
TREE_BYTES = 24 + 2 * NODE_K * 8 + (2 * NODE_K + 1) * 8
FIELD_ALIGN = 4096

INT_NAMES = ("nparams", "numerop", "mgalx", "my", "mz", "mx1")
DBL_NAMES = ("alp", "aspect", "time", "fnu", "cfl", "dtfixed", "cmassflow", "SLIP-VELOCITY", "DIVERGENCE")
HEADER_KEYS = {"SLIP-VELOCITY": "slip", "DIVERGENCE": "divergence"}


def _pad8(n):
    return (n + 7) & ~7


def uvwp_filename(fuvwpout, iimag):
    """concat5b(fuvwpout,'uvwp_',5,ext,4,'.',1,'h5',2,filename) with ext the
    Fortran i4.4 of iimag (src/readwrite_hdf5.f90:326-330, src/concat.F:74-87)."""
    head = fuvwpout.split(" ", 1)[0]
    ext = "%04d" % iimag if 0 <= iimag <= 9999 else "****"
    return head + "uvwp_" + ext + ".h5"


def _header_values(hdr):
    vals = {"nparams": 7, "numerop": hdr.get("numerop", 1) if hdr.get("numerop", 1) > 0 else 1}
    for k in ("mgalx", "my", "mz", "mx1"):
        vals[k] = int(hdr[k])
    for k in DBL_NAMES:
        vals[k] = float(hdr.get(HEADER_KEYS.get(k, k), 0.0))
    return vals


def write_datasets(datasets):
    """The bytes of an HDF5 file holding the given datasets in its root group,
    laid out as the library lays it out: superblock, root group header, local
    heap, B-tree, symbol table nodes, dataset headers (in strcmp order of
    the names), the data of the non-streamed datasets (8-byte aligned), then
    the streamed ones from the next 4 KiB boundary on, in stream order.
    datasets: list of dict(name, kind 'i4' | 'f8' | '>f8', dims (HDF5
    C-order shape), data (numpy array of that shape), stream None or int)."""
    ds = sorted(datasets, key=lambda d: d["name"].encode())
    item = {"i4": 4, "f8": 8, ">f8": 8}
    nbytes = {d["name"]: int(np.prod(d["dims"])) * item[d["kind"]] for d in ds}

    def oh_bytes(d):
        rank = len(d["dims"])
        return 16 + (8 + 8 + 8 * rank) + (8 + (16 if d["kind"] == "i4" else 24)) + 16 + 32

    heap_off, h = {}, 8
    for d in ds:
        heap_off[d["name"]] = h
        h += _pad8(len(d["name"]) + 1)
    heap_bytes = h
    nsnod = (len(ds) + 2 * LEAF_K - 1) // (2 * LEAF_K)
    a = 96
    root_oh = a
    a += 40
    heap_hdr = a
    a += 32
    heap_data = a
    a += heap_bytes
    btree = a
    a += TREE_BYTES
    snod = []
    for _ in range(nsnod):
        snod.append(a)
        a += SNOD_BYTES
    oh = {}
    for d in ds:
        oh[d["name"]] = a
        a += oh_bytes(d)
    data = {}
    for d in ds:
        if d.get("stream") is None:
            data[d["name"]] = a
            a += _pad8(nbytes[d["name"]])
    meta_end = a
    streamed = sorted([d for d in ds if d.get("stream") is not None], key=lambda d: d["stream"])
    if streamed:
        a = (a + FIELD_ALIGN - 1) // FIELD_ALIGN * FIELD_ALIGN
        for d in streamed:
            data[d["name"]] = a
            a += nbytes[d["name"]]
    eof = a

    b = bytearray(eof)

    def put(off, fmt, *v):
        struct.pack_into("<" + fmt, b, off, *v)

    b[0:8] = SIGNATURE
    put(8, "8B", 0, 0, 0, 0, 0, 8, 8, 0)
    put(16, "HHI", LEAF_K, NODE_K, 0)
    put(24, "QQQQ", 0, UNDEF, eof, UNDEF)
    put(56, "QQII", 0, root_oh, 1, 0)
    put(80, "QQ", btree, heap_hdr)
    put(root_oh, "BBHII4x", 1, 0, 1, 1, 24)
    put(root_oh + 16, "HHB3xQQ", 0x0011, 16, 0, btree, heap_hdr)
    b[heap_hdr:heap_hdr + 4] = b"HEAP"
    put(heap_hdr + 8, "QQQ", heap_bytes, HEAP_FREE_NULL, heap_data)
    for d in ds:
        nb = d["name"].encode() + b"\0"
        o = heap_data + heap_off[d["name"]]
        b[o:o + len(nb)] = nb
    b[btree:btree + 4] = b"TREE"
    put(btree + 4, "BBH", 0, 0, nsnod)
    put(btree + 8, "QQQ", UNDEF, UNDEF, 0)
    for s in range(nsnod):
        last = ds[min(len(ds), (s + 1) * 2 * LEAF_K) - 1]["name"]
        put(btree + 32 + 16 * s, "QQ", snod[s], heap_off[last])
    for s in range(nsnod):
        group = ds[s * 2 * LEAF_K:(s + 1) * 2 * LEAF_K]
        b[snod[s]:snod[s] + 4] = b"SNOD"
        put(snod[s] + 4, "BBH", 1, 0, len(group))
        for j, d in enumerate(group):
            put(snod[s] + 8 + 40 * j, "QQII16x", heap_off[d["name"]], oh[d["name"]], 0, 0)
    for d in ds:
        n, dims = d["name"], tuple(d["dims"])
        rank = len(dims)
        o = oh[n]
        put(o, "BBHII4x", 1, 0, 4, 1, oh_bytes(d) - 16)
        p = o + 16
        put(p, "HHB3x", 0x0001, 8 + 8 * rank, 0)
        put(p + 8, "BBBB4x", 1, rank, 0, 0)
        put(p + 16, "%dQ" % rank, *dims)
        p += 16 + 8 * rank
        if d["kind"] == "i4":
            put(p, "HHB3x", 0x0003, 16, 1)
            put(p + 8, "BBBBIHH4x", 0x10, 0x08, 0, 0, 4, 0, 32)
            p += 24
        else:
            put(p, "HHB3x", 0x0003, 24, 1)
            put(p + 8, "BBBBIHHBBBBI4x", 0x11, 0x21 if d["kind"] == ">f8" else 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52,
                1023)
            p += 32
        put(p, "HHB3x", 0x0005, 8, 1)
        put(p + 8, "BBBB4x", 2, 2, 2, 0)
        p += 16
        put(p, "HHB3x", 0x0008, 24, 0)
        put(p + 8, "BBQQ6x", 3, 1, data[n], nbytes[n])
        raw = np.ascontiguousarray(d["data"], dtype={"i4": "<i4", "f8": "<f8", ">f8": ">f8"}[d["kind"]])
        assert raw.size == int(np.prod(dims)), n
        b[data[n]:data[n] + nbytes[n]] = raw.tobytes()
    assert meta_end <= eof
    return bytes(b)


def write_4fields(fields, hdr, omit=()):
    """The bytes of the file save_4fields_fou_hdf5 + writeheader_hdf5 give for
    complex (my, mz, mx1+1) fields u, v, w, p (Fortran order) and the header
    dict (my, mz, mx1, mgalx, numerop, alp, aspect, time, fnu, cfl, dtfixed,
    cmassflow, slip, divergence).  omit: header scalars to leave out (an
    older file's header)."""
    my, mz, mx1 = int(hdr["my"]), int(hdr["mz"]), int(hdr["mx1"])
    nm = mx1 + 1
    vals = _header_values(hdr)
    ds = [dict(name=n, kind="i4", dims=(1,), data=np.array([vals[n]])) for n in INT_NAMES if n not in omit]
    ds += [dict(name=n, kind="f8", dims=(1,), data=np.array([vals[n]])) for n in DBL_NAMES if n not in omit]
    for k, (n, f) in enumerate(zip(("u", "v", "w", "p"), fields)):
        f = np.asfortranarray(f, dtype=np.complex128)
        assert f.shape == (my, mz, nm), (f.shape, (my, mz, nm))
        ds.append(dict(name=n, kind=">f8", dims=(nm, mz, my, 2), stream=k,
                       data=f.reshape(-1, order="F").view(np.float64)))
    return write_datasets(ds)


def write_statistics(st):
    """The bytes of the file write_statistics_hdf5 (src/readwrite_hdf5.f90:
    388-648, one rank, no temperature) gives: st = dict(mgalx, my, mz,
    nstat, timef, time, fnu, alp, aspect, mean (4,my,mz), prod (6,my,mz) in
    the order uu, vv, ww, uv, uw, vw, ppb (my,mz), spec (4,7,M), om2
    (3,my,mz)) -- the layout of the stepper's statistics."""
    my, mz = int(st["my"]), int(st["mz"])

    def plane(a):   # Fortran (my, mz) -> HDF5 (mz, my)
        return np.asarray(a, dtype=np.float64).T

    ds = [dict(name=n, kind="i4", dims=(1,), data=np.array([int(st[n])])) for n in ("mgalx", "my", "mz", "nstat")]
    ds += [dict(name=n, kind="f8", dims=(1,), data=np.array([float(st[n])]))
           for n in ("timef", "time", "fnu", "alp", "aspect")]
    for c, n in enumerate(("um", "vm", "wm", "pm")):
        ds.append(dict(name=n, kind="f8", dims=(mz, my), data=plane(st["mean"][c])))
    for c, n in enumerate(("uub", "vvb", "wwb", "uvb", "uwb", "vwb")):
        ds.append(dict(name=n, kind="f8", dims=(mz, my), data=plane(st["prod"][c])))
    ds.append(dict(name="ppb", kind="f8", dims=(mz, my), data=plane(st["ppb"])))
    for c, n in enumerate(("ox2", "oy2", "oz2")):
        ds.append(dict(name=n, kind="f8", dims=(mz, my), data=plane(st["om2"][c])))
    M = np.asarray(st["spec"]).shape[2]
    for c, n in enumerate(("uust", "vvst", "wwst", "ppst")):
        ds.append(dict(name=n, kind="f8", dims=(7, M), data=np.asarray(st["spec"][c], dtype=np.float64)))
    # the seven spectra points of statistics_fou (src/operators.F:1680-1693)
    ds.append(dict(name="jinco", kind="i4", dims=(7,),
                   data=np.array([my // 16, my // 8, my // 4, my // 2, my // 16, my // 8, my // 4])))
    ds.append(dict(name="kinco", kind="i4", dims=(7,),
                   data=np.array([mz // 2, mz // 2, mz // 2, mz // 2, mz // 16, mz // 8, mz // 4])))
    return write_datasets(ds)


class FormatError(ValueError):
    pass


def _need(cond, why):
    if not cond:
        raise FormatError(why)


def read(buf):
    """Decode an HDF5 file (superblock 0/1, symbol-table root group,
    contiguous or compact datasets) from its bytes: {name: numpy array}, the
    arrays in their HDF5 (C-order) shape and native byte order."""
    buf = bytes(buf)
    size = len(buf)
    at = None
    o = 0
    while o + 8 <= size:
        if buf[o:o + 8] == SIGNATURE:
            at = o
            break
        o = 512 if o == 0 else 2 * o
    _need(at is not None, "no HDF5 signature")
    base = at

    def get(addr, n):
        _need(addr != UNDEF and base + addr + n <= size, "address %#x + %d outside the file" % (addr, n))
        return buf[base + addr:base + addr + n]

    ver = buf[at + 8]
    _need(ver in (0, 1), "superblock version %d" % ver)
    _need(buf[at + 13] == 8 and buf[at + 14] == 8, "offset / length sizes")
    leaf_k, node_k = struct.unpack_from("<HH", buf, at + 16)
    _need(leaf_k > 0 and node_k > 0, "group K values")
    q = at + (28 if ver == 1 else 24)
    _, _, eof, _ = struct.unpack_from("<QQQQ", buf, q)
    _need(base + eof <= size, "file shorter than its end-of-file address")
    _, root_oh, cache, _ = struct.unpack_from("<QQII", buf, q + 32)

    def messages(addr):
        pre = get(addr, 16)
        ohv, _, nmesgs, _, chunk = struct.unpack_from("<BBHII", pre)
        _need(ohv == 1, "object header version %d" % ohv)
        out, chunks, seen = [], [(addr + 16, chunk)], 0
        while chunks:
            caddr, clen = chunks.pop(0)
            c = get(caddr, clen)
            p = 0
            while p < clen:
                _need(p + 8 <= clen, "message header overruns the chunk")
                typ, sz, flags = struct.unpack_from("<HHB", c, p)
                _need(sz % 8 == 0, "message size %d not 8-aligned" % sz)
                _need(p + 8 + sz <= clen, "message overruns the chunk")
                body = c[p + 8:p + 8 + sz]
                seen += 1
                if typ == 0x0010:
                    chunks.append(struct.unpack_from("<QQ", body))
                elif typ != 0:
                    out.append((typ, flags, body))
                p += 8 + sz
        _need(seen == nmesgs, "object header holds %d messages, prefix says %d" % (seen, nmesgs))
        return out

    stab = [m for m in messages(root_oh) if m[0] == 0x0011]
    _need(len(stab) == 1, "root group without a symbol table message")
    bt, hp = struct.unpack_from("<QQ", stab[0][2])
    if cache == 1:
        cbt, chp = struct.unpack_from("<QQ", buf, q + 56)
        _need((cbt, chp) == (bt, hp), "superblock's cached B-tree / heap differ from the root group's")
    hh = get(hp, 32)
    _need(hh[:4] == b"HEAP" and hh[4] == 0, "local heap header")
    hsize, free, haddr = struct.unpack_from("<QQQ", hh, 8)
    _need(free == HEAP_FREE_NULL or free < hsize, "local heap free list")
    heap = get(haddr, hsize)
    _need(hsize >= 1 and heap[0] == 0, "local heap offset 0 is not the empty name")

    def name_at(off):
        _need(off < hsize, "name offset outside the heap")
        end = heap.index(b"\0", off)
        return heap[off:end].decode()

    entries = []
    visits = [0]

    def tree(addr, depth):
        _need(depth < 16, "B-tree too deep")
        visits[0] += 1
        _need(visits[0] <= 65536, "B-tree too large")
        node = get(addr, 24 + (2 * node_k) * 16 + 8)
        _need(node[:4] == b"TREE" and node[4] == 0, "group B-tree node")
        level, used = node[5], struct.unpack_from("<H", node, 6)[0]
        _need(used <= 2 * node_k, "B-tree node over-full")
        keys = [struct.unpack_from("<Q", node, 24 + 16 * i)[0] for i in range(used + 1)]
        kids = [struct.unpack_from("<Q", node, 32 + 16 * i)[0] for i in range(used)]
        for i, kid in enumerate(kids):
            lo, hi = name_at(keys[i]), name_at(keys[i + 1])
            if level:
                tree(kid, depth + 1)
                continue
            sn = get(kid, 8 + 2 * leaf_k * 40)
            _need(sn[:4] == b"SNOD" and sn[4] == 1, "symbol table node")
            n = struct.unpack_from("<H", sn, 6)[0]
            _need(n <= 2 * leaf_k, "symbol table node over-full")
            names = []
            for j in range(n):
                off, ohaddr = struct.unpack_from("<QQ", sn, 8 + 40 * j)
                names.append(name_at(off))
                entries.append((names[-1], ohaddr))
            _need(names == sorted(names, key=lambda s: s.encode()), "symbol table node not sorted")
            # the B-tree keys bracket the node's names: lo < name <= hi
            _need(all(lo.encode() < s.encode() <= hi.encode() for s in names), "B-tree keys do not bracket the names")

    tree(bt, 0)
    out = {}
    for name, ohaddr in entries:
        rank, dims, dt, lay = None, None, None, None
        for typ, flags, body in messages(ohaddr):
            if typ == 0x0001:
                v, rank = body[0], body[1]
                off = 8 if v == 1 else 4
                dims = struct.unpack_from("<%dQ" % rank, body, off)
            elif typ == 0x0003:
                cls, bits, tsize = body[0] & 15, body[1], struct.unpack_from("<I", body, 4)[0]
                _need(body[0] >> 4 == 1, "datatype version")
                if cls == 1:
                    _need((bits >> 4) & 3 == 2 and body[2] == 63 and tsize == 8, "not an IEEE double")
                    _need(struct.unpack_from("<HHBBBBI", body, 8) == (0, 64, 52, 11, 0, 52, 1023), "double layout")
                    dt = np.dtype(">f8" if bits & 1 else "<f8")
                elif cls == 0:
                    dt = np.dtype(("%si%d" if (bits >> 3) & 1 else "%su%d") % (">" if bits & 1 else "<", tsize))
                else:
                    raise FormatError("datatype class %d" % cls)
            elif typ == 0x0008:
                _need(body[0] == 3, "layout version %d" % body[0])
                if body[1] == 1:
                    lay = ("c",) + struct.unpack_from("<QQ", body, 2)
                elif body[1] == 0:
                    n = struct.unpack_from("<H", body, 2)[0]
                    lay = ("k", body[4:4 + n])
                else:
                    raise FormatError("layout class %d" % body[1])
            elif typ == 0x000B:
                raise FormatError("filters")
        _need(all(x is not None for x in (rank, dims, dt, lay)), "dataset %s incomplete" % name)
        count = int(np.prod(dims)) if rank else 1
        if lay[0] == "c":
            _need(lay[2] == count * dt.itemsize, "%s: storage size" % name)
            raw = get(lay[1], lay[2])
        else:
            raw = lay[1]
        out[name] = np.frombuffer(raw, dtype=dt, count=count).reshape(dims).astype(dt.newbyteorder("="))
    return out


def fields_of(datasets):
    """u, v, w, p of a decoded file as complex (my, mz, mx1+1) Fortran arrays."""
    res = []
    for n in ("u", "v", "w", "p"):
        a = datasets[n]                                    # (mx1+1, mz, my, 2)
        c = a[..., 0] + 1j * a[..., 1]
        res.append(np.asfortranarray(np.transpose(c, (2, 1, 0))))
    return res


def header_of(datasets):
    """writeheader_hdf5's scalars of a decoded file, as ductgpu_h5_header keys."""
    h = {}
    for n in INT_NAMES:
        h[n] = int(datasets[n][0])
    for n in DBL_NAMES:
        h[HEADER_KEYS.get(n, n)] = float(datasets[n][0])
    return h
