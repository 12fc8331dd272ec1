"""Minimal reader for the PSI HDF5 layout used by POT3D's Br input maps.

POT3D reads its boundary map with ``rdhdf_2d`` (src/psi_io.f90:996), which
calls ``rdh5`` (src/psi_io.f90:285-625): one dataset named ``Data`` in the
root group, plus optional dimension-scale datasets ``dim1``, ``dim2``,
``dim3`` holding the coordinate of each (Fortran-order) axis.  The files the
reference ships are HDF5 superblock version 0, with a v1 B-tree symbol-table
root group and contiguous, unfiltered datasets.  This module parses exactly
that subset with no libhdf5 dependency, so host code and fixture scripts can
read the maps on machines without HDF5.

Array convention: HDF5 stores dims in C order, so a Fortran array
``f(nx, ny)`` appears as a C array of shape ``(ny, nx)``.  ``read_psi`` returns
the data transposed back to Fortran axis order, ``f[ix, iy]``, with
``scales[0]`` the ``dim1`` coordinate (length nx) and ``scales[1]`` ``dim2``.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class PsiFormatError(ValueError):
    """Raised when a file is not in the supported PSI HDF5 subset."""


@dataclass
class _Dataset:
    shape: tuple = ()
    dtype: np.dtype | None = None
    address: int = _UNDEF
    size: int = 0
    compact: bytes | None = None
    filtered: bool = False


@dataclass
class PsiData:
    """A PSI data set: ``data`` in Fortran axis order and its scales."""

    data: np.ndarray
    scales: list = field(default_factory=list)
    dtype: np.dtype | None = None

    @property
    def has_scales(self) -> bool:
        return len(self.scales) == self.data.ndim and all(s is not None for s in self.scales)


class _Reader:
    def __init__(self, buf: bytes):
        self.b = buf
        if buf[:8] != _SIG:
            raise PsiFormatError("not an HDF5 file (bad signature)")
        if buf[8] != 0:
            raise PsiFormatError(f"unsupported HDF5 superblock version {buf[8]}")
        self.so = buf[13]
        self.sl = buf[14]
        if self.so != 8 or self.sl != 8:
            raise PsiFormatError("only 8-byte offsets/lengths are supported")
        self.base = self._u(24, 8)
        # Root group symbol table entry starts at byte 56.
        ent = 56
        cache = self._u(ent + 16, 4)
        if cache != 1:
            raise PsiFormatError("root group entry has no cached symbol table")
        self.root_btree = self._u(ent + 24, 8)
        self.root_heap = self._u(ent + 32, 8)

    def _u(self, off: int, n: int) -> int:
        if off + n > len(self.b):
            raise PsiFormatError("truncated HDF5 file")
        return int.from_bytes(self.b[off:off + n], "little")

    def _addr(self, a: int) -> int:
        return self.base + a

    # ---- groups -------------------------------------------------------
    def _heap_data(self, heap_addr: int) -> int:
        off = self._addr(heap_addr)
        if self.b[off:off + 4] != b"HEAP":
            raise PsiFormatError("bad local heap signature")
        return self._addr(self._u(off + 24, 8))

    def _name(self, heap_data: int, name_off: int) -> str:
        s = heap_data + name_off
        e = self.b.index(b"\x00", s)
        return self.b[s:e].decode("ascii")

    def _walk_btree(self, addr: int, out: list) -> None:
        off = self._addr(addr)
        if self.b[off:off + 4] != b"TREE":
            raise PsiFormatError("bad B-tree node signature")
        level = self.b[off + 5]
        used = self._u(off + 6, 2)
        p = off + 24  # after signature, type, level, used, two siblings
        children = []
        for _ in range(used):
            p += self.sl  # key
            children.append(self._u(p, self.so))
            p += self.so
        for c in children:
            if level > 0:
                self._walk_btree(c, out)
            else:
                out.append(c)

    def root_members(self) -> dict:
        heap_data = self._heap_data(self.root_heap)
        snods: list = []
        self._walk_btree(self.root_btree, snods)
        members = {}
        for sn in snods:
            off = self._addr(sn)
            if self.b[off:off + 4] != b"SNOD":
                raise PsiFormatError("bad symbol-table node signature")
            nsym = self._u(off + 6, 2)
            e = off + 8
            for _ in range(nsym):
                name = self._name(heap_data, self._u(e, 8))
                members[name] = self._u(e + 8, 8)
                e += 40
        return members

    # ---- object headers -----------------------------------------------
    def _messages(self, oh_addr: int):
        off = self._addr(oh_addr)
        ver = self.b[off]
        if ver != 1:
            raise PsiFormatError(f"unsupported object header version {ver}")
        nmsg = self._u(off + 2, 2)
        hsize = self._u(off + 8, 4)
        blocks = [(off + 16, hsize)]
        seen = 0
        while blocks and seen < nmsg:
            start, length = blocks.pop(0)
            p = start
            end = start + length
            while p + 8 <= end and seen < nmsg:
                mtype = self._u(p, 2)
                msize = self._u(p + 2, 2)
                body = p + 8
                seen += 1
                if mtype == 0x0010:
                    blocks.append((self._addr(self._u(body, 8)), self._u(body + 8, 8)))
                else:
                    yield mtype, body, msize
                p = body + msize

    def dataset(self, oh_addr: int) -> _Dataset:
        ds = _Dataset()
        for mtype, body, msize in self._messages(oh_addr):
            if mtype == 0x0001:  # dataspace
                ver = self.b[body]
                ndim = self.b[body + 1]
                p = body + (8 if ver == 1 else 4)
                ds.shape = tuple(self._u(p + 8 * i, 8) for i in range(ndim))
            elif mtype == 0x0003:  # datatype
                cls = self.b[body] & 0x0F
                bits0 = self.b[body + 1]
                size = self._u(body + 4, 4)
                if cls != 1:
                    raise PsiFormatError("only floating-point datasets are supported")
                if bits0 & 1:
                    raise PsiFormatError("big-endian data is not supported")
                if size == 4:
                    ds.dtype = np.dtype("<f4")
                elif size == 8:
                    ds.dtype = np.dtype("<f8")
                else:
                    raise PsiFormatError(f"unsupported float size {size}")
            elif mtype == 0x0008:  # data layout
                ver = self.b[body]
                if ver == 3:
                    lcls = self.b[body + 1]
                    if lcls == 1:
                        ds.address = self._u(body + 2, 8)
                        ds.size = self._u(body + 10, 8)
                    elif lcls == 0:
                        n = self._u(body + 2, 2)
                        ds.compact = self.b[body + 4:body + 4 + n]
                    else:
                        raise PsiFormatError("chunked datasets are not supported")
                elif ver in (1, 2):
                    ndim = self.b[body + 1]
                    lcls = self.b[body + 2]
                    if lcls != 1:
                        raise PsiFormatError("only contiguous v1/v2 layouts are supported")
                    ds.address = self._u(body + 8, 8)
                    dims = [self._u(body + 16 + 4 * i, 4) for i in range(ndim)]
                    ds.size = int(np.prod(dims))
                else:
                    raise PsiFormatError(f"unsupported layout message version {ver}")
            elif mtype == 0x000B:  # filter pipeline
                ds.filtered = True
        return ds

    def read(self, oh_addr: int) -> np.ndarray:
        ds = self.dataset(oh_addr)
        if ds.dtype is None:
            raise PsiFormatError("dataset without a datatype message")
        if ds.filtered:
            raise PsiFormatError("filtered (compressed) datasets are not supported")
        count = int(np.prod(ds.shape)) if ds.shape else 1
        nbytes = count * ds.dtype.itemsize
        if ds.compact is not None:
            raw = ds.compact[:nbytes]
        else:
            if ds.address == _UNDEF:
                return np.zeros(ds.shape, ds.dtype)
            off = self._addr(ds.address)
            if off + nbytes > len(self.b):
                raise PsiFormatError("dataset extends past the end of the file")
            raw = self.b[off:off + nbytes]
        return np.frombuffer(raw, dtype=ds.dtype, count=count).reshape(ds.shape)


def read_psi(path) -> PsiData:
    """Read a PSI HDF5 file; return data in Fortran axis order plus scales.

    Mirrors ``rdh5`` (src/psi_io.f90:285-625): the dataset ``Data`` and its
    scales ``dim1..dimN``.  Raises ``PsiFormatError`` on anything outside the
    supported subset (the reference reports such files with a nonzero IERR).
    """
    with open(path, "rb") as fh:
        buf = fh.read()
    rd = _Reader(buf)
    members = rd.root_members()
    if "Data" not in members:
        raise PsiFormatError("no 'Data' dataset in the root group")
    c_arr = rd.read(members["Data"])
    data = np.ascontiguousarray(c_arr.T)  # back to Fortran axis order
    scales = []
    for d in range(data.ndim):
        nm = f"dim{d + 1}"
        if nm in members:
            s = np.array(rd.read(members[nm]), dtype=np.float64).reshape(-1)
            if s.size != data.shape[d]:
                raise PsiFormatError(f"scale {nm} has {s.size} points, data axis has {data.shape[d]}")
            scales.append(s)
        else:
            scales.append(None)
    return PsiData(data=data, scales=scales, dtype=c_arr.dtype)


# ---- writer -------------------------------------------------------------
#
# The files POT3D writes (wrhdf_2d/wrhdf_3d, src/psi_io.f90:629-925) hold
# ``Data`` plus one scale dataset ``dimN`` per axis, each scale marked with
# the string attribute CLASS = "DIMENSION_SCALE" (h5DSset_scale_f) so that
# rdh5's h5DSis_scale_f check accepts it, and named with NAME = "dimN".
# The writer below lays out the same HDF5 subset the reader parses:
# superblock version 0, one symbol-table root group (a v1 B-tree with one
# leaf, one local heap, one symbol-table node), version-1 object headers
# and contiguous, unfiltered little-endian floating-point datasets.  The
# DIMENSION_LIST / REFERENCE_LIST attributes that the HDF5 library adds
# when it attaches scales are not written: reading PSI files does not use
# them (rdh5 matches scales to axes by member order).

_GROUP_LEAF_K = 4
_GROUP_INTERNAL_K = 16
_HEAP_FREE_NULL = 1


def _pad8(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 8)


def _u(v: int, n: int) -> bytes:
    return int(v).to_bytes(n, "little")


def _msg(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = _pad8(body)
    return _u(mtype, 2) + _u(len(body), 2) + bytes([flags, 0, 0, 0]) + body


def _dataspace(shape) -> bytes:
    # version 1; the maximum dimensions equal the dimensions
    body = bytes([1, len(shape), 1 if shape else 0, 0]) + _u(0, 4)
    for d in shape:
        body += _u(d, 8)
    for d in shape:
        body += _u(d, 8)
    return body


def _float_type(itemsize: int) -> bytes:
    # class 1 (floating point), version 1, little-endian, IEEE layout
    if itemsize == 8:
        sign, eloc, esize, msize, bias = 63, 52, 11, 52, 1023
    else:
        sign, eloc, esize, msize, bias = 31, 23, 8, 23, 127
    return (bytes([0x11, 0x20, sign, 0]) + _u(itemsize, 4) + _u(0, 2) + _u(8 * itemsize, 2)
            + bytes([eloc, esize, 0, msize]) + _u(bias, 4))


def _string_attr(name: str, value: str) -> bytes:
    nm = name.encode("ascii") + b"\x00"
    val = value.encode("ascii") + b"\x00"
    dtype = bytes([0x13, 0, 0, 0]) + _u(len(val), 4)  # string, null-terminated, ASCII
    space = bytes([1, 0, 0, 0]) + _u(0, 4)              # scalar
    body = (bytes([1, 0]) + _u(len(nm), 2) + _u(len(dtype), 2) + _u(len(space), 2)
            + _pad8(nm) + _pad8(dtype) + _pad8(space) + val)
    return _msg(0x000C, body)


def _object_header(messages) -> bytes:
    body = b"".join(messages)
    return bytes([1, 0]) + _u(len(messages), 2) + _u(1, 4) + _u(len(body), 4) + _u(0, 4) + body


def write_psi(path, data, scales=None, hdf32: bool = False) -> None:
    """Write a PSI HDF5 file readable by ``read_psi`` and by rdh5.

    ``data`` is in Fortran axis order (as ``read_psi`` returns it), 1-3
    axes; ``scales`` is None or one 1-D array per axis; ``hdf32`` stores
    FP32 (POT3D's hdf32 option, src/psi_io.f90:629-925), else FP64.
    """
    data = np.asarray(data)
    if not 1 <= data.ndim <= 3:
        raise ValueError("PSI files hold 1-3 dimensional data")
    dt = np.dtype("<f4") if hdf32 else np.dtype("<f8")
    objs = [("Data", np.ascontiguousarray(data.T, dtype=dt), False)]
    if scales is not None:
        if len(scales) != data.ndim:
            raise ValueError("one scale per axis is required")
        for d, s in enumerate(scales):
            s = np.ascontiguousarray(np.asarray(s).reshape(-1), dtype=dt)
            if s.size != data.shape[d]:
                raise ValueError(f"scale {d + 1} has {s.size} points, axis has {data.shape[d]}")
            objs.append((f"dim{d + 1}", s, True))
    objs.sort(key=lambda o: o[0].encode("ascii"))

    # local heap data segment: "" at offset 0, then the names, then one
    # free block (next = end of list, size 16)
    heap_names = b"\x00" * 8
    name_off = {}
    for name, _, _ in objs:
        name_off[name] = len(heap_names)
        heap_names += _pad8(name.encode("ascii") + b"\x00")
    free_off = len(heap_names)
    heap_data = heap_names + _u(_HEAP_FREE_NULL, 8) + _u(16, 8)

    root_oh_addr = 96
    root_oh_size = 16 + 8 + 16
    btree_addr = root_oh_addr + root_oh_size
    btree_size = 24 + (2 * _GROUP_INTERNAL_K) * 8 + (2 * _GROUP_INTERNAL_K + 1) * 8
    heap_addr = btree_addr + btree_size
    heap_data_addr = heap_addr + 32
    snod_addr = heap_data_addr + len(heap_data)
    snod_size = 8 + 2 * _GROUP_LEAF_K * 40
    if len(objs) > 2 * _GROUP_LEAF_K:
        raise ValueError("too many datasets for one symbol-table node")

    # object headers (their data addresses are patched in below)
    def headers(data_addrs):
        out = []
        for (name, arr, is_scale), da in zip(objs, data_addrs):
            msgs = [_msg(0x0001, _dataspace(arr.shape)), _msg(0x0003, _float_type(arr.itemsize), 1),
                    _msg(0x0005, bytes([2, 2, 2, 1]) + _u(0, 4), 1),
                    _msg(0x0008, bytes([3, 1]) + _u(da, 8) + _u(arr.nbytes, 8))]
            if is_scale:
                msgs += [_string_attr("CLASS", "DIMENSION_SCALE"), _string_attr("NAME", name)]
            out.append(_object_header(msgs))
        return out

    hdrs = headers([0] * len(objs))
    addr = snod_addr + snod_size
    oh_addrs = []
    for h in hdrs:
        oh_addrs.append(addr)
        addr += len(h)
    data_addrs = []
    for _, arr, _ in objs:
        addr += -addr % 8
        data_addrs.append(addr)
        addr += arr.nbytes
    eof = addr
    hdrs = headers(data_addrs)

    buf = bytearray(eof)
    sb = (_SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + _u(_GROUP_LEAF_K, 2) + _u(_GROUP_INTERNAL_K, 2) + _u(0, 4)
          + _u(0, 8) + _u(_UNDEF, 8) + _u(eof, 8) + _u(_UNDEF, 8))
    root_entry = _u(0, 8) + _u(root_oh_addr, 8) + _u(1, 4) + _u(0, 4) + _u(btree_addr, 8) + _u(heap_addr, 8)
    buf[0:96] = sb + root_entry
    buf[root_oh_addr:root_oh_addr + root_oh_size] = _object_header([_msg(0x0011, _u(btree_addr, 8)
                                                                         + _u(heap_addr, 8))])
    tree = (b"TREE" + bytes([0, 0]) + _u(1, 2) + _u(_UNDEF, 8) + _u(_UNDEF, 8)
            + _u(0, 8) + _u(snod_addr, 8) + _u(name_off[objs[-1][0]], 8))
    buf[btree_addr:btree_addr + len(tree)] = tree
    heap = b"HEAP" + bytes([0, 0, 0, 0]) + _u(len(heap_data), 8) + _u(free_off, 8) + _u(heap_data_addr, 8)
    buf[heap_addr:heap_addr + 32] = heap
    buf[heap_data_addr:heap_data_addr + len(heap_data)] = heap_data
    snod = b"SNOD" + bytes([1, 0]) + _u(len(objs), 2)
    for (name, _, _), oa in zip(objs, oh_addrs):
        snod += _u(name_off[name], 8) + _u(oa, 8) + _u(0, 4) + _u(0, 4) + b"\x00" * 16
    buf[snod_addr:snod_addr + len(snod)] = snod
    for h, oa in zip(hdrs, oh_addrs):
        buf[oa:oa + len(h)] = h
    for (_, arr, _), da in zip(objs, data_addrs):
        buf[da:da + arr.nbytes] = arr.tobytes()
    with open(path, "wb") as fh:
        fh.write(bytes(buf))
