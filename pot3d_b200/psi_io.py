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
