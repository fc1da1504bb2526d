"""GIO POSIX file format, restated in numpy (TEST INFRASTRUCTURE ONLY).

Used by tests/ as the checker of the library's GIO reader and writer; the
product never imports it.  Follows GeoFLOW src/cdg/io/gio.ipp:
  - header field order and types: write_header_posix (459-503) and
    read_header (587-660): int32 ivers, int32 dim, uint64 nelems,
    int32 porder[numr*dim] (numr = 1 if ivers == 0 else nelems), int32 gtype,
    uint64 cycle, Ftype time, int32 multivar, uint64 elemids[nelems];
  - header size: sz_header (676-690);
  - field length: read_posix (416-429);
  - collective layout: init (100-128, each rank's slab at the prefix sum of
    the ranks' ndof) and write_coll (735-790, component j of a multivar file
    at header + j * global ndof * sizeof(Ftype)).
Parity is pinned to the reference's own byte layout read from those lines,
and to the header fields the reference's Python reader
(analysis/python/g2vtk:158-195) parses from files of this layout
(tests/golden/gio_g2vtk.json).  The reference's writer cannot produce a
golden file (write_posix reopens the file with "wb" after the header,
gio.ipp:356-359, which truncates it).
"""
from __future__ import annotations

import struct

import numpy as np


def header_bytes(ivers, dim, nelems, fbytes=8):
    """GIO::sz_header (gio.ipp:676-690)."""
    numr = 1 if ivers == 0 else nelems
    return (numr * dim + 4) * 4 + 2 * 8 + fbytes + nelems * 8


def ndata(ivers, dim, nelems, porder):
    """Values per field from the expansion orders (gio.ipp:416-429)."""
    po = np.asarray(porder, dtype=np.int64).reshape(-1, dim)
    per = np.prod(po + 1, axis=1)
    return int(per[0]) * nelems if ivers == 0 else int(per.sum())


def header_image(ivers, dim, nelems, porder, gtype, cycle, time, multivar, elemids=None,
                 fbytes=8):
    """The header as bytes, one field after another (gio.ipp:474-496)."""
    numr = 1 if ivers == 0 else nelems
    po = np.asarray(porder, dtype=np.int32).reshape(numr, dim)
    keys = np.zeros(nelems, np.uint64) if elemids is None else np.asarray(elemids, np.uint64)
    assert keys.size == nelems
    b = bytearray()
    b += struct.pack("<iiQ", ivers, dim, nelems)
    b += po.astype("<i4").tobytes()
    b += struct.pack("<iQ", gtype, cycle)
    b += struct.pack("<d" if fbytes == 8 else "<f", time)
    b += struct.pack("<i", int(multivar))
    b += keys.astype("<u8").tobytes()
    assert len(b) == header_bytes(ivers, dim, nelems, fbytes)
    return bytes(b)


def write(path, data, ivers, dim, nelems, porder, gtype=0, cycle=0, time=0.0, multivar=0,
          elemids=None):
    """A POSIX GIO file: header, then the field (gio.ipp:347-377 as
    read_posix expects it)."""
    data = np.ascontiguousarray(data)
    fbytes = data.dtype.itemsize
    assert data.size == ndata(ivers, dim, nelems, porder)
    with open(path, "wb") as f:
        f.write(header_image(ivers, dim, nelems, porder, gtype, cycle, time, multivar, elemids,
                             fbytes))
        f.write(data.astype("<f8" if fbytes == 8 else "<f4").tobytes())


def read(path, fbytes=8):
    """(header dict, field) of a POSIX GIO file (gio.ipp:392-444, 587-620)."""
    raw = open(path, "rb").read()
    ivers, dim, nelems = struct.unpack_from("<iiQ", raw, 0)
    o = 16
    numr = 1 if ivers == 0 else nelems
    porder = np.frombuffer(raw, "<i4", numr * dim, o).reshape(numr, dim).copy()
    o += 4 * numr * dim
    gtype, cycle = struct.unpack_from("<iQ", raw, o)
    o += 12
    (time,) = struct.unpack_from("<d" if fbytes == 8 else "<f", raw, o)
    o += fbytes
    (multivar,) = struct.unpack_from("<i", raw, o)
    o += 4
    elemids = np.frombuffer(raw, "<u8", nelems, o).copy()
    o += 8 * nelems
    assert o == header_bytes(ivers, dim, nelems, fbytes)
    nd = ndata(ivers, dim, nelems, porder)
    data = np.frombuffer(raw, "<f8" if fbytes == 8 else "<f4", nd, o).copy()
    hdr = dict(ivers=ivers, dim=dim, nelems=nelems, porder=porder, gtype=gtype, cycle=cycle,
               time=time, multivar=multivar, elemids=elemids, header_bytes=o, ndata=nd)
    return hdr, data


def coll_offsets(ndof_per_rank, hbytes, fbytes=8, comp=0):
    """Byte offset of each rank's slab of component `comp` in a collective
    file (gio.ipp:100-128, 770-775)."""
    ext = np.asarray(ndof_per_rank, dtype=np.int64)
    disp = np.concatenate([[0], np.cumsum(ext)[:-1]])
    return [int(hbytes + comp * ext.sum() * fbytes + d * fbytes) for d in disp]


def filename(odir, svar, index, rank, sttype=0, wtime=6, wtask=5, coll=False):
    """GIO file names (gio.ipp:68-77 formats, filled by the sprintf calls of
    write_state_impl 203-216).  A grid file's POSIX format has one integer
    field, filled by `index` (the first integer argument)."""
    if coll:
        return "%s/%s.%0*d.out" % (odir, svar, wtime, index)
    if sttype == 0:
        return "%s/%s.%0*d.%0*d.out" % (odir, svar, wtime, index, wtask, rank)
    return "%s/%s.%0*d.out" % (odir, svar, wtask, index)
