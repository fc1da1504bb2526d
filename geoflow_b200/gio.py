"""GIO state I/O (pdeint/io_base.hpp, cdg/io/gio.hpp/.ipp) over device memory.

`GIO(grid, traits, ctx)` mirrors GIO<Types>(grid, traits, comm):
write_state / read_state / read_state_info with the reference's StateInfo
and Traits fields, file names and file layout:
  - GIO_POSIX: one file per state component and rank,
    "<odir>/<svar>.<index:0wtime>.<rank:0wtask>.out" (gio.ipp:68-77, 203-207);
  - GIO_COLL: one file per component (or, with multivar, one per state)
    holding every rank's slab at the prefix sum of the ranks' ndof
    (gio.ipp:100-128, 735-790), the collective MPI-IO write replaced by
    each rank writing its own byte range of the shared file between two
    barriers of the torch.distributed group.
The field bytes move between HBM and the file inside libgfgpu
(gf_gio_write_data / gf_gio_read_data: pinned double-buffered staging);
this module only names files, builds headers and computes offsets.

Departures from the reference, each a defect there:
  - write_posix reopens the file with "wb" after write_header_posix
    (gio.ipp:356-359), truncating the header that read_posix then expects;
    here the header is kept, so the files read back with read_posix's logic;
  - the multivar collective write passes a file name that was never set
    (gio.ipp:222-226 formats cfname_ but writes fname_); here the formatted
    name is used.
Consistency checks that the reference makes with assert (version, dim,
grid type, sizes) raise ValueError here.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

GIO_POSIX, GIO_COLL = 0, 1
# GElemType (include/gtypes.h:171)
GE_REGULAR, GE_DEFORMED, GE_2DEMBEDDED = 0, 1, 2
# GStateCompType (include/gtypes.h:190): prescribed components are not read
GSC_KINETIC, GSC_PRESCRIBED = 0, 7

_GTYPE_OF_GEOMETRY = {"affine": GE_REGULAR, "regular": GE_REGULAR, "deformed": GE_DEFORMED,
                      "embedded": GE_2DEMBEDDED}


@dataclass
class GIOTraits:
    """IOBase::Traits (pdeint/io_base.hpp:35-46)."""
    io_type: int = GIO_COLL
    ivers: int = 0
    multivar: bool = False
    prgrid: bool = False
    wtime: int = 6
    wtask: int = 5
    wfile: int = 2048
    dim: int = 3
    idir: str = "."
    odir: str = "."


@dataclass
class StateInfo:
    """GStateInfo (pdeint/equation_base.hpp:45-59): sttype 0 names files as
    a physical state, otherwise as a grid file (gio.ipp:68-77)."""
    sttype: int = 1
    gtype: int = 0
    index: int = 0
    nelems: int = 0
    cycle: int = 0
    time: float = 0.0
    svars: list = field(default_factory=list)
    icomptype: list = field(default_factory=list)
    porder: np.ndarray | None = None
    elemids: np.ndarray | None = None
    idir: str = "."
    odir: str = "."


def _dtype_code(t):
    import torch
    if t.dtype == torch.float64:
        return A.GF_F64, 8
    if t.dtype == torch.float32:
        return A.GF_F32, 4
    raise ValueError(f"GIO fields are float64 or float32, not {t.dtype}")


class GIO:
    """GIO<Types> over a grid (GridBox, ShardGrid or a Problem's grid).

    ctx: the Context whose device holds the fields; gtype: the grid's
    GElemType (taken from a Problem's geometry when one is passed);
    elemids: this rank's element keys (GGrid::elemids; the box grid leaves
    them 0); group: the torch.distributed group of the ranks sharing
    collective files (default: the default group when initialised)."""

    def __init__(self, grid, traits: GIOTraits, ctx=None, gtype=None, elemids=None, group=None):
        if hasattr(grid, "grid") and hasattr(grid, "ctx"):  # a Problem
            ctx = ctx or grid.ctx
            if gtype is None:
                gtype = _GTYPE_OF_GEOMETRY[getattr(grid, "geometry", "affine")]
            grid = grid.grid
        self.grid, self.traits, self.ctx = grid, traits, ctx
        self.gtype = GE_REGULAR if gtype is None else int(gtype)
        self.dim, self.p = int(grid.dim), int(grid.p)
        self.nelems = int(grid.nelems)
        self.ndof = self.nelems * int(grid.n) ** self.dim
        self.elemids = (np.zeros(self.nelems, np.uint64) if elemids is None
                        else np.ascontiguousarray(elemids, dtype=np.uint64))
        if self.elemids.size != self.nelems:
            raise ValueError("elemids needs one key per element")
        self.group = group
        self.rank, self.nranks = self._rank_world()
        self.init()

    # ---- ranks ----
    def _rank_world(self):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(self.group), dist.get_world_size(self.group)
        return 0, 1

    def _allgather(self, obj):
        if self.nranks == 1:
            return [obj]
        import torch.distributed as dist
        out = [None] * self.nranks
        dist.all_gather_object(out, obj, group=self.group)
        return out

    def _barrier(self):
        if self.nranks > 1:
            import torch.distributed as dist
            dist.barrier(group=self.group)

    def init(self):
        """GIO::init (gio.ipp:88-130): each rank's ndof extent, its
        displacement (prefix sum over lower ranks) and the global size."""
        ext = self._allgather(self.ndof)
        self.extent = [int(v) for v in ext]
        self.state_disp = int(sum(self.extent[:self.rank]))
        self.gdof = int(sum(self.extent))
        self.gnelems = int(sum(self._allgather(self.nelems)))

    # ---- names and headers ----
    def filename(self, dirname, svar, info: StateInfo, coll: bool):
        """gio.ipp:68-77 formats, filled as write_state_impl does (203-216)."""
        t = self.traits
        if coll:
            name = "%s/%s.%0*d.out" % (dirname, svar, t.wtime, info.index)
        elif info.sttype == 0:
            name = "%s/%s.%0*d.%0*d.out" % (dirname, svar, t.wtime, info.index, t.wtask, self.rank)
        else:  # grid-file format: one integer field, filled by the index
            name = "%s/%s.%0*d.out" % (dirname, svar, t.wtask, info.index)
        if len(name) >= t.wfile:
            raise ValueError(f"file name longer than wfile={t.wfile}")
        return name

    def _header(self, info: StateInfo, coll: bool):
        h = A.GioHeader()
        h.ivers, h.dim = self.traits.ivers, self.dim
        h.nelems = self.gnelems if coll else self.nelems
        h.gtype, h.cycle, h.time = self.gtype, int(info.cycle), float(info.time)
        h.multivar = int(bool(self.traits.multivar))
        numr = 1 if self.traits.ivers == 0 else h.nelems
        porder = np.full((numr, self.dim), self.p, dtype=np.int32)
        return h, porder

    def _keys(self, coll: bool):
        if not coll:
            return self.elemids
        return np.ascontiguousarray(np.concatenate(self._allgather(self.elemids)), np.uint64)

    # ---- data movement (libgfgpu) ----
    def _write_header(self, path, h, porder, keys, dtype):
        rc = A.load().gf_gio_write_header(self.ctx.handle if self.ctx else None, path.encode(),
                                          C.byref(h), porder.ctypes.data_as(C.c_void_p),
                                          keys.ctypes.data_as(C.c_void_p), dtype)
        self._check(rc, "gf_gio_write_header")

    def _write_data(self, path, t, offset):
        dtype, _ = _dtype_code(t)
        self._check(A.load().gf_gio_write_data(self.ctx.handle, path.encode(), dtype,
                                               C.c_void_p(t.data_ptr()), t.numel(), offset),
                    "gf_gio_write_data")

    def _read_data(self, path, t, offset):
        dtype, _ = _dtype_code(t)
        self._check(A.load().gf_gio_read_data(self.ctx.handle, path.encode(), dtype,
                                              C.c_void_p(t.data_ptr()), t.numel(), offset),
                    "gf_gio_read_data")

    def _read_header(self, path, fbytes):
        h = A.GioHeader()
        dtype = {8: A.GF_F64, 4: A.GF_F32}.get(fbytes, -1)
        lib = A.load()
        handle = self.ctx.handle if self.ctx else None
        self._check(lib.gf_gio_read_header(handle, path.encode(), dtype, C.byref(h), None, 0, None,
                                           0), "gf_gio_read_header")
        porder = np.zeros((h.porder_rows, h.dim), dtype=np.int32)
        keys = np.zeros(h.nelems, dtype=np.uint64)
        self._check(lib.gf_gio_read_header(handle, path.encode(), dtype, C.byref(h),
                                           porder.ctypes.data_as(C.c_void_p), porder.size,
                                           keys.ctypes.data_as(C.c_void_p), keys.size),
                    "gf_gio_read_header")
        return h, porder, keys

    def _check(self, rc, what):
        if rc < 0:
            msg = (A.load().gf_ctx_last_error(self.ctx.handle).decode()
                   if self.ctx is not None else "")
            raise A.GFError(rc, f"{what}: {msg}")

    def _check_field(self, t):
        if t.numel() != self.ndof or not t.is_contiguous():
            raise ValueError(f"state component must be a contiguous field of {self.ndof} values")

    # ---- IOBase interface ----
    def write_state(self, filepref: str, info: StateInfo, u):
        """GIO::write_state_impl (gio.ipp:155-231)."""
        t = self.traits
        coll = t.io_type == GIO_COLL
        info.gtype = self.gtype
        info.nelems = self.gnelems if coll else self.nelems
        h, porder = self._header(info, coll)
        info.porder = porder
        keys = self._keys(coll)
        for c in u:
            self._check_field(c)
        if not t.multivar:
            if len(info.svars) < len(u):
                raise ValueError("info.svars must name every state component")
            for j, c in enumerate(u):
                dtype, fb = _dtype_code(c)
                name = self.filename(info.odir, info.svars[j], info, coll)
                hb = A.load().gf_gio_header_bytes(t.ivers, self.dim, h.nelems, dtype)
                if not coll:
                    self._write_header(name, h, porder, keys, dtype)
                    self._write_data(name, c, hb)
                else:
                    if self.rank == 0:
                        self._write_header(name, h, porder, keys, dtype)
                    self._barrier()
                    self._write_data(name, c, hb + self.state_disp * fb)
                    self._barrier()
            return
        if not coll:
            raise ValueError("multivar files are collective (io_type GIO_COLL)")
        if not filepref:
            raise ValueError("a multivar write needs a file prefix")
        dtype, fb = _dtype_code(u[0])
        name = self.filename(info.odir, filepref, info, True)
        hb = A.load().gf_gio_header_bytes(t.ivers, self.dim, h.nelems, dtype)
        if self.rank == 0:
            self._write_header(name, h, porder, keys, dtype)
        self._barrier()
        for j, c in enumerate(u):
            if _dtype_code(c)[0] != dtype:
                raise ValueError("multivar components must share one dtype")
            self._write_data(name, c, hb + (j * self.gdof + self.state_disp) * fb)
        self._barrier()

    def _check_read(self, h, path):
        if h.ivers != self.traits.ivers:
            raise ValueError(f"{path}: incompatible file version number {h.ivers}")
        if h.dim != self.dim:
            raise ValueError(f"{path}: file dimension {h.dim} incompatible with the grid")
        if h.gtype != self.gtype:
            raise ValueError(f"{path}: file grid type {h.gtype} incompatible with the grid")

    def _fill_info(self, info, h, porder, keys):
        info.nelems, info.gtype = int(h.nelems), int(h.gtype)
        info.cycle, info.time = int(h.cycle), float(h.time)
        info.porder, info.elemids = porder, keys

    def read_state(self, filepref: str, info: StateInfo, u, bstate: bool = True):
        """GIO::read_state_impl (gio.ipp:245-307); components whose
        info.icomptype is GSC_PRESCRIBED are skipped."""
        t = self.traits
        coll = t.io_type == GIO_COLL
        if not t.multivar:
            nt = len(u) if bstate else 1
            for j in range(nt):
                if j < len(info.icomptype) and info.icomptype[j] == GSC_PRESCRIBED:
                    continue
                name = self.filename(info.idir, info.svars[j], info, coll)
                fb = _dtype_code(u[j])[1] if bstate else 0
                h, porder, keys = self._read_header(name, fb)
                self._check_read(h, name)
                self._fill_info(info, h, porder, keys)
                if not bstate:
                    continue
                self._check_field(u[j])
                if coll:
                    if h.ndata != self.gdof:
                        raise ValueError(f"{name} holds {h.ndata} values, the ranks {self.gdof}")
                    self._read_data(name, u[j], h.header_bytes + self.state_disp * fb)
                else:
                    if h.ndata != self.ndof:
                        raise ValueError(f"{name} holds {h.ndata} values, the field {self.ndof}")
                    self._read_data(name, u[j], h.header_bytes)
            return
        if not coll:
            raise ValueError("multivar files are collective (io_type GIO_COLL)")
        name = self.filename(info.idir, filepref, info, True)
        fb = _dtype_code(u[0])[1] if bstate else 0
        h, porder, keys = self._read_header(name, fb)
        self._check_read(h, name)
        self._fill_info(info, h, porder, keys)
        if not bstate:
            return
        for j, c in enumerate(u):
            self._check_field(c)
            self._read_data(name, c, h.header_bytes + (j * self.gdof + self.state_disp) * fb)

    def read_state_info(self, filename: str, info: StateInfo, fbytes: int = 0):
        """GIO::read_state_info_impl (gio.ipp:320-333): the header of one
        file into info (fbytes 0: Ftype inferred from the file size)."""
        h, porder, keys = self._read_header(filename, fbytes)
        self._fill_info(info, h, porder, keys)
        return h
