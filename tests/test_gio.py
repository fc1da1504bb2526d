"""GIO state files (cdg/io/gio.ipp) through libgfgpu and geoflow_b200.gio,
checked byte for byte against the numpy restatement in oracle/gio_oracle.py.

CPU: header bytes and sizes, header parsing (no device is touched with a
NULL context), file names, and the collective layout of two gloo ranks
(each rank's slab at the prefix sum of the ranks' ndof), with the field
bytes moved by a host stand-in for the device copy.  GPU: device fields
written and read back bit-exact, files identical to the oracle's, the
two-buffer staging across several 32 MiB chunks, and the consistency errors.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from geoflow_b200 import _abi as A
from geoflow_b200 import gio as G
import gio_oracle as GO

HEADER_CASES = [(0, 3, 8, 7, 8), (0, 2, 5, 4, 8), (1, 3, 3, 5, 8), (0, 3, 6, 3, 4),
                (1, 2, 4, 6, 4), (0, 1, 9, 2, 8)]


def _hdr(ivers, dim, nelems, p, gtype=0, cycle=17, time=0.125, multivar=0):
    h = A.GioHeader()
    h.ivers, h.dim, h.nelems, h.gtype = ivers, dim, nelems, gtype
    h.cycle, h.time, h.multivar = cycle, time, multivar
    numr = 1 if ivers == 0 else nelems
    porder = np.full((numr, dim), p, dtype=np.int32)
    if ivers:
        porder += (np.arange(numr * dim, dtype=np.int32) % 2).reshape(numr, dim)
    return h, porder


def test_header_size_matches_sz_header():
    lib = A.load()
    for ivers, dim, ne, p, fb in HEADER_CASES:
        dt = A.GF_F64 if fb == 8 else A.GF_F32
        assert lib.gf_gio_header_bytes(ivers, dim, ne, dt) == GO.header_bytes(ivers, dim, ne, fb)
    # a known answer: version 0, 3-d, 2 elements, double: 4+4+8 + 3*4 + 4+8+8+4 + 2*8
    assert GO.header_bytes(0, 3, 2, 8) == 68
    assert lib.gf_gio_header_bytes(0, 4, 2, A.GF_F64) == A.GF_ERR_ARG


@pytest.mark.parametrize("case", HEADER_CASES)
@pytest.mark.parametrize("keys", [False, True])
def test_write_header_bytes_match_oracle(tmp_path, case, keys):
    ivers, dim, ne, p, fb = case
    h, porder = _hdr(ivers, dim, ne, p, gtype=2 if dim == 2 else 0)
    ids = np.arange(ne, dtype=np.uint64) * 7919 + 3 if keys else None
    path = str(tmp_path / "h.out")
    dt = A.GF_F64 if fb == 8 else A.GF_F32
    rc = A.load().gf_gio_write_header(None, path.encode(), C.byref(h),
                                      porder.ctypes.data_as(C.c_void_p),
                                      ids.ctypes.data_as(C.c_void_p) if keys else None, dt)
    assert rc == 0
    ref = GO.header_image(ivers, dim, ne, porder, h.gtype, h.cycle, h.time, 0, ids, fb)
    assert open(path, "rb").read() == ref


@pytest.mark.parametrize("case", HEADER_CASES)
def test_read_header_parses_oracle_files(tmp_path, case):
    ivers, dim, ne, p, fb = case
    _, porder = _hdr(ivers, dim, ne, p)
    nd = GO.ndata(ivers, dim, ne, porder)
    rng = np.random.default_rng(ne)
    data = rng.standard_normal(nd).astype(np.float64 if fb == 8 else np.float32)
    ids = rng.integers(0, 2**62, ne, dtype=np.uint64)
    path = str(tmp_path / "f.out")
    GO.write(path, data, ivers, dim, ne, porder, gtype=1, cycle=42, time=2.5, elemids=ids)
    lib = A.load()
    for dt in (-1, A.GF_F64 if fb == 8 else A.GF_F32):  # inferred and given Ftype
        h = A.GioHeader()
        po = np.zeros_like(porder)
        ko = np.zeros(ne, np.uint64)
        assert lib.gf_gio_read_header(None, path.encode(), dt, C.byref(h),
                                      po.ctypes.data_as(C.c_void_p), po.size,
                                      ko.ctypes.data_as(C.c_void_p), ko.size) == 0
        assert (h.ivers, h.dim, h.nelems, h.gtype, h.cycle, h.multivar) == (ivers, dim, ne, 1, 42, 0)
        assert h.time == 2.5 and h.float_bytes == fb and h.ndata == nd
        assert h.header_bytes == GO.header_bytes(ivers, dim, ne, fb)
        assert np.array_equal(po, porder) and np.array_equal(ko, ids)
    # the other float size does not fit the file
    other = A.GF_F32 if fb == 8 else A.GF_F64
    h = A.GioHeader()
    assert lib.gf_gio_read_header(None, path.encode(), other, C.byref(h), None, 0, None,
                                  0) == A.GF_ERR_IO
    hdr, back = GO.read(path, fb)
    assert np.array_equal(back, data) and hdr["cycle"] == 42


def test_read_header_rejects_bad_files(tmp_path):
    lib = A.load()
    _, porder = _hdr(0, 3, 4, 3)
    path = str(tmp_path / "t.out")
    GO.write(path, np.zeros(GO.ndata(0, 3, 4, porder)), 0, 3, 4, porder)
    raw = open(path, "rb").read()
    h = A.GioHeader()
    for cut in (10, 40, len(raw) - 5):  # truncated header, truncated data
        open(path, "wb").write(raw[:cut])
        assert lib.gf_gio_read_header(None, path.encode(), A.GF_F64, C.byref(h), None, 0, None,
                                      0) == A.GF_ERR_IO
    assert lib.gf_gio_read_header(None, str(tmp_path / "none.out").encode(), A.GF_F64, C.byref(h),
                                  None, 0, None, 0) == A.GF_ERR_IO
    open(path, "wb").write(raw)
    small = np.zeros(1, np.uint64)
    assert lib.gf_gio_read_header(None, path.encode(), A.GF_F64, C.byref(h), None, 0,
                                  small.ctypes.data_as(C.c_void_p), 1) == A.GF_ERR_ARG


def test_files_match_reference_g2vtk_reader(tmp_path):
    """Pins: files of the oracle's layout, and the header fields the
    reference's own Python reader (analysis/python/g2vtk) parsed from them
    (tests/golden/make_gio_golden.py).  The library writes the same bytes
    and parses the same fields.  g2vtk stops after `time` (it predates the
    multivar flag and element keys of gio.ipp:489-496): its data offset is
    that of the multivar field."""
    import json
    from pathlib import Path
    golden = json.loads((Path(__file__).parent / "golden" / "gio_g2vtk.json").read_text())
    lib = A.load()
    for g in golden:
        dim, ne, p, fb, gtype, cycle, time = g["case"]
        raw = bytes.fromhex(g["file_hex"])
        hbytes = GO.header_bytes(0, dim, ne, fb)
        h, porder = _hdr(0, dim, ne, p, gtype=gtype, cycle=cycle, time=time)
        ids = np.arange(ne, dtype=np.uint64) * 11 + 5
        path = str(tmp_path / "g.out")
        dt = A.GF_F64 if fb == 8 else A.GF_F32
        assert lib.gf_gio_write_header(None, path.encode(), C.byref(h),
                                       porder.ctypes.data_as(C.c_void_p),
                                       ids.ctypes.data_as(C.c_void_p), dt) == 0
        assert open(path, "rb").read() == raw[:hbytes]
        open(path, "wb").write(raw)
        r = A.GioHeader()
        po = np.zeros(dim, np.int32)
        assert lib.gf_gio_read_header(None, path.encode(), -1, C.byref(r),
                                      po.ctypes.data_as(C.c_void_p), dim, None, 0) == 0
        ref = g["g2vtk"]
        assert (r.ivers, r.dim, r.nelems, list(po), r.gtype, r.cycle, r.time) == (
            ref["vers"], ref["dim"], ref["nelems"], ref["porder"], ref["gtype"], ref["cycle"],
            ref["time"])
        assert r.float_bytes == fb and ref["skip"] == hbytes - 4 - 8 * ne


class _Grid:
    def __init__(self, dim, nelems, p):
        self.dim, self.p, self.n, self.nelems = dim, p, p + 1, nelems


def test_file_names_follow_gio_formats():
    g = G.GIO(_Grid(3, 4, 3), G.GIOTraits(io_type=G.GIO_POSIX))
    info = G.StateInfo(sttype=0, index=12)
    assert g.filename("out", "u1", info, False) == GO.filename("out", "u1", 12, 0, sttype=0)
    assert g.filename("out", "u1", info, False) == "out/u1.000012.00000.out"
    info.sttype = 1
    assert g.filename("out", "xgrid", info, False) == "out/xgrid.00012.out"
    assert g.filename("out", "u1", info, True) == "out/u1.000012.out"


class HostGIO(G.GIO):
    """GIO whose field bytes move from CPU tensors (test stand-in for the
    device copy; headers, names and offsets are the product's)."""

    def _write_data(self, path, t, offset):
        with open(path, "r+b") as f:
            f.seek(offset)
            f.write(t.numpy().tobytes())

    def _read_data(self, path, t, offset):
        with open(path, "rb") as f:
            f.seek(offset)
            a = np.frombuffer(f.read(t.numel() * t.element_size()),
                              np.float64 if t.dtype == torch.float64 else np.float32)
        t.copy_(torch.from_numpy(a.copy()))


def _coll_worker(rank, world, port, outdir, multivar, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p, dim = 3, 3
        nel = [3, 5][rank]  # ragged shards
        ndof = nel * (p + 1) ** dim
        ids = np.arange(nel, dtype=np.uint64) + 100 * (rank + 1)
        io = HostGIO(_Grid(dim, nel, p), G.GIOTraits(io_type=G.GIO_COLL, multivar=multivar),
                     elemids=ids)
        rng = np.random.default_rng(rank)
        u = [torch.from_numpy(rng.standard_normal(ndof)) for _ in range(2)]
        info = G.StateInfo(sttype=0, index=3, cycle=9, time=0.5, svars=["u1", "u2"], odir=outdir,
                           idir=outdir)
        io.write_state("state", info, u)
        back = [torch.zeros(ndof, dtype=torch.float64) for _ in range(2)]
        info2 = G.StateInfo(sttype=0, index=3, svars=["u1", "u2"], idir=outdir)
        io.read_state("state", info2, back)
        ok = all(torch.equal(a, b) for a, b in zip(u, back))
        q.put((rank, ok, [a.numpy() for a in u], ids, info2.nelems, info2.cycle))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("multivar", [False, True])
def test_collective_layout_two_ranks(tmp_path, multivar):
    import torch.multiprocessing as mp
    from socket import socket
    with socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_coll_worker, args=(r, 2, port, str(tmp_path), multivar, q))
             for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda r: r[0])
    for pr in procs:
        pr.join(60)
        assert pr.exitcode == 0
    assert all(r[1] for r in res)
    assert all(r[4] == 8 and r[5] == 9 for r in res)  # global nelems and cycle read back
    keys = np.concatenate([res[0][3], res[1][3]])
    porder = np.full((1, 3), 3, np.int32)
    comps = [np.concatenate([res[0][2][j], res[1][2][j]]) for j in range(2)]
    if multivar:
        ref = GO.header_image(0, 3, 8, porder, 0, 9, 0.5, 1, keys) + b"".join(
            c.tobytes() for c in comps)
        assert open(tmp_path / "state.000003.out", "rb").read() == ref
    else:
        for j, name in enumerate(["u1", "u2"]):
            hdr, data = GO.read(str(tmp_path / f"{name}.000003.out"))
            assert hdr["nelems"] == 8 and np.array_equal(hdr["elemids"], keys)
            assert np.array_equal(data, comps[j])
            assert GO.coll_offsets([3 * 64, 5 * 64], hdr["header_bytes"])[1] == \
                hdr["header_bytes"] + 3 * 64 * 8


# ---------------------------------------------------------------- GPU ----

@pytest.mark.gpu
@pytest.mark.parametrize("ivers,dtype", [(0, torch.float64), (1, torch.float64),
                                         (0, torch.float32)])
def test_device_write_matches_oracle_and_reads_back(ctx, tmp_path, ivers, dtype):
    lib = A.load()
    dim, ne, p = 3, 11, 6
    h, porder = _hdr(ivers, dim, ne, p, cycle=5, time=1.75)
    if ivers:
        porder[:] = p  # uniform orders written as one row per element
    nd = GO.ndata(ivers, dim, ne, porder)
    rng = np.random.default_rng(1)
    host = rng.standard_normal(nd).astype(np.float64 if dtype == torch.float64 else np.float32)
    ids = np.arange(ne, dtype=np.uint64) * 3
    u = torch.from_numpy(host).cuda()
    dt = A.GF_F64 if dtype == torch.float64 else A.GF_F32
    path = str(tmp_path / "d.out")
    ctx.check(lib.gf_gio_write(ctx.handle, path.encode(), C.byref(h),
                               porder.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p),
                               dt, C.c_void_p(u.data_ptr()), nd))
    ref = str(tmp_path / "r.out")
    GO.write(ref, host, ivers, dim, ne, porder, gtype=0, cycle=5, time=1.75, elemids=ids)
    assert open(path, "rb").read() == open(ref, "rb").read()
    back = torch.full_like(u, -1.0)
    hout = A.GioHeader()
    ctx.check(lib.gf_gio_read(ctx.handle, ref.encode(), dt, C.c_void_p(back.data_ptr()), nd,
                              C.byref(hout)))
    assert torch.equal(back, u) and hout.cycle == 5 and hout.ndata == nd
    # a field of the wrong length is refused before any byte moves
    assert lib.gf_gio_read(ctx.handle, ref.encode(), dt, C.c_void_p(back.data_ptr()), nd - 1,
                           None) == A.GF_ERR_ARG


@pytest.mark.gpu
def test_device_streaming_across_chunks(ctx, tmp_path):
    """A 72 MiB field crosses three 32 MiB staging chunks each way."""
    lib = A.load()
    dim, p = 3, 7
    ne = (9 * 2**20) // 512 + 1  # > 9 Mi values of 8 bytes
    h, porder = _hdr(0, dim, ne, p)
    nd = GO.ndata(0, dim, ne, porder)
    u = torch.arange(nd, dtype=torch.float64, device="cuda") * 0.5 - 3.0
    path = str(tmp_path / "big.out")
    ctx.check(lib.gf_gio_write(ctx.handle, path.encode(), C.byref(h),
                               porder.ctypes.data_as(C.c_void_p), None, A.GF_F64,
                               C.c_void_p(u.data_ptr()), nd))
    hdr, data = GO.read(path)
    assert np.array_equal(data, u.cpu().numpy())
    back = torch.zeros_like(u)
    ctx.check(lib.gf_gio_read(ctx.handle, path.encode(), A.GF_F64, C.c_void_p(back.data_ptr()),
                              nd, None))
    assert torch.equal(back, u)


@pytest.mark.gpu
@pytest.mark.parametrize("io_type,multivar", [(G.GIO_POSIX, False), (G.GIO_COLL, False),
                                              (G.GIO_COLL, True)])
def test_gio_state_round_trip_on_problem(ctx, tmp_path, io_type, multivar):
    from geoflow_b200 import GridBox, Problem
    g = GridBox(3, [3, 2, 2], 5)
    prob = Problem(ctx, g)
    io = G.GIO(prob, G.GIOTraits(io_type=io_type, multivar=multivar))
    rng = np.random.default_rng(2)
    u = [torch.from_numpy(rng.standard_normal(g.ndof())).cuda() for _ in range(3)]
    info = G.StateInfo(sttype=0, index=40, cycle=40, time=0.04, svars=["u1", "u2", "u3"],
                       odir=str(tmp_path), idir=str(tmp_path))
    io.write_state("vel", info, u)
    names = os.listdir(tmp_path)
    if multivar:
        assert names == ["vel.000040.out"]
    elif io_type == G.GIO_POSIX:
        assert sorted(names) == [f"u{k}.000040.00000.out" for k in (1, 2, 3)]
    back = prob.zeros(ncomp=3)
    info2 = G.StateInfo(sttype=0, index=40, svars=["u1", "u2", "u3"], idir=str(tmp_path),
                        icomptype=[G.GSC_KINETIC, G.GSC_PRESCRIBED, G.GSC_KINETIC])
    io.read_state("vel", info2, back)
    assert torch.equal(back[0], u[0]) and torch.equal(back[2], u[2])
    if not multivar:  # the prescribed component is not read
        assert bool((back[1] == 0).all())
    assert info2.cycle == 40 and info2.time == 0.04 and info2.nelems == g.nelems
    # a grid-type mismatch is refused (gio.ipp:403-405 asserts it)
    other = G.GIO(prob, G.GIOTraits(io_type=io_type, multivar=multivar), gtype=G.GE_DEFORMED)
    with pytest.raises(ValueError):
        other.read_state("vel", G.StateInfo(sttype=0, index=40, svars=["u1", "u2", "u3"],
                                            idir=str(tmp_path)), back)
