"""Gather-scatter classes built on the device (gf_box_classes_device,
gf_classes_from_coords_device) against the host builders and the oracle's
GGFX-style coordinate matching: node_class, class_ptr and members bit for
bit, including periodic boxes, shuffled node order and coordinates jittered
within the tolerance.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O
from geoflow_b200 import _abi as A

pytestmark = pytest.mark.gpu


def host_box(dim, ne, p, per):
    lib = A.load()
    n = int(np.prod(ne)) * (p + 1) ** dim
    nc, cp, mem = (np.zeros(n, np.int32), np.zeros(n + 1, np.int32), np.zeros(n, np.int32))
    k = lib.gf_box_classes(dim, (C.c_int * 3)(*(list(ne) + [1] * (3 - dim))), p,
                           (C.c_int * 3)(*(list(per) + [0] * (3 - dim))), A.ptr(nc), A.ptr(cp),
                           A.ptr(mem))
    assert k > 0
    return k, nc, cp[: k + 1], mem


def device_out(n):
    return (torch.zeros(n, dtype=torch.int32, device="cuda"),
            torch.zeros(n + 1, dtype=torch.int32, device="cuda"),
            torch.zeros(n, dtype=torch.int32, device="cuda"))


BOXES = [(3, [2, 3, 2], 3, [0, 0, 0]), (3, [4, 2, 3], 5, [1, 0, 1]), (3, [1, 2, 1], 4, [1, 1, 0]),
         (3, [8, 8, 8], 7, [0, 0, 0]), (2, [5, 3], 6, [0, 1]), (2, [1, 4], 2, [1, 1]),
         (3, [2, 2, 2], 1, [1, 1, 1])]


@pytest.mark.parametrize("dim,ne,p,per", BOXES)
def test_box_classes_device_matches_host(ctx, dim, ne, p, per):
    k, nc, cp, mem = host_box(dim, ne, p, per)
    n = nc.size
    dnc, dcp, dmem = device_out(n)
    kd = A.load().gf_box_classes_device(
        ctx.handle, dim, (C.c_int * 3)(*(list(ne) + [1] * (3 - dim))), p,
        (C.c_int * 3)(*(list(per) + [0] * (3 - dim))), C.c_void_p(dnc.data_ptr()),
        C.c_void_p(dcp.data_ptr()), C.c_void_p(dmem.data_ptr()))
    assert kd == k
    assert np.array_equal(dnc.cpu().numpy(), nc)
    assert np.array_equal(dcp.cpu().numpy()[: k + 1], cp)
    assert np.array_equal(dmem.cpu().numpy(), mem)


def periodized(o, per):
    pc = [a.copy() for a in o.xyz[: o.dim]]
    eps = 0.125 * o.minnodedist
    for d in range(o.dim):
        if per[d]:
            pc[d][np.abs(pc[d] - (o.x0[d] + o.length[d])) < eps] = o.x0[d]
    return pc


def coords_classes(ctx, dim, pts, tol):
    n = pts[0].size
    lib = A.load()
    nc, cp, mem = (np.zeros(n, np.int32), np.zeros(n + 1, np.int32), np.zeros(n, np.int32))
    arr = (A.P_double * 3)(*([A.ptr(a) for a in pts] + [A.ptr(pts[0])] * (3 - dim)))
    k = lib.gf_classes_from_coords(dim, n, arr, tol, A.ptr(nc), A.ptr(cp), A.ptr(mem))
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pts]
    darr = (C.c_void_p * 3)(*([a.data_ptr() for a in dev] + [dev[0].data_ptr()] * (3 - dim)))
    dnc, dcp, dmem = device_out(n)
    kd = lib.gf_classes_from_coords_device(ctx.handle, dim, n, darr, tol,
                                           C.c_void_p(dnc.data_ptr()), C.c_void_p(dcp.data_ptr()),
                                           C.c_void_p(dmem.data_ptr()))
    return (k, nc, cp[: k + 1], mem), (kd, dnc.cpu().numpy(), dcp.cpu().numpy()[: kd + 1],
                                       dmem.cpu().numpy())


@pytest.mark.parametrize("dim,ne,p,per", [(3, [2, 2, 2], 3, [1, 0, 1]), (3, [3, 2, 4], 6, [0, 0, 0]),
                                          (2, [4, 3], 5, [1, 0]), (3, [4, 4, 4], 7, [1, 1, 1])])
def test_classes_from_coords_device_matches_oracle_and_host(ctx, dim, ne, p, per):
    o = O.OracleBox(dim, ne, p, periodic=per)
    pts = periodized(o, per)
    tol = 0.25 * o.minnodedist
    (k, nc, cp, mem), (kd, dnc, dcp, dmem) = coords_classes(ctx, dim, pts, tol)
    assert k == o.nclass and kd == k
    assert np.array_equal(cp, o.class_ptr) and np.array_equal(mem, o.members)
    assert np.array_equal(dnc, nc) and np.array_equal(dcp, cp) and np.array_equal(dmem, mem)


def test_classes_from_coords_device_shuffled_and_jittered(ctx):
    """A node order unrelated to the geometry and coordinates moved by up
    to 0.2 tol: the device and host builders still agree bit for bit."""
    o = O.OracleBox(3, [3, 3, 2], 5, periodic=[0, 1, 0])
    pts = periodized(o, [0, 1, 0])
    tol = 0.25 * o.minnodedist
    rng = np.random.default_rng(4)
    perm = rng.permutation(pts[0].size)
    pts = [a[perm] + 0.2 * tol * (2 * rng.random(a.size) - 1) for a in pts]
    (k, nc, cp, mem), (kd, dnc, dcp, dmem) = coords_classes(ctx, 3, pts, tol)
    assert kd == k == o.nclass
    assert np.array_equal(dnc, nc) and np.array_equal(dcp, cp) and np.array_equal(dmem, mem)


def test_device_classes_reject_bad_arguments(ctx):
    lib = A.load()
    dnc, dcp, dmem = device_out(8)
    assert lib.gf_box_classes_device(ctx.handle, 4, (C.c_int * 3)(2, 2, 2), 1, None,
                                     C.c_void_p(dnc.data_ptr()), C.c_void_p(dcp.data_ptr()),
                                     C.c_void_p(dmem.data_ptr())) == A.GF_ERR_ARG
    arr = (C.c_void_p * 3)(dnc.data_ptr(), dnc.data_ptr(), dnc.data_ptr())
    assert lib.gf_classes_from_coords_device(ctx.handle, 3, 8, arr, -1.0,
                                             C.c_void_p(dnc.data_ptr()),
                                             C.c_void_p(dcp.data_ptr()),
                                             C.c_void_p(dmem.data_ptr())) == A.GF_ERR_ARG
