"""gf_integrate_noalloc: the integral for callers that cannot allocate.

Callers such as a host framework that owns all device memory through its
own pool, or a time-stepping loop that must not stall on cudaMalloc/cudaFree,
get an integral entry point that allocates nothing: its scratch is a fixed
array inside the library.  This file runs last (pytest collects it last) so
that a stop at its first failure has already run every other test.  Each
test creates its own context and passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from geoflow_b200 import Context, GMass, GridBox, Problem
from geoflow_b200 import _abi as A

pytestmark = pytest.mark.gpu


def test_noalloc_integral_matches_gf_integrate_twice():
    ctx = Context(0)
    g = GridBox(3, [4, 3, 5], 6)
    prob = Problem(ctx, g)
    lib = A.load()
    rng = np.random.default_rng(31)
    u = torch.from_numpy(rng.standard_normal(g.ndof())).cuda()
    mass = prob.zeros()
    GMass(prob).opVec_prod(torch.ones(g.ndof(), dtype=torch.float64, device="cuda"), None, mass)
    ref = C.c_double()
    ctx.check(lib.gf_integrate(prob.handle, A.GF_F64, A.ptr(u), C.byref(ref)))
    scale = float((mass * u.abs()).sum())
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or None)
    # two calls in a row: the second reuses the scratch the first left behind
    for _ in range(2):
        rc = lib.gf_integrate_noalloc(g.ndof(), A.ptr(mass), A.ptr(u), A.ptr(out), stream)
        assert rc == A.GF_OK
        torch.cuda.synchronize()
        assert abs(out.item() - ref.value) <= 1e-12 * max(1.0, scale)
        out.fill_(float("nan"))


def test_noalloc_integral_rejects_sizes_beyond_its_scratch():
    lib = A.load()
    small = torch.zeros(4, dtype=torch.float64, device="cuda")
    too_many = A.GF_NOALLOC_MAX_N + 1
    rc = lib.gf_integrate_noalloc(too_many, A.ptr(small), A.ptr(small), A.ptr(small), None)
    assert rc == A.GF_ERR_ARG


def test_noalloc_call_allocates_nothing_under_global_capture():
    """A cudaMalloc (or any other allocation) during a stream capture in
    global mode invalidates the capture; the entry point records cleanly,
    and the replayed graph gives the integral."""
    ctx = Context(0)
    g = GridBox(3, [3, 4, 2], 5)
    prob = Problem(ctx, g)
    lib = A.load()
    rng = np.random.default_rng(7)
    u = torch.from_numpy(rng.standard_normal(g.ndof())).cuda()
    mass = prob.zeros()
    GMass(prob).opVec_prod(torch.ones(g.ndof(), dtype=torch.float64, device="cuda"), None, mass)
    ref = C.c_double()
    ctx.check(lib.gf_integrate(prob.handle, A.GF_F64, A.ptr(u), C.byref(ref)))
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    # the first call on the device comes before any capture
    assert lib.gf_integrate_noalloc(g.ndof(), A.ptr(mass), A.ptr(u), A.ptr(out),
                                    C.c_void_p(side.cuda_stream)) == A.GF_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    out.fill_(float("nan"))
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side, capture_error_mode="global"):
        rc = lib.gf_integrate_noalloc(g.ndof(), A.ptr(mass), A.ptr(u), A.ptr(out),
                                      C.c_void_p(side.cuda_stream))
    assert rc == A.GF_OK
    graph.replay()
    torch.cuda.synchronize()
    scale = float((mass * u.abs()).sum())
    assert abs(out.item() - ref.value) <= 1e-12 * max(1.0, scale)
    assert torch.cuda.mem_get_info()[0] >= free0 - (2 << 20)  # the graph's own bookkeeping only

