"""ctypes wrapper over the C oracle (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product library never imports it.  `OracleBox` builds a
GGridBox-equivalent grid with the oracle's own coordinate construction and
GGFX-style coordinate matching (after the periodize step of
grid/ggrid_box.ipp:753-806), independently of the product's lattice maps.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libgforacle.so"
# GFO_OPENMP=1 selects the OpenMP build of the same sources (every host
# core; dot products sum in thread order): the bench's CPU baseline only.
if os.environ.get("GFO_OPENMP") == "1":
    LIB = HERE / "_build" / "libgforacle_omp.so"
REFLIB = HERE / "_ref" / "libgfref.so"

P_double = C.POINTER(C.c_double)
P_int32 = C.POINTER(C.c_int32)
c_size_t = C.c_size_t

SUM, SMOOTH, MAX, MIN = 0, 1, 2, 3
NORM_INF, NORM_EUC, NORM_L2, NORM_L1 = 0, 1, 2, 3


class GfoGrid(C.Structure):
    _fields_ = [("dim", C.c_int), ("Ne", c_size_t), ("n", C.c_int * 3), ("D", P_double * 3),
                ("W", P_double * 3), ("dXidX", P_double * 3), ("Jac", P_double),
                ("mass", P_double)]


class GfoDefGrid(C.Structure):
    _fields_ = [("base", C.POINTER(GfoGrid)), ("nxy", C.c_int), ("X", (P_double * 3) * 3)]


class GfoBurgers(C.Structure):
    _fields_ = [("g", C.POINTER(GfoGrid)), ("kind", C.c_int), ("nu", C.c_double),
                ("imass", P_double), ("c", C.POINTER(P_double)), ("nclass", c_size_t),
                ("class_ptr", P_int32), ("members", P_int32)]


class GfoCGTraits(C.Structure):
    _fields_ = [("maxit", C.c_int), ("normtype", C.c_int), ("tol", C.c_double)]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            import subprocess
            subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
        _lib = C.CDLL(str(LIB))
        _lib.gfo_ggfx_init.restype = C.c_long
        _lib.gfo_integrate.restype = C.c_double
        _lib.gfo_cg_solve.restype = C.c_int
    return _lib


def load_ref():
    """The reference's own GLLBasis/GMTK compiled from its sources, or None."""
    if REFLIB.exists():
        lib = C.CDLL(str(REFLIB))
        return lib
    return None


def dp(a):
    return None if a is None else a.ctypes.data_as(P_double)


def ip(a):
    return a.ctypes.data_as(P_int32)


def gll(p):
    n = p + 1
    xi, w, D = np.zeros(n), np.zeros(n), np.zeros(n * n)
    load().gfo_gll(p, dp(xi), dp(w), dp(D))
    return xi, w, D


class OracleBox:
    """Box grid + GGFX classes + geometry, built by the oracle."""

    def __init__(self, dim, ne, p, x0=None, length=None, periodic=None, tol_frac=0.25):
        lib = load()
        self.dim, self.p, self.n = dim, p, p + 1
        self.ne = list(ne)[:dim]
        self.x0 = np.array(x0 if x0 is not None else [0.0] * dim, dtype=np.float64)
        self.length = np.array(length if length is not None else [1.0] * dim, dtype=np.float64)
        self.periodic = list(periodic if periodic is not None else [0] * dim)[:dim]
        self.nelems = int(np.prod(self.ne))
        self.nn = self.n ** dim
        N = self.N = self.nelems * self.nn
        ne3 = (C.c_int * 3)(*(self.ne + [1] * (3 - dim)))
        p3 = (C.c_int * 3)(*([p] * 3))
        per3 = (C.c_int * 3)(*(self.periodic + [0] * (3 - dim)))
        self.xyz = [np.zeros(N) for _ in range(3)]
        self.dXidX = [np.zeros(N) for _ in range(3)]
        self.Jac = np.zeros(N)
        self.mask = np.zeros(N)
        lib.gfo_box_build(dim, ne3, p3, dp(self.x0), dp(self.length), per3, dp(self.xyz[0]),
                          dp(self.xyz[1]), dp(self.xyz[2]), dp(self.dXidX[0]), dp(self.dXidX[1]),
                          dp(self.dXidX[2]), dp(self.Jac), dp(self.mask))
        self.xi, self.W, self.D = gll(p)
        # periodize (ggrid_box.ipp:753-806): nodes on the upper face of a
        # periodic direction take the lower coordinate
        h = self.length / np.array(self.ne, dtype=np.float64)
        minnodedist = float(np.min((self.xi[1] - self.xi[0]) * 0.5 * h))
        self.minnodedist = minnodedist
        eps = 0.125 * minnodedist
        pc = [a.copy() for a in self.xyz]
        for d in range(dim):
            if self.periodic[d]:
                top = self.x0[d] + self.length[d]
                pc[d][np.abs(pc[d] - top) < eps] = self.x0[d]
        self.node_class = np.zeros(N, dtype=np.int32)
        self.class_ptr = np.zeros(N + 1, dtype=np.int32)
        self.members = np.zeros(N, dtype=np.int32)
        nc = lib.gfo_ggfx_init(c_size_t(N), dim, dp(pc[0]), dp(pc[1]), dp(pc[2]),
                               C.c_double(tol_frac * minnodedist), ip(self.node_class),
                               ip(self.class_ptr), ip(self.members))
        assert nc > 0
        self.nclass = int(nc)
        self.class_ptr = self.class_ptr[: nc + 1].copy()
        self.mass = np.zeros(N)
        self._grid = self._make_grid()
        lib.gfo_mass(C.byref(self._grid), dp(self.mass))
        self._grid.mass = dp(self.mass)
        sm = self.mass.copy()
        self.dss(sm, SMOOTH)
        self.imass = 1.0 / sm

    def _make_grid(self):
        g = GfoGrid()
        g.dim, g.Ne = self.dim, self.nelems
        for d in range(3):
            g.n[d] = self.n
            g.D[d] = dp(self.D)
            g.W[d] = dp(self.W)
            g.dXidX[d] = dp(self.dXidX[d])
        g.Jac = dp(self.Jac)
        g.mass = dp(self.mass)
        return g

    # ---- operators ----
    def dss(self, u, op):
        f = load().gfo_ggfx_doop if u.dtype == np.float64 else load().gfo_ggfx_doop_f
        ptr = dp(u) if u.dtype == np.float64 else u.ctypes.data_as(C.POINTER(C.c_float))
        f(ptr, c_size_t(self.nclass), ip(self.class_ptr), ip(self.members), op)
        return u

    def mult(self):
        m = np.zeros(self.N)
        load().gfo_ggfx_mult(c_size_t(self.N), c_size_t(self.nclass), ip(self.class_ptr),
                             ip(self.members), dp(m))
        return m

    def helmholtz(self, u, p=1.0, p_vec=None, q_vec=None):
        uo = np.zeros(self.N)
        load().gfo_helmholtz(C.byref(self._grid), dp(u), C.c_double(p), dp(p_vec), dp(q_vec),
                             dp(uo))
        return uo

    def grefderiv(self, u, idir, dotrans=0):
        du = np.zeros(self.N)
        load().gfo_grefderiv(C.byref(self._grid), dp(u), idir, dotrans, dp(du))
        return du

    def grefdiv(self, us, dotrans=1):
        arr = (P_double * 3)(*[dp(a) for a in us] + [None] * (3 - len(us)))
        out = np.zeros(self.N)
        load().gfo_grefdiv(C.byref(self._grid), arr, dotrans, dp(out))
        return out

    def deriv(self, u, idir):
        du = np.zeros(self.N)
        load().gfo_deriv(C.byref(self._grid), dp(u), idir, dp(du))
        return du

    def advect(self, p, c):
        arr = (P_double * 3)(*[dp(a) for a in c] + [None] * (3 - len(c)))
        po = np.zeros(self.N)
        load().gfo_advect(C.byref(self._grid), dp(p), len(c), arr, dp(po))
        return po

    def dudt(self, kind, nu, u, c=None):
        nst = len(u)
        ua = (P_double * 3)(*[dp(a) for a in u] + [None] * (3 - nst))
        ca = (P_double * 3)(*([dp(a) for a in c] if c else []) + [None] * (3 - (len(c) if c else 0)))
        out = [np.zeros(self.N) for _ in range(nst)]
        oa = (P_double * 3)(*[dp(a) for a in out] + [None] * (3 - nst))
        load().gfo_dudt(C.byref(self._grid), kind, C.c_double(nu), dp(self.imass), nst, ua, ca, oa)
        return out

    def integrate(self, u):
        return load().gfo_integrate(C.byref(self._grid), dp(u))

    def rk_advance(self, kind, nu, scheme, u, c=None, dt=1e-4, nsteps=1):
        b = GfoBurgers()
        b.g = C.pointer(self._grid)
        b.kind, b.nu, b.imass = kind, nu, dp(self.imass)
        self._c = (P_double * 3)(*([dp(a) for a in c] if c else []) + [None] * (3 - (len(c) if c else 0)))
        b.c = self._c
        b.nclass, b.class_ptr, b.members = self.nclass, ip(self.class_ptr), ip(self.members)
        ua = (P_double * 3)(*[dp(a) for a in u] + [None] * (3 - len(u)))
        load().gfo_rk_advance(C.byref(b), scheme, len(u), ua, C.c_double(0.0), C.c_double(dt),
                              nsteps)
        return u

    def helmholtz_diag(self, p, q_vec=None):
        d = np.zeros(self.N)
        load().gfo_helmholtz_diag(C.byref(self._grid), C.c_double(p), dp(q_vec),
                                  c_size_t(self.nclass), ip(self.class_ptr), ip(self.members),
                                  dp(d))
        return d

    def cg_solve(self, b, x, p=1.0, q_vec=None, xb=None, maxit=512, normtype=NORM_INF, tol=1e-6,
                 dinv=None, use_mask=True):
        tr = GfoCGTraits()
        tr.maxit, tr.normtype, tr.tol = maxit, normtype, tol
        it = C.c_int(0)
        res = np.zeros(max(1, maxit))
        rc = load().gfo_cg_solve(C.byref(self._grid), C.c_double(p), dp(q_vec),
                                 dp(self.mask if use_mask else None), c_size_t(self.nclass),
                                 ip(self.class_ptr), ip(self.members), dp(dinv), C.byref(tr),
                                 dp(b), dp(xb), dp(x), C.byref(it), dp(res))
        return rc, it.value, res[: it.value]


class OracleDef:
    """Deformed (GE_DEFORMED) or 2-d embedded (GE_2DEMBEDDED) geometry on the
    elements, GLL basis and GGFX classes of an OracleBox: X[i][k] =
    dXi_i/dX_k per node (i < dim, k < nxy) and Jac, as the caller's grid
    would supply them."""

    def __init__(self, box, X, Jac, nxy):
        lib = load()
        self.box, self.dim, self.nxy, self.N = box, box.dim, nxy, box.N
        self.X = [[np.ascontiguousarray(X[i][k], dtype=np.float64) for k in range(nxy)]
                  for i in range(self.dim)]
        self.Jac = np.ascontiguousarray(Jac, dtype=np.float64)
        g = GfoGrid()
        g.dim, g.Ne = box.dim, box.nelems
        for d in range(3):
            g.n[d] = box.n
            g.D[d] = dp(box.D)
            g.W[d] = dp(box.W)
            g.dXidX[d] = dp(box.dXidX[d])
        g.Jac = dp(self.Jac)
        self.mass = np.zeros(self.N)
        lib.gfo_mass(C.byref(g), dp(self.mass))
        g.mass = dp(self.mass)
        self._g = g
        dg = GfoDefGrid()
        dg.base = C.pointer(self._g)
        dg.nxy = nxy
        for i in range(self.dim):
            for k in range(nxy):
                dg.X[i][k] = dp(self.X[i][k])
        self._dg = dg
        self.G = [[np.zeros(self.N) for _ in range(3)] for _ in range(3)]
        self._Garr = self._mat(self.G)
        lib.gfo_def_metric(C.byref(dg), self._Garr)
        sm = self.mass.copy()
        box.dss(sm, SMOOTH)
        self.imass = 1.0 / sm

    @staticmethod
    def _mat(G):
        arr = ((P_double * 3) * 3)()
        for i in range(3):
            for j in range(3):
                arr[i][j] = dp(G[i][j])
        return arr

    def node_geom(self):
        """[dXi_i/dX_k planes (i, k), Jac] as one array (gf_problem_desc)."""
        planes = [self.X[i][k] for i in range(self.dim) for k in range(self.nxy)]
        return np.concatenate(planes + [self.Jac])

    def helmholtz(self, u, p=1.0, p_vec=None, q_vec=None):
        uo = np.zeros(self.N)
        load().gfo_def_helmholtz(C.byref(self._dg), self._Garr, dp(u), C.c_double(p), dp(p_vec),
                                 dp(q_vec), dp(uo))
        return uo

    def deriv(self, u, idir):
        du = np.zeros(self.N)
        load().gfo_def_deriv(C.byref(self._dg), dp(u), idir, dp(du))
        return du

    def advect(self, p, c):
        arr = (P_double * 3)(*[dp(a) for a in c] + [None] * (3 - len(c)))
        po = np.zeros(self.N)
        load().gfo_def_advect(C.byref(self._dg), dp(p), arr, dp(po))
        return po

    def dudt(self, kind, nu, u, c=None):
        nst = len(u)
        ua = (P_double * 3)(*[dp(a) for a in u] + [None] * (3 - nst))
        nc = len(c) if c else 0
        ca = (P_double * 3)(*([dp(a) for a in c] if c else []) + [None] * (3 - nc))
        out = [np.zeros(self.N) for _ in range(nst)]
        oa = (P_double * 3)(*[dp(a) for a in out] + [None] * (3 - nst))
        load().gfo_def_dudt(C.byref(self._dg), self._Garr, kind, C.c_double(nu), dp(self.imass),
                            nst, ua, ca, oa)
        return out


def constrain2sphere(xyz, v):
    """GMTK::constrain2sphere (2) in place on v[0..2] (numpy FP64)."""
    xa = (P_double * 3)(*[dp(a) for a in xyz])
    va = (P_double * 3)(*[dp(a) for a in v])
    load().gfo_constrain2sphere(c_size_t(len(v[0])), xa, va)
    return v


# ---- the reference's own path code (oracle/_ref/libgfref{2,3}.so) ----
REFPATH = {2: HERE / "_ref" / "libgfref2.so", 3: HERE / "_ref" / "libgfref3.so"}
_refpath = {}
P_void = C.c_void_p


def load_refpath(dim):
    """The reference's GGridBox/GGFX/GHelmholtz/GAdvect/GCG/GBurgers compiled
    from its sources for GDIM = dim (oracle/ref/ref_path.cpp), or None."""
    if dim not in _refpath:
        if not REFPATH[dim].exists():
            return None
        lib = C.CDLL(str(REFPATH[dim]))
        lib.gfr_box_create.restype = P_void
        lib.gfr_box_create.argtypes = [C.POINTER(C.c_int), C.c_int, P_double, P_double, C.c_int,
                                       C.c_double]
        lib.gfr_ndof.restype = c_size_t
        lib.gfr_ndof.argtypes = [P_void]
        lib.gfr_path_error.restype = C.c_char_p
        for f in ("gfr_coords", "gfr_mass", "gfr_mask", "gfr_imult"):
            getattr(lib, f).argtypes = [P_void, P_double]
        lib.gfr_dss.argtypes = [P_void, P_double, C.c_int]
        lib.gfr_helmholtz.argtypes = [P_void, P_double, P_double, P_double, c_size_t, P_double]
        lib.gfr_advect.argtypes = [P_void, P_double, P_double, P_double]
        lib.gfr_cg_solve.argtypes = [P_void, C.c_double, P_double, P_double, P_double, P_double,
                                     C.c_int, C.c_double, C.c_int, P_double,
                                     C.POINTER(C.c_int), P_double]
        lib.gfr_burgers_run.argtypes = [P_void, C.c_int, C.c_double, C.c_int, C.c_int,
                                        C.c_double, C.c_int, P_double]
        lib.gfr_box_destroy.argtypes = [P_void]
        lib.gfr_nxyz.argtypes = [P_void]
        lib.gfr_metric.argtypes = [P_void, P_double, P_double]
        if dim == 2:
            lib.gfr_icos_create.restype = P_void
            lib.gfr_icos_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double]
        assert lib.gfr_path_dim() == dim
        _refpath[dim] = lib
    return _refpath[dim]


class RefBox:
    """A box grid run by the reference's own code (see load_refpath); the
    same layout as OracleBox (element-major, x fastest).  RefBox.icos(...)
    builds the reference's 2-d icosahedral sphere instead."""

    @classmethod
    def icos(cls, level, p, radius=1.0, refine=0, tol_frac=0.001):
        """GGridIcos (GE_2DEMBEDDED) of the 2-d build: refine 0
        GICOS_BISECTION, 1 GICOS_LAGRANGIAN."""
        self = cls.__new__(cls)
        self.lib = lib = load_refpath(2)
        if lib is None:
            raise FileNotFoundError(f"{REFPATH[2]} not built")
        self.dim, self.p = 2, p
        self.h = lib.gfr_icos_create(level, p, radius, refine, tol_frac)
        if not self.h:
            raise RuntimeError(lib.gfr_path_error().decode())
        self.N = int(lib.gfr_ndof(self.h))
        return self

    def nxyz(self):
        return int(self.lib.gfr_nxyz(self.h))

    def metric(self):
        """(dXi_i/dX_k planes, i < dim, k < nxyz; Jacobian)."""
        nx = self.nxyz()
        m = np.zeros(self.dim * nx * self.N)
        j = np.zeros(self.N)
        self.lib.gfr_metric(self.h, dp(m), dp(j))
        return m.reshape(self.dim * nx, self.N), j

    def __init__(self, dim, ne, p, periodic=None, x0=None, length=None, tol_frac=0.001):
        self.lib = lib = load_refpath(dim)
        if lib is None:
            raise FileNotFoundError(f"{REFPATH[dim]} not built")
        self.dim, self.p = dim, p
        per = list(periodic if periodic is not None else [0] * dim)
        mask = sum(1 << d for d in range(dim) if per[d])
        ne3 = (C.c_int * 3)(*(list(ne)[:dim] + [1] * (3 - dim)))
        x0 = np.array(list(x0 if x0 is not None else [0.0] * dim) + [0.0] * (3 - dim))
        ln = np.array(list(length if length is not None else [1.0] * dim) + [1.0] * (3 - dim))
        self.h = lib.gfr_box_create(ne3, p, dp(x0), dp(ln), mask, tol_frac)
        if not self.h:
            raise RuntimeError(lib.gfr_path_error().decode())
        self.N = int(lib.gfr_ndof(self.h))

    def close(self):
        if self.h:
            self.lib.gfr_box_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _vec(self, fn, nvec=1):
        a = np.zeros(self.N * nvec)
        getattr(self.lib, fn)(self.h, dp(a))
        return a

    def coords(self):
        nx = self.nxyz()
        return self._vec("gfr_coords", nx).reshape(nx, self.N)

    def mass(self):
        return self._vec("gfr_mass")

    def mask(self):
        return self._vec("gfr_mask")

    def imult(self):
        return self._vec("gfr_imult")

    def dss(self, u, op):
        rc = self.lib.gfr_dss(self.h, dp(u), op)
        assert rc == 0
        return u

    def helmholtz(self, u, p=1.0, p_vec=None, q_vec=None):
        pv = np.ascontiguousarray(p_vec if p_vec is not None else np.array([p], dtype=np.float64))
        out = np.zeros(self.N)
        self.lib.gfr_helmholtz(self.h, dp(u), dp(out), dp(pv), c_size_t(len(pv)), dp(q_vec))
        return out

    def advect(self, u, c):
        cc = np.ascontiguousarray(np.concatenate(c))
        out = np.zeros(self.N)
        self.lib.gfr_advect(self.h, dp(u), dp(cc), dp(out))
        return out

    def cg_solve(self, b, x, p=1.0, q_vec=None, xb=None, maxit=512, normtype=NORM_INF,
                 tol=1e-6, dinv=None):
        """GCG::solve(A, b, xb, x); returns (rc, iterations, residuals).  The
        reference's get_iteration_count() is iterations + 1 (gcg.hpp:75)."""
        q = q_vec if q_vec is not None else np.ones(self.N)
        xbv = xb if xb is not None else np.zeros(self.N)
        it = C.c_int(0)
        res = np.zeros(max(1, maxit))
        rc = self.lib.gfr_cg_solve(self.h, p, dp(q), dp(b), dp(xbv), dp(x), maxit, tol,
                                   normtype, dp(dinv), C.byref(it), dp(res))
        iters = it.value - 1
        return rc, iters, res[:iters]

    def burgers_run(self, kind, nu, order, ssp, state, dt, nsteps):
        """GBurgers stepped by its GExRKStepper; state: list of component
        arrays (kind 0: [u, c_1..c_dim]; 1: dim velocities; 2: [u]); the
        evolved components are updated in place."""
        st = np.ascontiguousarray(np.concatenate(state))
        rc = self.lib.gfr_burgers_run(self.h, kind, nu, order, 1 if ssp else 0, dt, nsteps,
                                      dp(st))
        if rc != 0:
            raise RuntimeError(self.lib.gfr_path_error().decode())
        for k, a in enumerate(state):
            a[:] = st[k * self.N:(k + 1) * self.N]
        return state
