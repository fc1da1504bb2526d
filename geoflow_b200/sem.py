"""Host-side mirror of the GeoFLOW interfaces on the hot path, over libgfgpu.

The classes keep the reference's names, argument meaning and error
behaviour so that code written against the reference reads the same:

  GridBox      grid/ggrid_box.ipp   (host set-up: elements, coordinates,
                                     regular geometry, Dirichlet mask)
  GGFX         comm/ggfx.hpp        (doOp with Sum/Smooth/Max/Min,
                                     get_mult/get_imult)
  GHelmholtz   sem/ghelmholtz.ipp   (set_Lap_scalar, set_mass_scalar,
                                     opVec_prod)
  GMass        sem/gmass.ipp        (opVec_prod; inverse = 1/Smooth(M))
  GCG          solvers/gcg.ipp      (solve(A, b, x) / solve(A, b, xb, x),
                                     GCGERR codes, iteration count,
                                     residual history)
  GExRKStepper pdes/gexrk_stepper.ipp and GBurgers pdes/gburgers.ipp

Fields are torch CUDA tensors in element-local (E-vector) layout; torch is
used only for device memory.  Every compute call goes through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A


def _lib():
    return A.load()


def gll_basis(p: int):
    """GLL nodes, weights and column-major D (GLLBasis, sem/gllbasis.ipp)."""
    n = p + 1
    xi, w, D = np.zeros(n), np.zeros(n), np.zeros(n * n)
    rc = _lib().gf_gll_basis(p, A.ptr(xi), A.ptr(w), A.ptr(D))
    if rc:
        raise A.GFError(rc, f"gf_gll_basis({p})")
    return xi, w, D


class Context:
    """A CUDA device + stream owning libgfgpu state (one per host thread)."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        self.device = device
        self.torch_device = torch.device("cuda", device)
        h = C.c_void_p()
        if stream is None:  # order the work with torch's current stream
            stream = torch.cuda.current_stream(device).cuda_stream
        s = C.c_void_p(stream) if stream else None
        rc = _lib().gf_ctx_create(device, s, C.byref(h))
        if rc:
            raise A.GFError(rc, "gf_ctx_create failed (no CUDA device?)")
        self.handle = h

    def check(self, rc: int, what: str = "") -> int:
        if rc < 0:
            msg = _lib().gf_ctx_last_error(self.handle).decode()
            raise A.GFError(rc, f"{what}: {msg}")
        return rc

    def synchronize(self):
        self.check(_lib().gf_ctx_synchronize(self.handle), "synchronize")

    def close(self):
        if self.handle:
            _lib().gf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GridBox:
    """Regular 2-d/3-d box grid as GGridBox builds it on one rank.

    ne: elements per direction, p: polynomial order, x0/length: box origin
    and extent, periodic: per-direction flags (else Dirichlet faces).
    """

    def __init__(self, dim, ne, p, x0=None, length=None, periodic=None):
        self.dim, self.p, self.n = int(dim), int(p), int(p) + 1
        self.ne = [int(v) for v in ne][:dim]
        self.x0 = np.array(x0 if x0 is not None else [0.0] * dim, dtype=np.float64)[:dim]
        self.length = np.array(length if length is not None else [1.0] * dim, dtype=np.float64)[:dim]
        self.periodic = [int(bool(v)) for v in (periodic if periodic is not None else [0] * dim)][:dim]
        self.nelems = int(np.prod(self.ne))
        self.nn = self.n ** self.dim
        N = self.nelems * self.nn
        self.xi, self.W, self.D = gll_basis(self.p)
        lib = _lib()
        ne_c = (C.c_int * 3)(*(self.ne + [1] * (3 - dim)))
        per_c = (C.c_int * 3)(*(self.periodic + [0] * (3 - dim)))
        self.xyz = [np.zeros(N) for _ in range(dim)]
        xyz_c = (A.P_double * 3)(*[A.ptr(a) for a in self.xyz])
        self.elem_geom = np.zeros(self.nelems * (dim + 1))
        self.mask = np.zeros(N)
        rc = lib.gf_box_grid(dim, ne_c, self.p, A.ptr(self.x0), A.ptr(self.length), per_c, xyz_c,
                             A.ptr(self.elem_geom), A.ptr(self.mask))
        if rc:
            raise A.GFError(rc, "gf_box_grid")
        self.node_class = np.zeros(N, dtype=np.int32)
        self.class_ptr = np.zeros(N + 1, dtype=np.int32)
        self.members = np.zeros(N, dtype=np.int32)
        nc = lib.gf_box_classes(dim, ne_c, self.p, per_c, A.ptr(self.node_class),
                                A.ptr(self.class_ptr), A.ptr(self.members))
        if nc < 0:
            raise A.GFError(nc, "gf_box_classes")
        self.nclass = int(nc)
        self.class_ptr = self.class_ptr[: nc + 1].copy()

    def ndof(self) -> int:
        return self.nelems * self.nn

    def xNodes(self):
        return self.xyz

    def mult(self):
        cnt = np.diff(self.class_ptr)
        return cnt[self.node_class].astype(np.float64)


class IcosGrid:
    """The 2-d icosahedral sphere of GGridIcos (GE_2DEMBEDDED): gf_icos_grid
    builds the node coordinates and the embedded metric, and the gather-
    scatter classes come from coordinate matching (gf_classes_from_coords,
    tolerance tol_frac times the smallest node spacing, as GGFX::init).
    refine: GF_ICOS_BISECTION or GF_ICOS_LAGRANGIAN."""

    def __init__(self, level, p, radius=1.0, refine=A.GF_ICOS_BISECTION, tol_frac=0.001,
                 ctx=None):
        """ctx: match the classes on that context's GPU
        (gf_classes_from_coords_device, the same classes bit for bit)."""
        lib = _lib()
        self.dim, self.p, self.n, self.level, self.radius = 2, int(p), int(p) + 1, level, radius
        ne, nl = C.c_int64(), C.c_int64()
        rc = lib.gf_icos_sizes(level, p, refine, C.byref(ne), C.byref(nl))
        if rc:
            raise A.GFError(rc, "gf_icos_sizes")
        self.nelems, N = int(ne.value), int(nl.value)
        self.ne = [self.nelems]
        self.nn = self.n * self.n
        self.xi, self.W, self.D = gll_basis(self.p)
        self.xyz = [np.zeros(N) for _ in range(3)]
        self.node_geom = np.zeros(7 * N)
        xyz_c = (A.P_double * 3)(*[A.ptr(a) for a in self.xyz])
        rc = lib.gf_icos_grid(level, p, float(radius), refine, xyz_c, A.ptr(self.node_geom))
        if rc:
            raise A.GFError(rc, "gf_icos_grid")
        self.mask = np.ones(N)
        self.elem_geom = np.zeros(self.nelems * 3)
        self.periodic = [0, 0]
        # smallest distance between neighbouring nodes of an element
        X = np.stack(self.xyz).reshape(3, self.nelems, self.n, self.n)
        dx = np.sqrt(((X[:, :, :, 1:] - X[:, :, :, :-1]) ** 2).sum(0)).min()
        dy = np.sqrt(((X[:, :, 1:, :] - X[:, :, :-1, :]) ** 2).sum(0)).min()
        self.minnodedist = float(min(dx, dy))
        self.node_class = np.zeros(N, dtype=np.int32)
        self.class_ptr = np.zeros(N + 1, dtype=np.int32)
        self.members = np.zeros(N, dtype=np.int32)
        if ctx is None:
            nc = lib.gf_classes_from_coords(3, N, xyz_c, tol_frac * self.minnodedist,
                                            A.ptr(self.node_class), A.ptr(self.class_ptr),
                                            A.ptr(self.members))
        else:
            import torch
            dev = ctx.torch_device
            xd = [torch.from_numpy(a).to(dev) for a in self.xyz]
            outs = [torch.zeros(N, dtype=torch.int32, device=dev),
                    torch.zeros(N + 1, dtype=torch.int32, device=dev),
                    torch.zeros(N, dtype=torch.int32, device=dev)]
            nc = lib.gf_classes_from_coords_device(ctx.handle, 3, N, A.ptr_array(xd),
                                                   tol_frac * self.minnodedist,
                                                   *[A.ptr(t) for t in outs])
            if nc >= 0:
                self.node_class, self.class_ptr, self.members = (t.cpu().numpy() for t in outs)
        if nc < 0:
            raise A.GFError(nc, "gf_classes_from_coords")
        self.nclass = int(nc)
        self.class_ptr = self.class_ptr[: nc + 1].copy()

    def ndof(self) -> int:
        return self.nelems * self.nn

    def xNodes(self):
        return self.xyz

    def mult(self):
        return np.diff(self.class_ptr)[self.node_class].astype(np.float64)

    def problem(self, ctx):
        """The device problem (GF_GEOM_EMBEDDED, no Dirichlet mask)."""
        return Problem(ctx, self, dirichlet_mask=False, structured=False, geometry="embedded",
                       node_geom=self.node_geom, node_xyz=np.concatenate(self.xyz))


class Problem:
    """Device-resident grid, operators and gather-scatter map (gf_problem)."""

    def __init__(self, ctx: Context, grid: GridBox, dirichlet_mask: bool = True,
                 structured: bool = True, geometry: str = "affine", node_geom=None,
                 node_xyz=None):
        """geometry: "affine" passes one (dXi/dX, Jac) set per element;
        "regular" passes the same factors per node (the GGrid per-node
        planes dXidX, Jac); "deformed" (GE_DEFORMED) and "embedded"
        (GE_2DEMBEDDED, a 2-d surface in 3-d space) take the caller's
        node_geom = [dXi_i/dX_k planes (i < dim, k < nxy), Jac] as one array
        of (dim*nxy + 1) * ndof values, nxy = dim or 3.  node_xyz (3 * ndof,
        optional) are the node coordinates used by constrain2sphere."""
        self.ctx, self.grid, self.geometry = ctx, grid, geometry
        self.structured = structured
        self.dim, self.n, self.nlocal = grid.dim, grid.n, grid.ndof()
        # velocity components: one per physical coordinate
        self.nvel = 3 if geometry == "embedded" else grid.dim
        d = A.ProblemDesc()
        d.dim, d.ne, d.n = grid.dim, grid.nelems, grid.n
        self._keep = [grid.D, grid.W, grid.elem_geom, grid.mask, grid.class_ptr, grid.members]
        d.D, d.W = A.ptr(grid.D), A.ptr(grid.W)
        if geometry == "affine":
            d.geom = A.GF_GEOM_AFFINE
            d.elem_geom = A.ptr(grid.elem_geom)
            d.node_geom = None
        elif geometry == "regular":
            npe = grid.n ** grid.dim
            eg = grid.elem_geom.reshape(grid.nelems, grid.dim + 1)
            ng = np.ascontiguousarray(np.concatenate(
                [np.repeat(eg[:, k], npe) for k in range(grid.dim + 1)]))
            self._keep.append(ng)
            d.geom = A.GF_GEOM_REGULAR
            d.elem_geom = None
            d.node_geom = A.ptr(ng)
        elif geometry in ("deformed", "embedded"):
            nxy = 3 if geometry == "embedded" else grid.dim
            ng = np.ascontiguousarray(node_geom, dtype=np.float64).ravel()
            if ng.size != (grid.dim * nxy + 1) * grid.ndof():
                raise ValueError("node_geom must hold (dim*nxy + 1) * ndof values")
            self._keep.append(ng)
            d.geom = A.GF_GEOM_EMBEDDED if geometry == "embedded" else A.GF_GEOM_DEFORMED
            d.elem_geom = None
            d.node_geom = A.ptr(ng)
        else:
            raise ValueError(f"unknown geometry {geometry!r}")
        d.mask = A.ptr(grid.mask) if dirichlet_mask else None
        d.nclass = grid.nclass
        d.class_ptr, d.members = A.ptr(grid.class_ptr), A.ptr(grid.members)
        if structured:  # unique nodes indexed by lattice point (no index arrays)
            for k in range(grid.dim):
                d.box_ne[k] = grid.ne[k]
                d.box_periodic[k] = grid.periodic[k]
        if node_xyz is not None:
            xyz = np.ascontiguousarray(node_xyz, dtype=np.float64).ravel()
            self._keep.append(xyz)
            d.node_xyz = A.ptr(xyz)
        h = C.c_void_p()
        ctx.check(_lib().gf_problem_create(ctx.handle, C.byref(d), C.byref(h)), "gf_problem_create")
        self.handle = h

    def zeros(self, dtype=None, ncomp=None):
        import torch
        dt = dtype or torch.float64
        if ncomp is None:
            return torch.zeros(self.nlocal, dtype=dt, device=self.ctx.torch_device)
        return [torch.zeros(self.nlocal, dtype=dt, device=self.ctx.torch_device) for _ in range(ncomp)]

    def close(self):
        if getattr(self, "handle", None):
            _lib().gf_problem_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dtype_code(t) -> int:
    import torch
    if t.dtype == torch.float64:
        return A.GF_F64
    if t.dtype == torch.float32:
        return A.GF_F32
    raise TypeError(f"unsupported dtype {t.dtype}")


def _check_field(prob: Problem, t):
    if not t.is_cuda or t.numel() != prob.nlocal or not t.is_contiguous():
        raise ValueError("fields must be contiguous CUDA tensors of N_local elements")


class GGFX:
    """Gather-scatter (GGFX::doOp) over the problem's equivalence classes."""
    Sum, Smooth, Max, Min = A.GF_DSS_SUM, A.GF_DSS_SMOOTH, A.GF_DSS_MAX, A.GF_DSS_MIN

    def __init__(self, prob: Problem):
        self.prob = prob

    def doOp(self, u, op) -> bool:
        _check_field(self.prob, u)
        self.prob.ctx.check(_lib().gf_dss(self.prob.handle, _dtype_code(u), int(op), A.ptr(u)),
                            "GGFX::doOp")
        return True

    def get_mult(self):
        m = self.prob.zeros()
        self.prob.ctx.check(_lib().gf_mult(self.prob.handle, 0, A.ptr(m)), "get_mult")
        return m

    def get_imult(self):
        m = self.prob.zeros()
        self.prob.ctx.check(_lib().gf_mult(self.prob.handle, 1, A.ptr(m)), "get_imult")
        return m


def tensor_apply(prob: Problem, A1, A2, A3, u, out):
    """out = (A3 x A2 x A1) u in every element (GMTK::D3_X_D2_X_D1 /
    D2_X_D1 with the matrices as given, n x n column-major numpy arrays;
    A3 unused in 2-d).  A spectral filter is A_d = the filter matrix."""
    mats = [np.ascontiguousarray(a, dtype=np.float64).ravel(order="F") if a is not None else None
            for a in (A1, A2, A3)]
    prob.ctx.check(_lib().gf_tensor_apply(prob.handle, _dtype_code(u), A.ptr(mats[0]),
                                          A.ptr(mats[1]), A.ptr(mats[2]), A.ptr(u), A.ptr(out)),
                   "tensor_apply")


def filter_matrix(kind: int, p: int, pdelta: int, strength: float) -> np.ndarray:
    """The (p+1) x (p+1) 1-d filter matrix of GBoydFilter::init
    (kind GF_FILTER_BOYD) or GProjectionFilter::init (GF_FILTER_PROJECTION)."""
    F = np.zeros((p + 1) * (p + 1))
    rc = _lib().gf_filter_matrix(kind, p, pdelta, strength, A.ptr(F))
    if rc < 0:
        raise A.GFError(rc, "gf_filter_matrix")
    return F.reshape(p + 1, p + 1, order="F")


class _Filter:
    """FilterBase over the library's in-place tensor filter: traits istate
    (state ids to filter; empty = all), pdelta and strength per direction."""
    KIND = A.GF_FILTER_BOYD

    def __init__(self, prob: Problem, pdelta, strength, istate=None):
        dim = prob.dim
        pd = [int(pdelta)] * dim if np.isscalar(pdelta) else [int(v) for v in pdelta][:dim]
        st = [float(strength)] * dim if np.isscalar(strength) else [float(v) for v in strength][:dim]
        if not all(0.0 <= v <= 1.0 for v in st):
            raise ValueError("filter strength must lie in [0, 1]")
        self.prob, self.istate = prob, list(istate or [])
        self.F = [filter_matrix(self.KIND, prob.n - 1, pd[d], st[d]) for d in range(dim)]
        self._flat = [np.ascontiguousarray(f.ravel(order="F")) for f in self.F]

    def apply(self, u, utmp=None, uo=None):
        """In place on the state list u (the selected components), or with
        uo given, out of place (u unchanged)."""
        ids = self.istate or list(range(len(u)))
        if uo is not None:
            for j in ids:
                uo[j].copy_(u[j])
            target = uo
        else:
            target = u
        comps = [target[j] for j in ids]
        f3 = self._flat[2] if self.prob.dim == 3 else None
        self.prob.ctx.check(_lib().gf_filter_apply(
            self.prob.handle, _dtype_code(comps[0]), A.ptr(self._flat[0]), A.ptr(self._flat[1]),
            A.ptr(f3), len(comps), A.ptr_array(comps)), "Filter::apply")


class GBoydFilter(_Filter):
    """GBoydFilter (sem/gboyd_filter.ipp): u <- (F x F x F) u, F = L Lambda L^-1."""
    KIND = A.GF_FILTER_BOYD


class GProjectionFilter(_Filter):
    """GProjectionFilter (sem/gprojection_filter.ipp): F = a Ihi Ilow + (1-a) I."""
    KIND = A.GF_FILTER_PROJECTION


class GMass:
    """Lumped mass W x W (x W) x Jac; inverse=True uses 1/Smooth(M)."""

    def __init__(self, prob: Problem, inverse: bool = False):
        self.prob, self.inverse = prob, inverse

    def opVec_prod(self, u, utmp, uo):
        _check_field(self.prob, u)
        self.prob.ctx.check(_lib().gf_mass_apply(self.prob.handle, _dtype_code(u), int(self.inverse),
                                                 A.ptr(u), A.ptr(uo)), "GMass::opVec_prod")


class GHelmholtz:
    """H = q M + p L (weak Laplacian L); p defaults to 1, no mass term until
    set_mass_scalar is called (ghelmholtz.ipp:30-45, 591-625)."""

    def __init__(self, prob: Problem):
        self.prob = prob
        self.p, self.q, self.bcompute_helm = 1.0, None, False

    def set_Lap_scalar(self, p):
        self.p = p

    def set_mass_scalar(self, q):
        self.q = q
        self.bcompute_helm = True

    def opVec_prod(self, u, utmp, uo):
        _check_field(self.prob, u)
        dt = _dtype_code(u)
        p_s, p_v = (float(self.p), None) if np.isscalar(self.p) else (1.0, self.p)
        q = self.q if self.q is not None else 0.0
        q_s, q_v = (float(q), None) if np.isscalar(q) else (1.0, q)
        self.prob.ctx.check(_lib().gf_helmholtz_apply(
            self.prob.handle, dt, p_s, A.ptr(p_v), q_s, A.ptr(q_v), int(self.bcompute_helm),
            A.ptr(u), A.ptr(uo)), "GHelmholtz::opVec_prod")


@dataclass
class CGTraits:
    """LinSolverBase::Traits (lin_solver_base.hpp:38-44) plus the B200 options."""
    maxit: int = 512
    normtype: int = A.GF_NORM_INF
    tol: float = 1e-6
    precond: int = A.GF_PRECOND_NONE
    precision: int = A.GF_CG_FP64
    inner_tol: float = 0.0
    max_refine: int = 40
    check_every: int = 16
    relative: int = 0
    mixed_apply: int = 0
    poly_degree: int = 2
    poly_ratio: float = 0.0

    def to_c(self) -> A.CGTraits:
        t = A.CGTraits()
        for f in ("maxit", "normtype", "tol", "precond", "precision", "inner_tol", "max_refine",
                  "check_every", "relative", "mixed_apply", "poly_degree", "poly_ratio"):
            setattr(t, f, getattr(self, f))
        return t


class GCG:
    """Conjugate gradient (GCG::solve_impl): returns GCGERR codes."""
    GCGERR_NONE, GCGERR_NOCONVERGE, GCGERR_SOLVE, GCGERR_PRECOND, GCGERR_BADITERNUM = 0, 1, 2, 3, 4

    def __init__(self, traits: CGTraits, prob: Problem):
        self.traits, self.prob = traits, prob
        self.iter_, self.rnorm_ = 0, 0.0
        self.residuals_ = np.zeros(max(1, traits.maxit))

    def solve(self, A_op: GHelmholtz, b, *args) -> int:
        if len(args) == 1:
            xb, x = None, args[0]
        elif len(args) == 2:
            xb, x = args
        else:
            raise TypeError("solve(A, b, x) or solve(A, b, xb, x)")
        for t in (b, x) + ((xb,) if xb is not None else ()):
            _check_field(self.prob, t)
        if not np.isscalar(A_op.p) or (A_op.q is not None and not np.isscalar(A_op.q)):
            raise ValueError("the device CG takes scalar p and q")
        it, rn = C.c_int(0), C.c_double(0.0)
        tr = self.traits.to_c()
        q = float(A_op.q) if A_op.q is not None else 0.0
        rc = _lib().gf_cg_solve(self.prob.handle, C.byref(tr), float(A_op.p), q,
                                int(A_op.bcompute_helm), A.ptr(b), A.ptr(xb), A.ptr(x),
                                C.byref(it), C.byref(rn), A.ptr(self.residuals_))
        self.prob.ctx.check(rc, "GCG::solve")
        self.iter_, self.rnorm_ = it.value, rn.value
        return rc

    def get_iteration_count(self) -> int:
        """As the reference's GCG::get_iteration_count (solvers/gcg.hpp:75):
        the number of iterations taken plus one.  `iter_` holds the number
        of iterations."""
        return self.iter_ + 1

    def get_residuals(self):
        return self.residuals_[: self.iter_]


class GBurgers:
    """Burgers / advection-diffusion / heat on GExRKStepper (gburgers.ipp)."""
    ADVECT, BURGERS, HEAT = A.GF_EQN_ADVECT, A.GF_EQN_BURGERS, A.GF_EQN_HEAT

    def __init__(self, prob: Problem, eqn: int, nu: float, scheme: int = A.GF_RK4):
        self.prob, self.eqn, self.nu, self.scheme = prob, eqn, float(nu), scheme
        self.nstate = prob.nvel if eqn == A.GF_EQN_BURGERS else 1

    def traits(self) -> A.RKTraits:
        t = A.RKTraits()
        t.eqn, t.nu, t.nstate, t.scheme = self.eqn, self.nu, self.nstate, self.scheme
        return t

    def dudt(self, u, c, dudt):
        lib = _lib()
        self.prob.ctx.check(lib.gf_dudt(self.prob.handle, _dtype_code(u[0]), self.eqn, self.nu,
                                        len(u), A.ptr_array(u), A.ptr_array(c or []),
                                        A.ptr_array(dudt)), "GBurgers::dudt")

    def step(self, u, c=None, dt=1e-4, nsteps=1, t0=0.0, filters=None):
        """nsteps steps in place; with `filters` (a filter list, as
        EquationBase::set_filter_list) each filter is applied in place after
        every step, as GMConv::step_impl does (gmconv.ipp:648-653)."""
        tr = self.traits()
        if not filters:
            self.prob.ctx.check(_lib().gf_rk_advance(self.prob.handle, _dtype_code(u[0]),
                                                     C.byref(tr), A.ptr_array(u),
                                                     A.ptr_array(c or []), t0, dt, nsteps),
                                "GBurgers::step")
            return
        for k in range(nsteps):
            self.prob.ctx.check(_lib().gf_rk_advance(self.prob.handle, _dtype_code(u[0]),
                                                     C.byref(tr), A.ptr_array(u),
                                                     A.ptr_array(c or []), t0 + k * dt, dt, 1),
                                "GBurgers::step")
            for f in filters:
                if f is not None:
                    f.apply(u)

    def capture(self, u, c=None, dt=1e-4, nsteps=1):
        """Record `nsteps` steps advancing u in place as a CUDA graph
        (Graph.launch replays them; same result as step())."""
        tr = self.traits()
        h = C.c_void_p()
        self.prob.ctx.check(_lib().gf_rk_graph_create(
            self.prob.handle, _dtype_code(u[0]), C.byref(tr), A.ptr_array(u),
            A.ptr_array(c or []), dt, nsteps, C.byref(h)), "GBurgers::capture")
        return Graph(self.prob.ctx, h, [u, c, self.prob])

    # ---- adjoint (no reference counterpart; FP64 only) ----
    def dudt_vjp(self, u, c, lam, ubar):
        """ubar = (d dudt/du)^T lam at state u (velocity c for advection)."""
        self.prob.ctx.check(_lib().gf_dudt_vjp(self.prob.handle, _dtype_code(lam[0]), self.eqn,
                                               self.nu, len(lam), A.ptr_array(u or []),
                                               A.ptr_array(c or []), A.ptr_array(lam),
                                               A.ptr_array(ubar)), "GBurgers::dudt_vjp")

    def step_vjp(self, u0, c, dt, lam):
        """lam <- (d step/d u0)^T lam for one step from u0 (in place)."""
        tr = self.traits()
        self.prob.ctx.check(_lib().gf_rk_step_vjp(self.prob.handle, _dtype_code(lam[0]),
                                                  C.byref(tr), A.ptr_array(u0),
                                                  A.ptr_array(c or []), dt, A.ptr_array(lam)),
                            "GBurgers::step_vjp")

    def adjoint_gradient(self, u0, c, u_obs, dt, nsteps, checkpoint_every=10):
        """(J, grad): J = 1/2 sum_k ||u_k(T) - obs_k||_M^2 after nsteps steps
        from u0, and dJ/du0, with a checkpoint every `checkpoint_every`
        steps and recomputation."""
        import torch
        tr = self.traits()
        grad = [torch.empty_like(a) for a in u0]
        J = C.c_double(0.0)
        self.prob.ctx.check(_lib().gf_adjoint_gradient(
            self.prob.handle, C.byref(tr), A.ptr_array(u0), A.ptr_array(c or []),
            A.ptr_array(u_obs), dt, nsteps, checkpoint_every, C.byref(J), A.ptr_array(grad)),
            "GBurgers::adjoint_gradient")
        return J.value, grad


class Graph:
    """A CUDA graph of RK steps (GBurgers.capture) or an ensemble of such
    graphs (Graph.ensemble): launch() replays the recorded work in one call.
    Keeps the tensors it was recorded with alive."""

    def __init__(self, ctx: Context, handle, keep):
        self.ctx, self.handle, self._keep = ctx, handle, keep

    @staticmethod
    def ensemble(graphs):
        arr = (C.c_void_p * len(graphs))(*[g.handle.value for g in graphs])
        h = C.c_void_p()
        ctx = graphs[0].ctx
        ctx.check(_lib().gf_graph_ensemble(len(graphs), arr, C.byref(h)), "gf_graph_ensemble")
        return Graph(ctx, h, list(graphs))

    def launch(self):
        self.ctx.check(_lib().gf_graph_launch(self.handle), "gf_graph_launch")

    def nodes(self) -> int:
        return _lib().gf_graph_nodes(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            _lib().gf_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

