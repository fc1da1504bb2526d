"""Ensembles of independent problems advanced together (gf_ensemble_*).

The reference runs one problem per process; an ensemble runs many small
ones at once on one GPU: one persistent cooperative launch per RK stage of
every member (deformed / embedded 2-d members, e.g. icosahedral-sphere
advection) or per CG iteration of every member (2-d box Helmholtz solves:
FP64 iterations, or FP32 iterations with FP64 residual refinement),
captured in CUDA graphs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from .sem import CGTraits, Context, Problem, _lib


class Ensemble:
    """gf_ensemble over `problems` (all deformed/embedded, or all box)."""

    def __init__(self, ctx: Context, problems):
        self.ctx = ctx
        self.problems = list(problems)
        hs = (C.c_void_p * len(self.problems))(*[p.handle.value for p in self.problems])
        h = C.c_void_p()
        ctx.check(_lib().gf_ensemble_create(ctx.handle, len(self.problems),
                                            C.cast(hs, A.P_void), C.byref(h)),
                  "gf_ensemble_create")
        self.handle = h
        self.kind = _lib().gf_ensemble_kind(h)

    @staticmethod
    def _code(t) -> int:
        import torch
        return A.GF_F64 if t.dtype == torch.float64 else A.GF_F32

    # ---- RK ----
    def advance(self, u, c=None, dt=1e-3, nsteps=1, eqn=A.GF_EQN_ADVECT, nu=0.0,
                scheme=A.GF_RK4):
        """Advances every member's state u[m] in place by nsteps step_b steps
        of dt[m] (a scalar applies to all); c[m] = the member's velocity
        components (advection)."""
        n = len(self.problems)
        if len(u) != n:
            raise ValueError(f"{n} states expected")
        dts = np.full(n, float(dt)) if np.isscalar(dt) else np.asarray(dt, dtype=np.float64)
        tr = A.RKTraits()
        tr.eqn, tr.nu, tr.nstate, tr.scheme = eqn, float(nu), 1, scheme
        cp = None
        if c is not None:
            flat = []
            for m in range(n):
                cm = list(c[m]) + [None] * (3 - len(c[m]))
                flat += cm[:3]
            cp = A.ptr_array(flat)
        rc = _lib().gf_ensemble_rk_advance(self.handle, self._code(u[0]), C.byref(tr),
                                           A.ptr_array(u), cp, A.ptr(dts), int(nsteps))
        return self.ctx.check(rc, "gf_ensemble_rk_advance")

    # ---- CG ----
    def solve(self, b, x, traits: CGTraits, p=1.0, q=1.0):
        """Solves (p L + q M) x[m] = b[m] (device FP64 E-vectors, x the
        initial guess); returns (rc, iterations, final FP64 residual norms,
        statuses) per member."""
        n = len(self.problems)
        it = np.zeros(n, dtype=np.intc)
        nrm = np.zeros(n)
        st = np.zeros(n, dtype=np.intc)
        tr = traits.to_c()
        rc = _lib().gf_ensemble_cg_solve(self.handle, C.byref(tr), float(p), float(q),
                                         A.ptr_array(b), A.ptr_array(x), A.ptr(it), A.ptr(nrm),
                                         A.ptr(st))
        self.ctx.check(rc, "gf_ensemble_cg_solve")
        return rc, it, nrm, st

    # ---- launch shapes ----
    def tune(self, dtype=None, reps=5):
        import torch
        code = A.GF_F32 if dtype in (None, torch.float32) else A.GF_F64
        return self.ctx.check(_lib().gf_ensemble_tune(self.handle, code, int(reps)),
                              "gf_ensemble_tune")

    def shape(self, dtype=None):
        import torch
        code = A.GF_F32 if dtype in (None, torch.float32) else A.GF_F64
        th, bl, tu, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        team = np.zeros(11, dtype=np.intc)
        self.ctx.check(_lib().gf_ensemble_shape(self.handle, code, C.byref(th), C.byref(bl),
                                                A.ptr(team), C.byref(tu), C.byref(ms)),
                       "gf_ensemble_shape")
        ns = sorted({p.n for p in self.problems})
        return {"threads": th.value, "blocks": bl.value, "tuned": bool(tu.value),
                "tuned_ms_per_launch": ms.value if tu.value else None,
                "team_by_n": {n: int(team[n]) for n in ns}}

    def set_shape(self, threads, blocks_per_sm=0, team_by_n=None, dtype=None):
        import torch
        code = A.GF_F32 if dtype in (None, torch.float32) else A.GF_F64
        tp = None
        if team_by_n is not None:
            team = np.zeros(11, dtype=np.intc)
            cur = self.shape(dtype)["team_by_n"]
            for n in range(3, 11):
                team[n] = team_by_n.get(n, cur.get(n, 16))
            tp = A.ptr(team)
        return self.ctx.check(_lib().gf_ensemble_set_shape(self.handle, code, int(threads),
                                                           int(blocks_per_sm), tp),
                              "gf_ensemble_set_shape")

    def launches(self) -> int:
        return int(_lib().gf_ensemble_launches(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            _lib().gf_ensemble_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def box_problem(ctx, ne, p, length=(1.0, 1.0)):
    """A 2-d Dirichlet box member (GridBox + Problem, affine elements)."""
    from .sem import GridBox
    g = GridBox(2, [ne, ne] if np.isscalar(ne) else list(ne), p, length=list(length))
    return g, Problem(ctx, g)
