"""Generates tests/golden/ref_path.npz from the reference's own path code.

Runs in the build container only: it needs oracle/_ref/libgfref{2,3}.so,
which `make -C oracle ref REF=<reference checkout>` compiles from the
reference's GGridBox, GGFX, GHelmholtz, GAdvect, GCG, GBurgers and
GExRKStepper sources (oracle/ref/ref_path.cpp).  Every array in the fixture
is an input handed to the reference or an output it produced:

  grid_{tag}_{mass,mask,imult}       GGrid massop, Dirichlet mask, GGFX imult
  grid_{tag}_u, grid_{tag}_dss{op}   GGFX::doOp(u, Sum/Smooth/Max/Min)
  grid_{tag}_{q,pv,helm_s,helm_v}    GHelmholtz(p = 0.7 or p = pv, q) u
  grid_{tag}_{c,adv}                 GAdvect::apply(u, c)
  cg_{tag}_...                       GCG::solve(H, b, xb, x): x, residuals,
                                     iterations, GCGERR code
  rk_{tag}_...                       GBurgers stepped by GExRKStepper
  cgt_{tag}_...                      the same, Jacobi, to 1e-13
  cfg1_{u0,u200}                     the 2-d periodic advection case at its
                                     full length (16^2 elements, p = 4,
                                     c = (1, 0.5), nu = 0.01, RK4,
                                     dt = 1e-4, 200 steps)
  icos_{tag}_{xyz,metric,jac,mass}   GGridIcos (GE_2DEMBEDDED) nodes, dXi/dX
                                     (2 x 3 planes), Jacobian, mass
  icos_{tag}_{u,dss*,q,helm,c,adv}   GGFX, GHelmholtz (embed_prod), GAdvect on it
  icosadv_{u0,u,c,dt}                the cosine bell in the solid-body wind
                                     advected by GBurgers (RK4, nu = 1e-3) on
                                     the level-1 p = 3 sphere
  cfg3s_{u0,u100,dt}                 the 3-d Burgers case (its initial
                                     velocity, nu = 1e-3, SSP-RK3, CFL 0.3,
                                     100 steps) on a 3^3-element p = 5
                                     periodic box

The grids' node order is the reference's (element-major, x fastest); the
oracle's OracleBox builds the same order, which the test checks through
the mass and mask arrays.

Usage: python tests/golden/make_path_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))
import oracle as O  # noqa: E402
from geoflow_b200 import workloads as W  # noqa: E402

SEED = 20261203

# Mixed periodicity is left out: the reference's GGridBox::periodize
# (grid/ggrid_box.ipp:753-806) moves every coordinate at the upper bound of
# a periodic-face node, in non-periodic directions too, so it merges the
# corners of a partly periodic box; and its 2-d faces are named
# bdy_x_0/x_1/y_0/y_1 but found as south/east/north/west
# (ggrid_box.ipp:1043-1048, 1540-1560).
GRIDS = [  # tag, dim, ne, p, periodic
    ("2d_dir", 2, [4, 3], 4, [0, 0]),
    ("2d_per", 2, [4, 3], 4, [1, 1]),
    ("3d_dir", 3, [2, 3, 2], 3, [0, 0, 0]),
    ("3d_per", 3, [2, 2, 3], 4, [1, 1, 1]),
]

CGS = [  # tag, dim, ne, p, precond, norm, maxit
    ("2d_none_inf", 2, [4, 4], 5, False, O.NORM_INF, 400),
    ("2d_jac_euc", 2, [4, 4], 5, True, O.NORM_EUC, 400),
    ("3d_none_euc", 3, [3, 2, 2], 4, False, O.NORM_EUC, 400),
    ("3d_jac_inf", 3, [3, 2, 2], 4, True, O.NORM_INF, 400),
    ("3d_jac_maxit", 3, [3, 2, 2], 4, True, O.NORM_INF, 5),
]
# Solves run to 1e-13, so a solver with other rounding (the GPU's) can be
# compared with the reference's solution at 1e-10.
CG_TIGHT = [  # tag, dim, ne, p
    ("2d", 2, [5, 4], 5),
    ("3d", 3, [3, 3, 2], 4),
]

RK = [  # tag, dim, ne, p, order, ssp, kind, nsteps, dt
    *[(f"2d_o{o}{'s' if s else ''}_k{k}", 2, [4, 4], 4, o, s, k, 5, 1e-3)
      for (o, s) in [(1, 0), (2, 0), (3, 0), (4, 0), (2, 1), (3, 1)] for k in (0, 1, 2)],
    ("3d_o3s_k1", 3, [2, 2, 2], 4, 3, 1, 1, 3, 1e-3),
    ("3d_o4_k1", 3, [2, 2, 2], 4, 4, 0, 1, 3, 1e-3),
    ("3d_o2_k2", 3, [2, 2, 2], 3, 2, 0, 2, 3, 1e-3),
    ("3d_o4_k0", 3, [2, 2, 2], 3, 4, 0, 0, 3, 1e-3),
]


def continuous(o, rng):
    """A seeded field with one value per GGFX class (continuous)."""
    return rng.standard_normal(o.nclass)[o.node_class]


def config1_initial():
    o = O.OracleBox(2, [16, 16], 4, periodic=[1, 1])
    return o, W.advection2d_initial(o.xyz, o.node_class, o.nclass)


def main():
    if O.load_refpath(2) is None or O.load_refpath(3) is None:
        raise SystemExit("oracle/_ref/libgfref{2,3}.so missing: run "
                         "`make -C oracle ref REF=<reference checkout>` first")
    out = {}
    rng = np.random.default_rng(SEED)
    for tag, dim, ne, p, per in GRIDS:
        r = O.RefBox(dim, ne, p, periodic=per)
        o = O.OracleBox(dim, ne, p, periodic=per)
        k = f"grid_{tag}_"
        out[k + "mass"], out[k + "mask"], out[k + "imult"] = r.mass(), r.mask(), r.imult()
        u = rng.standard_normal(r.N)
        out[k + "u"] = u
        for op in range(4):
            out[k + f"dss{op}"] = r.dss(u.copy(), op)
        q = 0.5 + rng.random(r.N)
        pv = 0.5 + rng.random(r.N)
        out[k + "q"], out[k + "pv"] = q, pv
        out[k + "helm_s"] = r.helmholtz(u, p=0.7, q_vec=q)
        out[k + "helm_v"] = r.helmholtz(u, p_vec=pv, q_vec=q)
        c = [continuous(o, rng) for _ in range(dim)]
        out[k + "c"] = np.stack(c)
        out[k + "adv"] = r.advect(u, c)
    for tag, dim, ne, p, pc, norm, maxit in CGS:
        r = O.RefBox(dim, ne, p, periodic=[0] * dim)
        o = O.OracleBox(dim, ne, p, periodic=[0] * dim)
        k = f"cg_{tag}_"
        q = np.ones(r.N)
        b = o.mass * continuous(o, rng)
        dinv = 1.0 / o.helmholtz_diag(1.0, q) if pc else None
        x = np.zeros(r.N)
        rc, it, res = r.cg_solve(b, x, p=1.0, q_vec=q, maxit=maxit, normtype=norm, tol=1e-10,
                                 dinv=dinv)
        out[k + "b"], out[k + "x"], out[k + "res"] = b, x, res
        out[k + "info"] = np.array([rc, it, maxit, norm, int(pc)], dtype=np.int64)
        if pc:
            out[k + "dinv"] = dinv
    for tag, dim, ne, p, order, ssp, kind, nsteps, dt in RK:
        r = O.RefBox(dim, ne, p, periodic=[1] * dim)
        o = O.OracleBox(dim, ne, p, periodic=[1] * dim)
        k = f"rk_{tag}_"
        nsolve = dim if kind == 1 else 1
        u0 = [continuous(o, rng) for _ in range(nsolve)]
        c = [np.full(r.N, 1.0 - 0.5 * d) for d in range(dim)] if kind == 0 else []
        st = [a.copy() for a in u0] + [a.copy() for a in c]
        r.burgers_run(kind, 0.01, order, ssp, st, dt, nsteps)
        out[k + "u0"] = np.stack(u0)
        out[k + "u"] = np.stack(st[:nsolve])
        out[k + "info"] = np.array([dim, p, order, ssp, kind, nsteps], dtype=np.int64)
        out[k + "dt"] = np.array([dt])
        out[k + "ne"] = np.array(ne, dtype=np.int64)
    for tag, dim, ne, p in CG_TIGHT:
        r = O.RefBox(dim, ne, p, periodic=[0] * dim)
        o = O.OracleBox(dim, ne, p, periodic=[0] * dim)
        k = f"cgt_{tag}_"
        q = np.ones(r.N)
        b = o.mass * continuous(o, rng)
        dinv = 1.0 / o.helmholtz_diag(1.0, q)
        x = np.zeros(r.N)
        rc, it, res = r.cg_solve(b, x, p=1.0, q_vec=q, maxit=2000, normtype=O.NORM_INF,
                                 tol=1e-13, dinv=dinv)
        assert rc == 0
        out[k + "b"], out[k + "x"] = b, x
        out[k + "info"] = np.array([rc, it], dtype=np.int64)
    # the icosahedral sphere (GE_2DEMBEDDED)
    for tag, level, p, refine in (("l0p4", 0, 4, 0), ("l1p2lag", 1, 2, 1)):
        r = O.RefBox.icos(level, p, 1.0, refine)
        k = f"icos_{tag}_"
        out[k + "xyz"] = r.coords()
        m, j = r.metric()
        out[k + "metric"], out[k + "jac"], out[k + "mass"] = m, j, r.mass()
        u = rng.standard_normal(r.N)
        out[k + "u"] = u
        for op in range(4):
            out[k + f"dss{op}"] = r.dss(u.copy(), op)
        q = 0.5 + rng.random(r.N)
        out[k + "q"] = q
        out[k + "helm"] = r.helmholtz(u, p=0.7, q_vec=q)
        c = W.icos_solid_body_wind(list(r.coords()), u0=1.0, alpha=0.3)
        out[k + "c"] = np.stack(c)
        out[k + "adv"] = r.advect(u, c)
    r = O.RefBox.icos(1, 3, 1.0, 0)
    xyz = list(r.coords())
    u0 = W.icos_cosine_bell(xyz, 0.3, 4.0)
    c = W.icos_solid_body_wind(xyz, u0=1.0, alpha=0.3)
    st = [u0.copy()] + [a.copy() for a in c]
    r.burgers_run(0, 1e-3, 4, False, st, 2e-3, 20)
    out["icosadv_u0"], out["icosadv_u"], out["icosadv_c"] = u0, st[0], np.stack(c)
    out["icosadv_dt"] = np.array([2e-3])
    # 3-d Burgers, SSP-RK3, 100 steps, on 3^3 elements at p = 5
    ne3, p3 = 3, 5
    r = O.RefBox(3, [ne3] * 3, p3, periodic=[1] * 3, length=[2 * np.pi] * 3)
    o = O.OracleBox(3, [ne3] * 3, p3, periodic=[1] * 3, length=[2 * np.pi] * 3)
    u0 = W.burgers_velocity([o.xyz[0], o.xyz[1], o.xyz[2]], W.burgers_modes())
    dt3 = W.burgers_dt(max(float(np.abs(a).max()) for a in u0), ne3, p3, o.xi)
    st = [a.copy() for a in u0]
    r.burgers_run(1, 1e-3, 3, True, st, dt3, 100)
    out["cfg3s_u0"], out["cfg3s_u100"], out["cfg3s_dt"] = np.stack(u0), np.stack(st), np.array([dt3])
    o, u0 = config1_initial()
    r = O.RefBox(2, [16, 16], 4, periodic=[1, 1])
    st = [u0.copy(), np.full(r.N, 1.0), np.full(r.N, 0.5)]
    r.burgers_run(0, 0.01, 4, False, st, 1e-4, 200)
    out["cfg1_u0"], out["cfg1_u200"] = u0, st[0]
    dst = Path(__file__).resolve().parent / "ref_path.npz"
    np.savez_compressed(dst, **out)
    print(dst, len(out), dst.stat().st_size)


if __name__ == "__main__":
    main()
