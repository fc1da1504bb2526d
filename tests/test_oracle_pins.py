"""Pins the C oracle: against the reference's own GLLBasis/GMTK outputs
(golden fixture and, where present, oracle/_ref), and against the known
answers of the reference's own tests (test/actions/cdg/*.cpp,
src/apps/hackathon_driver.cpp)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("p", range(2, 17))
def test_gll_bit_exact_vs_reference(golden, p):
    xi, w, D = O.gll(p)
    assert np.array_equal(bits(xi), bits(golden[f"gll_p{p}_xi"]))
    assert np.array_equal(bits(w), bits(golden[f"gll_p{p}_w"]))
    assert np.array_equal(bits(D), bits(golden[f"gll_p{p}_D"]))


def test_gll_properties():
    # D(0,0) = -N(N+1)/4 (the hackathon probe value -5 at p=4), weights sum to 2
    for p in range(2, 13):
        xi, w, D = O.gll(p)
        n = p + 1
        assert D[0] == -p * (p + 1) / 4.0 and D[n * n - 1] == p * (p + 1) / 4.0
        assert abs(w.sum() - 2.0) < 1e-14
        Dm = D.reshape(n, n, order="F")
        assert np.max(np.abs(Dm @ xi ** p - p * xi ** (p - 1))) < 1e-12 * p ** 3


def _oracle_gmtk(which, g):
    N = [int(v) for v in g[f"gmtk_{which}_N"]]
    ne = int(g[f"gmtk_{which}_Ne"][0])
    u, A, B, Cm = (g[f"gmtk_{which}_{k}"] for k in "uABC")
    y = np.zeros_like(u)
    lib = O.load()
    dp, sz = O.dp, C.c_size_t
    if which == 0:
        lib.gfo_I2_X_D1(dp(A), dp(u), sz(N[0]), sz(N[1]), sz(ne), dp(y))
    elif which == 1:
        lib.gfo_D2_X_I1(dp(A), dp(u), sz(N[0]), sz(N[1]), sz(ne), dp(y))
    elif which == 2:
        lib.gfo_I3_X_I2_X_D1(dp(A), dp(u), sz(N[0]), sz(N[1]), sz(N[2]), sz(ne), dp(y))
    elif which == 3:
        lib.gfo_I3_X_D2_X_I1(dp(A), dp(u), sz(N[0]), sz(N[1]), sz(N[2]), sz(ne), dp(y))
    elif which == 4:
        lib.gfo_D3_X_I2_X_I1(dp(A), dp(u), sz(N[0]), sz(N[1]), sz(N[2]), sz(ne), dp(y))
    else:
        return None
    return y


@pytest.mark.parametrize("which", range(5))
def test_tensor_products_bit_exact_vs_reference(golden, which):
    y = _oracle_gmtk(which, golden)
    assert np.array_equal(bits(y), bits(golden[f"gmtk_{which}_y"]))


def test_full_tensor_products_vs_kronecker(golden):
    # D2_X_D1 / D3_X_D2_X_D1 reference outputs equal the explicit Kronecker
    # products (the structure of cdg_gmtk.cpp:75-282)
    for which in (5, 6):
        N = [int(v) for v in golden[f"gmtk_{which}_N"]]
        u, A, B, Cm, y = (golden[f"gmtk_{which}_{k}"] for k in "uABCy")
        A_ = A.reshape(N[0], N[0], order="F")
        BT = B.reshape(N[1], N[1], order="F")  # passed as D2^T
        big = np.kron(BT.T, A_)
        if which == 6:
            big = np.kron(Cm.reshape(N[2], N[2], order="F").T, big)
        assert np.allclose(big @ u, y, rtol=1e-13, atol=1e-12)


def test_cdg_gmtk_integer_kat_exact():
    # cdg_gmtk.cpp:75-282: integer-valued D(i,j) = 2i + N0 j, u = 2i + N0 j,
    # N = (np+1, np+2, np+3); results must equal the Kronecker product exactly
    np_ = 4
    N = [np_ + 1, np_ + 2, np_ + 3]
    D1 = np.array([[2 * i + N[0] * j for j in range(N[0])] for i in range(N[0])], dtype=float)
    D2 = np.array([[2 * i + N[0] * j for j in range(N[1])] for i in range(N[1])], dtype=float)
    u2 = np.array([2 * i + N[0] * j for j in range(N[1]) for i in range(N[0])], dtype=float)
    lib = O.load()
    y = np.zeros(N[0] * N[1])
    D1f = np.asfortranarray(D1).ravel(order="F")
    lib.gfo_I2_X_D1(O.dp(D1f), O.dp(u2), C.c_size_t(N[0]), C.c_size_t(N[1]), C.c_size_t(1), O.dp(y))
    big = np.kron(np.eye(N[1]), D1)
    assert np.array_equal(y, big @ u2)
    D2T = np.asfortranarray(D2.T).ravel(order="F")
    lib.gfo_D2_X_I1(O.dp(D2T), O.dp(u2), C.c_size_t(N[0]), C.c_size_t(N[1]), C.c_size_t(1), O.dp(y))
    big = np.kron(D2, np.eye(N[0]))
    assert np.array_equal(y, big @ u2)


def _poly_box(dim, ne, p, periodic=None):
    return O.OracleBox(dim, ne, p, periodic=periodic)


def test_ggfx_smooth_preserves_continuous_field_bit_exact():
    # cdg_ggfx.cpp:158-235: Smooth of a linear field leaves every value
    # bit-identical
    for dim, ne in ((2, [3, 4]), (3, [2, 3, 2])):
        g = _poly_box(dim, ne, 4)
        f = 1.0 + 2.0 * g.xyz[0] + 3.0 * g.xyz[1] + (0.5 * g.xyz[2] if dim == 3 else 0)
        # make duplicates bitwise identical (coordinates of shared nodes are
        # computed per element and may differ in the last bit)
        first = g.members[g.class_ptr[:-1]]
        f = f[first][g.node_class]
        h = f.copy()
        g.dss(h, O.SMOOTH)
        assert np.array_equal(bits(h), bits(f))


def test_ggfx_multiplicity_box():
    g = _poly_box(3, [2, 2, 2], 3)
    m = g.mult()
    assert m.max() == 8 and m.min() == 1
    gp = _poly_box(2, [3, 3], 3, periodic=[1, 1])
    assert gp.mult().max() == 4 and gp.nclass == (3 * 3) ** 2


def test_cdg_cg_poisson_known_answer():
    # cdg_cg.cpp:113-341 with data/cg_input.jsn: 2D box 4x4 elements, p=6,
    # -lap u = f, u = y(1-y)x^3, Dirichlet data, CG tol 1e-7, INF norm,
    # maxit 256; pass criterion: integral of (u-ua)^2 / volume < 1e-12
    g = _poly_box(2, [4, 4], 6)
    x, y = g.xyz[0], g.xyz[1]
    f = 6.0 * x * y * (1.0 - y) - 2.0 * x ** 3
    ua = y * (1.0 - y) * x ** 3
    eps = 100 * np.finfo(float).eps
    ub = np.zeros(g.N)
    ub[np.abs(x - 1.0) <= eps] = (y * (1.0 - y))[np.abs(x - 1.0) <= eps]
    b = -(f * g.mass)
    u = np.zeros(g.N)
    rc, it, res = g.cg_solve(b, u, p=1.0, xb=ub, maxit=256, normtype=O.NORM_INF, tol=1e-7)
    assert rc == 0 and it > 0
    err = g.integrate((u - ua) ** 2) / g.integrate(np.ones(g.N))
    assert err < 1e-12


def test_laplacian_symmetric_spd():
    # cdg_cg.cpp:214-244: the assembled operator is symmetric
    g = _poly_box(2, [2, 2], 3)
    n = g.N
    H = np.zeros((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[:] = 0
        e[j] = 1.0
        H[:, j] = g.helmholtz(e)
    assert np.allclose(H, H.T, rtol=0, atol=100 * np.finfo(float).eps * np.abs(H).max())


def test_hackathon_derivative_known_answer():
    # hackathon_driver.cpp:224-252: d/dx of x^p y^q z^r within 100 eps (L2)
    g = _poly_box(3, [3, 2, 2], 4)
    x, y, z = g.xyz[0], g.xyz[1], g.xyz[2]
    u = x ** 2 * y ** 2 * z
    for idir, exact in ((1, 2 * x * y ** 2 * z), (2, 2 * x ** 2 * y * z), (3, x ** 2 * y ** 2)):
        du = g.deriv(u, idir)
        err = np.sqrt(g.integrate((du - exact) ** 2) / g.integrate(exact ** 2))
        assert err < 100 * np.finfo(float).eps


def test_integrate_volume_and_polynomial():
    # cdg_mass.cpp checks integrate(1) = volume; on the box also a monomial
    g = O.OracleBox(3, [2, 3, 2], 5, length=[2.0, 1.0, 0.5])
    assert abs(g.integrate(np.ones(g.N)) - 1.0) < 1e-13
    x = g.xyz[0]
    assert abs(g.integrate(x ** 3) - (2.0 ** 4 / 4) * 0.5) < 1e-12


def test_rk_advection_converges_to_exact():
    # periodic advection of a smooth mode: RK4 with Smooth converges
    # spectrally in p toward the exact translated solution
    errs = []
    for p in (4, 6, 8):
        g = O.OracleBox(2, [4, 4], p, periodic=[1, 1])
        x, y = g.xyz[0], g.xyz[1]
        u0 = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
        first = g.members[g.class_ptr[:-1]]
        u0 = u0[first][g.node_class]
        c = [np.ones(g.N), 0.5 * np.ones(g.N)]
        dt, nsteps = 5e-4, 100
        u = [u0.copy()]
        g.rk_advance(0, 0.0, 4, u, c=c, dt=dt, nsteps=nsteps)
        T = dt * nsteps
        exact = np.sin(2 * np.pi * (x - T)) * np.cos(2 * np.pi * (y - 0.5 * T))
        errs.append(np.max(np.abs(u[0] - exact)))
    assert errs[0] > 10 * errs[1] > 100 * errs[2] and errs[2] < 1e-6


def test_oracle_vs_ref_build_if_present():
    ref = O.load_ref()
    if ref is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    P = C.POINTER(C.c_double)
    for p in (2, 5, 8, 11):
        n = p + 1
        a = [np.zeros(n), np.zeros(n), np.zeros(n * n)]
        ref.gfr_gll(p, *[v.ctypes.data_as(P) for v in a])
        b = O.gll(p)
        for u, v in zip(a, b):
            assert np.array_equal(bits(u), bits(v))


def test_deformed_oracle_reduces_to_regular():
    """The deformed-element oracle (def_prod, deriv, GAdvect, dudt with a
    full metric) equals the regular-element oracle when dXi/dX is diagonal."""
    b = O.OracleBox(3, [2, 1, 2], 5, periodic=[1, 0, 0])
    rng = np.random.default_rng(4)
    N = b.N
    X = [[b.dXidX[i] if i == k else np.zeros(N) for k in range(3)] for i in range(3)]
    d = O.OracleDef(b, X, b.Jac, 3)
    u = rng.standard_normal(N)
    c = [rng.standard_normal(N) for _ in range(3)]
    ref = b.helmholtz(u, p=0.7, q_vec=np.full(N, 0.3))
    assert np.max(np.abs(d.helmholtz(u, p=0.7, q_vec=np.full(N, 0.3)) - ref)) <= 1e-14 * np.max(np.abs(ref))
    for k in (1, 2, 3):
        assert np.array_equal(d.deriv(u, k), b.deriv(u, k))
    ra = b.advect(u, c)
    assert np.max(np.abs(d.advect(u, c) - ra)) <= 1e-14 * np.max(np.abs(ra))
    for kind, nst in ((0, 1), (1, 3), (2, 1)):
        us = [rng.standard_normal(N) for _ in range(nst)]
        r1 = d.dudt(kind, 0.02, us, c if kind == 0 else None)
        r2 = b.dudt(kind, 0.02, us, c if kind == 0 else None)
        for a, bb in zip(r1, r2):
            assert np.max(np.abs(a - bb)) <= 1e-13 * np.max(np.abs(bb))


def test_constrain2sphere_oracle_known_values():
    """GMTK::constrain2sphere (2) updates the components in turn: a radial
    vector loses its x component exactly, and y then sees the updated x."""
    xyz = [np.array([1.0, 0.0]), np.array([2.0, 0.0]), np.array([2.0, 3.0])]
    v = [xyz[0].copy(), xyz[1].copy(), xyz[2].copy()]
    O.constrain2sphere(xyz, v)
    r2 = 9.0
    assert v[0][0] == 0.0
    assert v[1][0] == (2.0 * (r2 - 4.0) - 2.0 * 2.0 * 2.0) / r2
    # node 1 (0, 0, 3): only z survives the x/y terms
    assert v[0][1] == 0.0 and v[1][1] == 0.0
    assert v[2][1] == (3.0 * (r2 - 9.0)) / r2
