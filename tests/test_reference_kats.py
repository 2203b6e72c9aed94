"""Known-answer tests of the reference's own test suite, restated against the
oracle and the library's host code (no GPU).

Each case names the reference test it mirrors and keeps that test's inputs
and expected values:

* tests/unit/test_scalar_diffusion.cpp:156-233 -- the 1-D chain of n hex
  cells with phi = x^2 (source -2): Dirichlet/Dirichlet and
  Dirichlet/Neumann give x_c^2 - dx^2/4 (the two-point stencil's known
  offset), pure Neumann with the reference-cell gauge gives x_c^2 + 3, each
  with a zero conservation balance;
* tests/unit/test_gmres_solver.cpp:125-233 -- the diagonal 3x3, the 1-D
  Poisson system, an already converged solve, a restarted solve and the exact
  nonsymmetric 3x3;
* tests/validation/test_mms_scalar_diffusion.cpp:277-380 -- the 3-D
  manufactured solution sin(pi x) sin(pi y) sin(pi z) on 4^3 .. 32^3 hex
  cubes (Dirichlet at the face centres, source 3 pi^2 phi): observed L2 order
  >= 1.80 between successive refinements;
* tests/validation/test_n12_pressure_continuity_mms.cpp -- on the y-channel
  of n hex cells the divergence-free face flux sin^2(pi y_f) Sf_x has a cell
  continuity defect below 1e-13 (L1, L2, max) for n = 16, 32, 64;
* tests/validation/test_n9_s9_rhie_chow_consistency.cpp:324-422 -- the
  Rhie-Chow face flux on channels of hex cells: invariant under a constant
  pressure offset, and on a non-uniform channel under an affine pressure the
  face-averaged gradient is exact and each internal face carries the linear
  flux minus the pressure-jump response;
* tests/validation/test_amg_preconditioner_qualification.cpp -- the small
  multilevel case (1-D Poisson, N = 17, :805-830), the transfer gates
  (Galerkin and symmetric coarse operators, unit row sums of P, no empty
  column, :262-273) and the stable smoother damping (:1018-1047).
"""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200.api import HostMesh
from oracle import cfdx_oracle as co
from tests import cases
from tests.test_poisson_driver import oracle_poisson_mixed


# ------------------------------------------------------------ 1-D chain mesh
def chain_mesh(n, nodes=None):
    """make_1d_chain (test_scalar_diffusion.cpp:12-71): n unit-section hex cells
    along x with their own 8 points each; faces: left end, right end, then per
    cell y0, y1, z0, z1, then the n-1 internal faces.  ``nodes`` (n + 1 x
    positions) replaces the uniform spacing on [0, 1]; patches are the left
    end (0), the right end (1) and the side walls (2)."""
    xs = np.linspace(0.0, 1.0, n + 1) if nodes is None else np.asarray(nodes, float)
    pts = []
    for i in range(n):
        x0, x1 = (i / n, (i + 1) / n) if nodes is None else (xs[i], xs[i + 1])
        pts += [(x0, 0, 0), (x1, 0, 0), (x1, 1, 0), (x0, 1, 0), (x0, 0, 1), (x1, 0, 1), (x1, 1, 1), (x0, 1, 1)]
    pts = np.array(pts, float)
    faces, owner, neighbour, patch = [], [], [], []

    def add(v, o, nb, pt):
        faces.append(v)
        owner.append(o)
        neighbour.append(nb)
        patch.append(pt)
        return len(faces) - 1

    left = add([0, 4, 7, 3], 0, -1, 0)
    b = 8 * (n - 1)
    right = add([b + 1, b + 2, b + 6, b + 5], n - 1, -1, 1)
    side = []
    for i in range(n):
        b = 8 * i
        side.append([add([b, b + 1, b + 5, b + 4], i, -1, 2), add([b + 3, b + 7, b + 6, b + 2], i, -1, 2),
                     add([b, b + 3, b + 2, b + 1], i, -1, 2), add([b + 4, b + 5, b + 6, b + 7], i, -1, 2)])
    internal = [add([8 * i + 1, 8 * i + 2, 8 * i + 6, 8 * i + 5], i, i + 1, -1) for i in range(n - 1)]
    cells = [[left if i == 0 else internal[i - 1], right if i + 1 == n else internal[i]] + side[i] for i in range(n)]
    fo = np.concatenate([[0], np.cumsum([len(f) for f in faces])]).astype(np.int64)
    co_ = np.concatenate([[0], np.cumsum([len(c) for c in cells])]).astype(np.int64)
    types = cg.hex_case(1).patch_types[:3].copy()
    return HostMesh(px=pts[:, 0].copy(), py=pts[:, 1].copy(), pz=pts[:, 2].copy(), face_offsets=fo,
                    face_vertices=np.concatenate(faces).astype(np.int64), owner=np.array(owner, np.int64),
                    neighbour=np.array(neighbour, np.int64), cell_offsets=co_,
                    cell_faces=np.concatenate(cells).astype(np.int64), patch_of_face=np.array(patch, np.int32),
                    patch_types=types)


def conservation_balance(m, bc, types, src, x, diffusivity=1.0):
    """poisson_conservation_balance (core/solvers/scalar_diffusion.h:241-300):
    the sources plus the prescribed boundary fluxes."""
    g = co.geometry(m)
    balance = float(np.sum(src * g["cell_volumes"]))
    nf = m.owner.size
    for f in range(nf):
        if m.neighbour[f] >= 0 or not np.isfinite(bc[f]):
            continue
        o = m.owner[f]
        area = np.linalg.norm(g["face_Sf"][[f, nf + f, 2 * nf + f]])
        if types is not None and types[f] == 1:
            balance += bc[f] * area
        else:
            fc = g["face_centres"][[f, nf + f, 2 * nf + f]]
            nc = m.cell_offsets.size - 1
            cc = g["cell_centres"][[o, nc + o, 2 * nc + o]]
            d = np.linalg.norm(fc - cc)
            balance += diffusivity * area * (bc[f] - x[o]) / d
    return balance


N_CHAIN = 8


def _chain_case(kind):
    m = chain_mesh(N_CHAIN)
    nf = m.owner.size
    bc = np.full(nf, np.nan)
    types = np.zeros(nf, np.int32)
    if kind == "dirichlet":
        bc[0], bc[1] = 0.0, 1.0
    elif kind == "mixed":
        bc[0], bc[1] = 0.0, 2.0
        types[1] = 1
    else:                                   # pure Neumann: every face a flux
        types[:] = 1
        bc[0], bc[1] = 0.0, 2.0
    return m, bc, types, np.full(N_CHAIN, -2.0)


@pytest.mark.parametrize("kind", ["dirichlet", "mixed", "neumann"])
def test_chain_poisson_known_answers(kind):
    m, bc, types, src = _chain_case(kind)
    xc = co.geometry(m)["cell_centres"][:N_CHAIN]
    dx = 1.0 / N_CHAIN
    if kind == "neumann":
        ref_value = xc[0] ** 2 + 3.0
        x, rep = oracle_poisson_mixed(m, bc, src, types, tolerance=1e-12, ref_cell=0, ref_value=ref_value)
        want = xc ** 2 + 3.0
    else:
        x, rep = oracle_poisson_mixed(m, bc, src, types, tolerance=1e-12)
        want = xc ** 2 - dx * dx / 4.0
    assert rep["status"] == 0
    np.testing.assert_allclose(x, want, rtol=0, atol=1e-12)
    assert abs(conservation_balance(m, bc, types, src, x)) <= 1e-12


def test_chain_mesh_matches_reference_solver(ref):
    """The same chain through the reference's own solve_poisson_mixed."""
    for kind in ("dirichlet", "mixed"):
        m, bc, types, src = _chain_case(kind)
        x, rep = oracle_poisson_mixed(m, bc, src, types, tolerance=1e-12)
        xr, rr = ref.solve_poisson_mixed(m, bc, src, types, tolerance=1e-12)
        assert rep["iterations"] == rr["iterations"] and np.array_equal(x, xr)


def test_poisson_3d_manufactured_solution_is_second_order():
    l2 = []
    for n in (4, 8, 16, 32):
        m = cg.hex_case(n)
        g = co.geometry(m)
        nf, nc = m.owner.size, m.cell_offsets.size - 1
        fc = g["face_centres"].reshape(3, nf)
        cc = g["cell_centres"].reshape(3, nc)
        phi = lambda p: np.sin(np.pi * p[0]) * np.sin(np.pi * p[1]) * np.sin(np.pi * p[2])  # noqa: E731
        bc = phi(fc)                                 # every face a Dirichlet value; internal ones unused
        bc[m.neighbour >= 0] = np.nan
        src = 3.0 * np.pi ** 2 * phi(cc)
        x, rep = oracle_poisson_mixed(m, bc, src, max_iterations=10000, tolerance=1e-12)
        assert rep["status"] == 0
        err = x - phi(cc)
        vol = g["cell_volumes"]
        l2.append(np.sqrt(np.sum(vol * err * err) / np.sum(vol)))
    orders = [np.log(l2[i - 1] / l2[i]) / np.log(2.0) for i in range(1, len(l2))]
    assert min(orders) >= 1.80, orders


def channel_mesh(n):
    """make_channel (test_n12_pressure_continuity_mms.cpp:13-88): n hex cells
    stacked in y on the unit cube, 8 points each; faces: bottom, top, then per
    cell x0, x1, z0, z1, then the n-1 internal faces."""
    pts = []
    for j in range(n):
        y0, y1 = j / n, (j + 1) / n
        pts += [(0, y0, 0), (1, y0, 0), (1, y1, 0), (0, y1, 0), (0, y0, 1), (1, y0, 1), (1, y1, 1), (0, y1, 1)]
    pts = np.array(pts, float)
    faces, owner, neighbour = [], [], []

    def add(v, o, nb):
        faces.append(v)
        owner.append(o)
        neighbour.append(nb)
        return len(faces) - 1

    bottom = add([0, 1, 5, 4], 0, -1)
    b = 8 * (n - 1)
    top = add([b + 3, b + 7, b + 6, b + 2], n - 1, -1)
    side = []
    for j in range(n):
        b = 8 * j
        side.append([add([b, b + 4, b + 7, b + 3], j, -1), add([b + 1, b + 2, b + 6, b + 5], j, -1),
                     add([b, b + 3, b + 2, b + 1], j, -1), add([b + 4, b + 5, b + 6, b + 7], j, -1)])
    internal = [add([8 * j + 3, 8 * j + 7, 8 * j + 6, 8 * j + 2], j, j + 1) for j in range(n - 1)]
    cells = [[bottom if j == 0 else internal[j - 1], top if j + 1 == n else internal[j]] + side[j] for j in range(n)]
    nf = len(faces)
    patch = np.where(np.array(neighbour) < 0, 0, -1).astype(np.int32)
    return HostMesh(px=pts[:, 0].copy(), py=pts[:, 1].copy(), pz=pts[:, 2].copy(),
                    face_offsets=np.arange(0, 4 * nf + 1, 4, dtype=np.int64),
                    face_vertices=np.concatenate(faces).astype(np.int64), owner=np.array(owner, np.int64),
                    neighbour=np.array(neighbour, np.int64), cell_offsets=np.arange(0, 6 * n + 1, 6, dtype=np.int64),
                    cell_faces=np.concatenate(cells).astype(np.int64), patch_of_face=patch,
                    patch_types=cg.hex_case(1).patch_types[:1].copy())


@pytest.mark.parametrize("n", [16, 32, 64])
def test_manufactured_divergence_free_flux_has_no_continuity_defect(n):
    m = channel_mesh(n)
    g = co.geometry(m)
    nf = m.owner.size
    fy = g["face_centres"][nf:2 * nf]
    phi = np.sin(np.pi * fy) ** 2 * g["face_Sf"][:nf]
    vol = g["cell_volumes"]
    r = np.zeros(n)
    for c in range(n):
        net = 0.0
        for f in m.cell_faces[m.cell_offsets[c]:m.cell_offsets[c + 1]]:
            net += phi[f] if m.owner[f] == c else -phi[f]
        r[c] = net / vol[c]
    V = vol.sum()
    assert np.sum(np.abs(r) * vol) / V < 1e-13
    assert np.sqrt(np.sum(r * r * vol) / V) < 1e-13
    assert np.max(np.abs(r)) < 1e-13


# ------------------------------------------------------------ Rhie-Chow KATs
def test_rhie_chow_flux_pressure_offset_invariance():
    m = chain_mesh(2)
    nf = m.owner.size
    U = np.zeros(6)
    rAU = np.ones(6)
    fixed, value = np.zeros(3, np.int32), np.zeros(3)            # zero-gradient pressure everywhere
    phi0 = co.rhie_chow_flux(m, U, rAU, np.array([-2.0, 4.0]), 1.0, fixed, value)
    phi1 = co.rhie_chow_flux(m, U, rAU, np.array([1002.0, 1008.0]), 1.0, fixed, value)
    assert phi0.size == nf
    np.testing.assert_allclose(phi0, phi1, rtol=0, atol=1e-12)


def test_rhie_chow_flux_affine_pressure_nonuniform_channel():
    nodes = [0.0, 0.5, 2.0, 4.0, 7.0]
    m = chain_mesh(4, nodes)
    g = co.geometry(m)
    nc, nf = 4, m.owner.size
    xc = g["cell_centres"][:nc]
    U = np.concatenate([np.full(nc, 2.0), np.zeros(2 * nc)])
    rAU = np.ones(3 * nc)
    p = 1.0 + 2.0 * xc
    fixed = np.array([1, 1, 0], np.int32)                          # inlet, outlet fixed; walls zero-gradient
    value = np.array([1.0, 15.0, 0.0])
    phi = co.rhie_chow_flux(m, U, rAU, p, 1.0, fixed, value)
    grad = co.gauss_gradient(m, p, fixed, value)
    vol = g["cell_volumes"]
    internal = np.nonzero(m.neighbour >= 0)[0]
    assert internal.size == 3
    for f in internal:
        o, n_ = m.owner[f], m.neighbour[f]
        dau = 0.5 * (vol[o] * rAU[o] + vol[n_] * rAU[n_])
        dx = xc[n_] - xc[o]
        sfx = g["face_Sf"][f]
        grad_face = 0.5 * (grad[o] + grad[n_])
        assert grad_face == pytest.approx(2.0, abs=1e-12)
        linear = 2.0 * sfx
        assert phi[f] == pytest.approx(linear - dau * (p[n_] - p[o]) / dx * sfx, abs=1e-12)


# ---------------------------------------------------------------- GMRES KATs
def _csr(dense):
    ro, cols, va = [0], [], []
    for row in dense:
        nz = np.nonzero(row)[0]
        cols += nz.tolist()
        va += row[nz].tolist()
        ro.append(len(cols))
    return np.array(ro), np.array(cols), np.array(va, float)


def _poisson_1d(n):
    return _csr(2 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1))


def test_gmres_diagonal_and_1d_poisson():
    ro, cols, va = _csr(np.diag([2.0, 3.0, 4.0]))
    x, rep = co.solve_gmres(ro, cols, va, np.array([2.0, 6.0, 12.0]), None, tolerance=1e-12)
    assert rep["status"] == 0 and rep["iterations"] > 0 and rep["residual_relative"] < 1e-10
    np.testing.assert_allclose(x, [1.0, 2.0, 3.0], atol=1e-10)
    ro, cols, va = _poisson_1d(5)
    b = np.array([0.0, 1.0, 1.0, 1.0, 0.0])
    x, rep = co.solve_gmres(ro, cols, va, b, None, tolerance=1e-12)
    assert rep["status"] == 0 and rep["residual_relative"] < 1e-10
    np.testing.assert_allclose(co.spmv(ro, cols, va, x), b, atol=1e-10)


def test_gmres_already_converged_and_restarted():
    ro, cols, va = _csr(np.eye(2))
    x, rep = co.solve_gmres(ro, cols, va, np.zeros(2), None, tolerance=1e-12)
    assert rep["status"] == 0 and rep["iterations"] == 0
    ro, cols, va = _poisson_1d(10)
    b = np.ones(10)
    x, rep = co.solve_gmres(ro, cols, va, b, None, restart=5, tolerance=1e-12)
    assert rep["status"] == 0 and rep["residual_relative"] < 1e-10
    np.testing.assert_allclose(co.spmv(ro, cols, va, x), b, atol=1e-10)


def test_gmres_exact_nonsymmetric_3x3():
    A = np.array([[4.0, 1.0, 0.0], [-2.0, 5.0, 1.0], [1.0, -1.0, 3.0]])
    ro, cols, va = _csr(A)
    x_exact = np.array([1.0, -2.0, 0.5])
    b = co.spmv(ro, cols, va, x_exact)
    x, rep = co.solve_gmres(ro, cols, va, b, None, restart=3, max_iterations=20, tolerance=1e-12)
    assert rep["status"] == 0 and rep["residual_relative"] < 1e-11
    np.testing.assert_allclose(x, x_exact, atol=1e-10)
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1e-9


# ------------------------------------------------------------- AMG KATs
def _levels(ro, cols, va):
    amg = cg.NativeBoomerAMGPreconditioner()
    assert amg.setup_host(ro, cols, va), amg.last_error()
    return amg, [amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))]


def _dense(ro, cols, va, n_cols):
    D = np.zeros((ro.size - 1, n_cols))
    for i in range(ro.size - 1):
        for k in range(ro[i], ro[i + 1]):
            D[i, cols[k]] += va[k]
    return D


def test_small_multilevel_poisson_17():
    amg, levels = _levels(*_poisson_1d(17))
    assert len(levels) >= 2
    lv = levels[0]
    assert lv["p_columns"].size > 0
    P = _dense(lv["p_offsets"], lv["p_columns"], lv["p_values"], levels[1]["inv_diag"].size)
    assert np.max(np.abs(P.sum(axis=1) - 1.0)) < 1e-12


@pytest.mark.parametrize("system", ["poisson_hex6", "pressure_tet5"])
def test_transfer_gates(system):
    if system == "poisson_hex6":
        m, bc, src = cases.poisson_case(6)
        ro, cols, va, _ = co.assemble_diffusion(m, bc, 1.0, src)
    else:
        m = cases.simple_mesh(5)
        g = co.geometry(m)
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
        a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
        ro, cols, va = a["row_offsets"], a["columns"], a["values"]
    amg, levels = _levels(ro, cols, va)
    for l in range(len(levels) - 1):
        f, c = levels[l], levels[l + 1]
        nf, nc = f["inv_diag"].size, c["inv_diag"].size
        A = _dense(f["row_offsets"], f["columns"], f["values"], nf)
        P = _dense(f["p_offsets"], f["p_columns"], f["p_values"], nc)
        Ac = _dense(c["row_offsets"], c["columns"], c["values"], nc)
        galerkin = P.T @ A @ P
        assert np.linalg.norm(Ac - galerkin) <= 1e-12 * np.linalg.norm(galerkin)
        assert np.linalg.norm(Ac - Ac.T) <= 1e-12 * np.linalg.norm(Ac)
        assert np.max(np.abs(P.sum(axis=1) - 1.0)) <= 1e-12
        assert np.all(np.count_nonzero(P, axis=0) > 0)                 # no empty coarse column


def test_stable_smoother_damping():
    high = _csr(np.where(np.eye(3) > 0, 1.0, 0.9))                    # normalised Gershgorin bound 2.8
    low = _csr(np.where(np.eye(3) > 0, 1.0, 0.1))
    amg = cg.NativeBoomerAMGPreconditioner()
    assert amg.setup_host(*high)
    assert amg.omega == pytest.approx(1.8 / 2.8, abs=1e-14)
    assert amg.update_values_host(*low)
    assert amg.omega == pytest.approx(0.7, abs=1e-14)
    assert amg.setup_host(*high)
    assert amg.omega == pytest.approx(1.8 / 2.8, abs=1e-14)
