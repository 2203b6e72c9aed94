"""Host logic without a GPU: synthetic meshes and the bit-exact AMG setup.

The reference-built oracle (oracle/_ref) is the checker: mesh connectivity
must equal the reference's own tet fixture, and every level of the AMG
hierarchy (CSR, inverse diagonal, prolongation, aggregates, damping) must be
bit-identical to MatrixFreeVcyclePreconditioner::setup with the Balanced
NativeAMG parameters (core/linalg/hypre_amg.cpp:172-219)."""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from tests import cases


@pytest.mark.parametrize("n", [3, 4, 7])
def test_tet_generator_matches_reference_fixture(ref, n):
    mine = cg.tet_case(n)
    fix = ref.fixture_tet_v52(n)
    for k in ("face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets", "cell_faces"):
        assert np.array_equal(getattr(mine, k), fix[k]), k


def test_hex_generator_counts():
    m = cg.hex_case(4, 5, 6)
    nc = 4 * 5 * 6
    nf_int = 3 * 4 * 5 * 6 - (5 * 6 + 4 * 6 + 4 * 5)
    nf_bnd = 2 * (5 * 6 + 4 * 6 + 4 * 5)
    assert m.n_cells == nc and m.n_faces == nf_int + nf_bnd
    assert (m.neighbour >= 0).sum() == nf_int
    assert set(np.unique(m.patch_of_face[m.neighbour < 0])) == {0, 1, 2, 3, 4, 5}
    assert np.all(m.patch_of_face[m.neighbour >= 0] == -1)
    # every cell lists 6 faces and each face belongs to its owner (and neighbour)
    assert np.all(np.diff(m.cell_offsets) == 6)


def test_jittered_tets_keep_positive_face_orientation(ref):
    m = cases.simple_mesh(10)
    g = ref.geometry(m)
    nf, nc = m.n_faces, m.n_cells
    sf = g["face_Sf"].reshape(3, nf)
    cc = g["cell_centres"].reshape(3, nc)
    internal = m.neighbour >= 0
    d = cc[:, m.neighbour[internal]] - cc[:, m.owner[internal]]
    assert np.all((sf[:, internal] * d).sum(0) > 0)
    assert np.all(g["cell_volumes"] > 0)


def _compare_hierarchy(ref, ro, co, va):
    R = ref.Amg(ro, co, va)
    amg = cg.NativeBoomerAMGPreconditioner(None)
    assert amg.setup_host(ro, co, va), amg.last_error()
    assert R.num_levels() == len(amg.hierarchy_level_sizes())
    for l in range(R.num_levels()):
        a, b = R.level(l), amg.export_level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag", "p_columns", "p_values"):
            assert np.array_equal(a[k], b[k]), (l, k)
        if a["p_offsets"] is not None:
            assert np.array_equal(a["p_offsets"], b["p_offsets"])
            assert np.array_equal(a["aggregate"], b["aggregate"])
    assert R.omega == amg.omega
    return amg


@pytest.mark.parametrize("n", [8, 16, 32])   # 32: the 32^3 hex Poisson benchmark system itself
def test_amg_setup_bit_exact_poisson_hex(ref, n):
    m, bc, src = cases.poisson_case(n)
    ro, co, va, rhs, _ = ref.assemble_diffusion(m, bc, 1.0, src)
    amg = _compare_hierarchy(ref, ro, co, va)
    assert amg.hierarchy_level_sizes()[0] == n ** 3


@pytest.mark.parametrize("n", [4, 8, 12])
def test_amg_setup_bit_exact_pressure_tets(ref, n):
    m = cases.simple_mesh(n)
    g = ref.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    _compare_hierarchy(ref, r["row_offsets"], r["columns"], r["values"])


def test_amg_setup_bit_exact_anisotropic_boundary_layer(ref):
    m = cg.boundary_layer_case(12, 10, 6, dy0=1e-3, growth=1.2, jitter=0.05, seed=5)
    bc = np.full(m.n_faces, np.nan)
    bc[m.patch_of_face == 0] = 0.0
    src = cg.random_field(m.n_cells, "uniform", -1.0, 1.0, 3)
    ro, co, va, rhs, _ = ref.assemble_diffusion(m, bc, 1.0, src)
    _compare_hierarchy(ref, ro, co, va)


def test_reference_rebuild_from_stored_transfers_is_its_own_setup(ref):
    # The reference's setup with each level's C/F interpolation read back from
    # an earlier complete run (the way the benchmark's CPU legs rebuild the
    # reference's own 64^3 hierarchy) gives the identical hierarchy.
    m = cases.simple_mesh(12)
    g = ref.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    R = ref.Amg(r["row_offsets"], r["columns"], r["values"])
    transfers, rows = {}, []
    for l in range(R.num_levels()):
        lv = R.level(l)
        rows.append(lv["inv_diag"].size)
        if lv["p_offsets"] is not None:
            for k in ("p_offsets", "p_columns", "p_values", "aggregate"):
                transfers[f"{k}_{l}"] = lv[k]
    T = ref.AmgFromTransfers(r["row_offsets"], r["columns"], r["values"], transfers, rows)
    assert ref.hierarchy_sha256(T) == ref.hierarchy_sha256(R)
    assert T.omega == R.omega
    x0, rep0 = R.solve_gmres(r["b"])
    x1, rep1 = T.solve_gmres(r["b"])
    assert rep0["iterations"] == rep1["iterations"] and np.array_equal(x0, x1)


def test_amg_setup_rejects_zero_diagonal():
    ro = np.array([0, 2, 4])
    co = np.array([0, 1, 0, 1])
    va = np.array([0.0, -1.0, -1.0, 2.0])
    amg = cg.NativeBoomerAMGPreconditioner(None)
    assert not amg.setup_host(ro, co, va)
    assert "diagonal" in amg.last_error()


def test_amg_setup_is_deterministic_across_thread_counts(ref, monkeypatch):
    # host threads only change the schedule, never the arithmetic
    m = cases.simple_mesh(8)
    g = ref.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    a = cg.NativeBoomerAMGPreconditioner(None)
    a.setup_host(r["row_offsets"], r["columns"], r["values"])
    b = cg.NativeBoomerAMGPreconditioner(None)
    b.setup_host(r["row_offsets"], r["columns"], r["values"])
    for l in range(len(a.hierarchy_level_sizes())):
        la, lb = a.export_level(l), b.export_level(l)
        assert np.array_equal(la["values"], lb["values"])


def test_host_setup_reproduces_golden_hierarchy():
    # the reference's own hierarchy of the 4^3 x 6 tet pressure system, stored
    # by tests/golden/make_golden.py: no reference build needed
    from pathlib import Path
    z = dict(np.load(Path(__file__).resolve().parent / "golden" / "pressure_tet4.npz"))
    amg = cg.NativeBoomerAMGPreconditioner(None)
    assert amg.setup_host(z["row_offsets"], z["columns"], z["values"]), amg.last_error()
    assert len(amg.hierarchy_level_sizes()) == int(z["n_levels"])
    for l in range(int(z["n_levels"])):
        mine = amg.export_level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag"):
            assert np.array_equal(mine[k], z[f"L{l}_{k}"]), (l, k)
        if f"L{l}_p_offsets" in z:
            for k in ("p_offsets", "p_columns", "p_values"):
                assert np.array_equal(mine[k], z[f"L{l}_{k}"]), (l, k)
    assert amg.omega == float(z["omega"])


def _pressure_pair(n):
    """Two pressure-correction systems on one mesh (same pattern, other a_P)."""
    from oracle import cfdx_oracle as co
    m = cases.simple_mesh(n)
    g = co.geometry(m)
    out = []
    for off in (0, 11):
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=off)
        a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
        out.append((a["row_offsets"], a["columns"], a["values"]))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    return out


def test_host_numeric_refresh_matches_reference(ref):
    (ro, co_, va1), (_, _, va2) = _pressure_pair(8)
    R = ref.Amg(ro, co_, va1)
    assert R.update_values(ro, co_, va2)
    amg = cg.NativeBoomerAMGPreconditioner(None)
    assert amg.setup_host(ro, co_, va1)
    assert amg.update_values_host(ro, co_, va2)
    assert R.num_levels() == len(amg.hierarchy_level_sizes())
    for l in range(R.num_levels()):
        a, b = R.level(l), amg.export_level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag", "p_values"):
            assert np.array_equal(a[k], b[k]), (l, k)
    assert R.omega == amg.omega
    # a changed pattern is refused and leaves the hierarchy as it was
    before = amg.export_level(1)["values"].copy()
    assert not amg.update_values_host(ro, np.roll(co_, 1), va2)
    assert "pattern" in amg.last_error()
    assert np.array_equal(amg.export_level(1)["values"], before)


def test_reusable_context_lifecycle_on_the_host():
    """linear_solver_context.h:30-65: structure change -> setup, value change ->
    refresh, unchanged -> reuse; a refused refresh rebuilds."""
    import cfdx_dev_b200 as cg
    from tests import cases
    from oracle import cfdx_oracle as co_
    m = cases.simple_mesh(4)
    g = co_.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = co_.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, co, va = a["row_offsets"], a["columns"], a["values"]
    ctx = cg.ReusablePreconditionerContext(cg.NativeBoomerAMGPreconditioner())
    assert ctx.prepare((ro, co, va))
    assert ctx.prepare((ro, co, va))
    assert ctx.prepare((ro, co, va * 1.5))                 # same pattern, new values
    assert ctx.stats == dict(full_setups=1, numeric_updates=1, unchanged_reuses=1, solves=0)
    # a different structure (one coupling dropped symmetrically) sets up again
    rows = np.repeat(np.arange(ro.size - 1), np.diff(ro))
    drop = np.nonzero((rows != co) & (((rows == 0) & (co == co[ro[0]:ro[1]][-1])) |
                                      ((co == 0) & (rows == co[ro[0]:ro[1]][-1]))))[0]
    keep = np.setdiff1d(np.arange(co.size), drop)
    ro2 = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=ro.size - 1))])
    assert ctx.prepare((ro2, co[keep], va[keep]))
    assert ctx.stats["full_setups"] == 2
    assert not ctx.prepare((ro, co, np.where(np.arange(va.size) == 3, np.nan, va)))   # rejected input


def test_oracle_case_library_builds_the_same_inputs(ref):
    # the CPU reference legs build their inputs with the generator compiled
    # alone (oracle/cases.py); they must equal the package's, bit for bit
    from oracle import cases as oc
    a, b = cases.simple_mesh(9), oc.simple_mesh(9)
    for k in ("px", "py", "pz", "face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets",
              "cell_faces", "patch_of_face", "patch_types"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    cc = ref.geometry(a)["cell_centres"]
    for s in (0, 3):
        for x, y in zip(cases.simple_fields(a, cc, seed_offset=s), oc.simple_fields(b, cc, seed_offset=s)):
            assert np.array_equal(x, y)


def test_null_space_setup_contract_and_hierarchy(ref):
    """NativeBoomerAMGPreconditioner(constant_null_space=true): setup and
    update_values require vanishing row sums (amg_preconditioner.h:84, 250,
    1289-1308); the hierarchy itself is the ordinary one, bit for bit."""
    m = cases.simple_mesh(6)
    g = ref.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    neumann = ref.simple_assemble(m, U, rAU, p, 1.0, np.zeros_like(fixed), value)
    dirichlet = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, co_, va = neumann["row_offsets"], neumann["columns"], neumann["values"]
    R = ref.Amg(ro, co_, va, constant_null_space=True)
    amg = cg.NativeBoomerAMGPreconditioner(None, constant_null_space=1)
    assert amg.setup_host(ro, co_, va), amg.last_error()
    assert R.num_levels() == len(amg.hierarchy_level_sizes())
    for l in range(R.num_levels()):
        a, b = R.level(l), amg.export_level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag", "p_columns", "p_values"):
            assert np.array_equal(a[k], b[k]), (l, k)
    assert R.omega == amg.omega
    # a refresh with values that keep the row sums zero is accepted (a scaled copy) ...
    assert amg.update_values_host(ro, co_, 2.0 * va)
    # ... one that breaks them is refused, as is a setup on the Dirichlet-fixed operator
    assert not amg.update_values_host(ro, co_, va + 1e-3 * np.abs(va))
    other = cg.NativeBoomerAMGPreconditioner(None, constant_null_space=1)
    assert not other.setup_host(dirichlet["row_offsets"], dirichlet["columns"], dirichlet["values"])
    assert "null-space" in other.last_error()
    with pytest.raises(RuntimeError):
        ref.Amg(dirichlet["row_offsets"], dirichlet["columns"], dirichlet["values"], constant_null_space=True)
