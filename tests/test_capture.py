"""Linear-system replay files (.cfdxlin) without a GPU.

Mirrors the reference's tests/unit/test_linear_system_capture.cpp (exact FP64
round trip with the initial guess, checksum detection of a changed matrix,
truncated files, refusal of non-finite or mis-sized input and of unknown
metadata before anything is written, constant null-space metadata) and
checks the library against the reference's own writer and reader built into
oracle/_ref: files written by either are byte-identical and each side reads
the other's exactly.  The golden file tests/golden/pressure_tet4.cfdxlin was
written by the reference (tests/golden/make_golden.py)."""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200.api import CAPTURE_DIFFUSION, CAPTURE_PRESSURE_POISSON, CfdxgError
from tests import cases

GOLDEN = cases.ROOT / "tests" / "golden"


def _matrix3():
    # the 3x3 matrix of test_linear_system_capture.cpp:17-27
    ro = np.array([0, 2, 5, 7])
    co = np.array([0, 1, 0, 1, 2, 1, 2])
    va = np.array([5.0, -2.0, -2.0, 5.0, -1.0, -1.0, 3.0])
    return ro, co, va


def test_exact_fp64_round_trip_with_initial_guess(tmp_path):
    ro, co, va = _matrix3()
    b, x = np.array([1.25, -2.0, 3.25]), np.array([0.125, -0.125, 0.75])
    path = tmp_path / "c.cfdxlin"
    checksum = cg.write_linear_system_capture(path, ro, co, va, b, x, problem=CAPTURE_DIFFUSION,
                                              max_iterations=130, tolerance=1e-12)
    c = cg.read_linear_system_capture(path)
    for k, v in (("row_offsets", ro), ("columns", co), ("values", va), ("rhs", b), ("initial_solution", x)):
        assert np.array_equal(c[k], v), k
    assert c["max_iterations"] == 130 and c["tolerance"] == 1e-12 and c["checksum"] == checksum
    assert c["problem"] == CAPTURE_DIFFUSION and c["null_space"] == 0 and c["scaling"] == 0
    assert not (tmp_path / "c.cfdxlin.tmp").exists()


def test_checksum_detects_changed_matrix(tmp_path):
    ro, co, va = _matrix3()
    path = tmp_path / "c.cfdxlin"
    cg.write_linear_system_capture(path, ro, co, va, np.ones(3), np.zeros(3), tolerance=1e-12)
    text = path.read_text()
    assert "4014000000000000" in text                        # bit pattern of 5.0
    path.write_text(text.replace("4014000000000000", "4018000000000000", 1))   # 6.0
    with pytest.raises(CfdxgError, match="checksum"):
        cg.read_linear_system_capture(path)


def test_truncated_and_malformed_files_are_rejected(tmp_path):
    path = tmp_path / "c.cfdxlin"
    path.write_text("CFDX_LINEAR_REPLAY_V1\n0 0 0\n3 3 7 50\n")
    with pytest.raises(CfdxgError, match="truncated"):
        cg.read_linear_system_capture(path)
    path.write_text("CFDX_LINEAR_REPLAY_V2\n")
    with pytest.raises(CfdxgError, match="unsupported"):
        cg.read_linear_system_capture(path)
    path.write_text("CFDX_LINEAR_REPLAY_V1\n9 0 0\n3 3 7 50\n")
    with pytest.raises(CfdxgError, match="metadata"):
        cg.read_linear_system_capture(path)
    path.write_text("CFDX_LINEAR_REPLAY_V1\n0 0 0\n2000001 2000001 7 50\n")
    with pytest.raises(CfdxgError, match="limits"):
        cg.read_linear_system_capture(path)
    with pytest.raises(CfdxgError, match="open"):
        cg.read_linear_system_capture(tmp_path / "missing.cfdxlin")
    # a complete file followed by more data is not the file that was written
    ro, co, va = _matrix3()
    cg.write_linear_system_capture(path, ro, co, va, np.ones(3), np.zeros(3))
    path.write_text(path.read_text() + "0\n")
    with pytest.raises(CfdxgError, match="trailing"):
        cg.read_linear_system_capture(path)


def test_writer_refuses_invalid_input_before_writing(tmp_path):
    ro, co, va = _matrix3()
    path = tmp_path / "c.cfdxlin"
    b = np.ones(3)
    b[1] = np.nan
    for kw in (dict(rhs=b, initial_solution=np.zeros(3)),
               dict(rhs=np.ones(3), initial_solution=np.array([0.0, np.inf, 0.0])),
               dict(rhs=np.ones(3), initial_solution=np.zeros(3), problem=999),
               dict(rhs=np.ones(3), initial_solution=np.zeros(3), null_space=2),
               dict(rhs=np.ones(3), initial_solution=np.zeros(3), scaling=5),
               dict(rhs=np.ones(3), initial_solution=np.zeros(3), max_iterations=0),
               dict(rhs=np.ones(3), initial_solution=np.zeros(3), tolerance=0.0)):
        with pytest.raises(CfdxgError):
            cg.write_linear_system_capture(path, ro, co, va, **kw)
        assert not path.exists() and not (tmp_path / "c.cfdxlin.tmp").exists()
    with pytest.raises(CfdxgError):           # unsorted columns in row 1
        cg.write_linear_system_capture(path, ro, [0, 1, 1, 0, 2, 1, 2], va, np.ones(3), np.zeros(3))
    with pytest.raises(ValueError):
        cg.write_linear_system_capture(path, ro, co, va, np.ones(2), np.zeros(3))
    assert not path.exists()


def test_constant_null_space_metadata_preserved(tmp_path):
    path = tmp_path / "c.cfdxlin"
    cg.write_linear_system_capture(path, [0, 2, 4], [0, 1, 0, 1], [1.0, -1.0, -1.0, 1.0], [-1.0, 1.0], [0.0, 0.0],
                                   problem=CAPTURE_PRESSURE_POISSON, null_space=1, max_iterations=70,
                                   tolerance=1e-11)
    c = cg.read_linear_system_capture(path)
    assert c["null_space"] == 1 and c["problem"] == CAPTURE_PRESSURE_POISSON


def test_capture_iteration_list():
    # test_linear_system_capture.cpp:29-37
    assert cg.parse_linear_capture_iterations("20,21,600") == [20, 21, 600]
    for bad in ("20,20", "20,abc", "0", "20,", "", ",5", "-3", "1 2"):
        with pytest.raises(ValueError):
            cg.parse_linear_capture_iterations(bad)
    with pytest.raises(ValueError):
        cg.parse_linear_capture_iterations(",".join(str(i) for i in range(1, 34)))
    assert len(cg.parse_linear_capture_iterations(",".join(str(i) for i in range(1, 33)))) == 32


def test_golden_capture_matches_fixture():
    c = cg.read_linear_system_capture(GOLDEN / "pressure_tet4.cfdxlin")
    z = np.load(GOLDEN / "pressure_tet4.npz")
    for a, b in (("row_offsets", "row_offsets"), ("columns", "columns"), ("values", "values"), ("rhs", "b")):
        assert np.array_equal(c[a], z[b]), a
    assert not c["initial_solution"].any()
    assert c["problem"] == CAPTURE_PRESSURE_POISSON and c["max_iterations"] == 1000 and c["tolerance"] == 1e-8


def test_writer_is_byte_identical_to_golden(tmp_path):
    c = cg.read_linear_system_capture(GOLDEN / "pressure_tet4.cfdxlin")
    path = tmp_path / "mine.cfdxlin"
    cg.write_linear_system_capture(path, c["row_offsets"], c["columns"], c["values"], c["rhs"],
                                   c["initial_solution"], problem=c["problem"], null_space=c["null_space"],
                                   scaling=c["scaling"], max_iterations=c["max_iterations"],
                                   tolerance=c["tolerance"])
    assert path.read_bytes() == (GOLDEN / "pressure_tet4.cfdxlin").read_bytes()


def test_cross_read_write_with_reference(ref, tmp_path):
    rng = np.random.default_rng(5)
    m = cases.simple_mesh(5)
    g = ref.geometry(m, "fv")
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, co, va, b = a["row_offsets"], a["columns"], a["values"], a["b"]
    x0 = rng.standard_normal(b.size) * 1e-3
    theirs, mine = tmp_path / "ref.cfdxlin", tmp_path / "mine.cfdxlin"
    ref.write_capture(theirs, ro, co, va, b, x0, problem=1, null_space=1, scaling=3, max_iterations=777,
                      tolerance=3e-9)
    cg.write_linear_system_capture(mine, ro, co, va, b, x0, problem=1, null_space=1, scaling=3,
                                   max_iterations=777, tolerance=3e-9)
    assert mine.read_bytes() == theirs.read_bytes()
    c, r = cg.read_linear_system_capture(theirs), ref.read_capture(mine)
    for k in ("row_offsets", "columns", "values", "rhs", "initial_solution", "problem", "null_space", "scaling",
              "max_iterations", "tolerance"):
        assert np.array_equal(c[k], r[k]), k
    assert np.array_equal(c["initial_solution"], x0)


def test_reference_rejects_what_the_library_rejects(ref, tmp_path):
    ro, co, va = _matrix3()
    path = tmp_path / "c.cfdxlin"
    cg.write_linear_system_capture(path, ro, co, va, np.ones(3), np.zeros(3))
    good = path.read_text()
    for bad in (good.replace("4014000000000000", "4018000000000000", 1),   # changed value
                good + "0\n",                                              # trailing data
                "\n".join(good.split("\n")[:8]) + "\n"):                   # truncated
        path.write_text(bad)
        with pytest.raises(RuntimeError):
            ref.read_capture(path)
        with pytest.raises(CfdxgError):
            cg.read_linear_system_capture(path)
