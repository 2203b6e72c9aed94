"""The replay tool (python -m cfdx_dev_b200.replay) without a GPU: usage, the
reference tool's CSR diagnosis line, and a loud failure when no device is
present (the tool has no CPU solve)."""
import numpy as np
import pytest
import torch

from cfdx_dev_b200 import replay
from tests import cases

GOLDEN = cases.ROOT / "tests" / "golden" / "pressure_tet4.cfdxlin"


def test_usage():
    assert replay.main([]) == 2


def test_diagnosis_line_of_the_golden_capture():
    import cfdx_dev_b200 as cg
    c = cg.read_linear_system_capture(GOLDEN)
    line = replay.diagnosis(c)
    assert line == f"CSR rows=384 nnz=1728 missing_diagonal=0 near_zero_diagonal=0 checksum={c['checksum']:x}"
    va = c["values"].copy()
    ro, co = c["row_offsets"], c["columns"]
    diag_k = [k for k in range(ro[2], ro[3]) if co[k] == 2][0]
    va[diag_k] = 0.0
    assert "near_zero_diagonal=1" in replay.diagnosis(dict(c, values=va))


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a GPU")
def test_fails_loudly_without_a_device(capsys):
    assert replay.main([str(GOLDEN), "auto"]) == 1
    assert "CFDX_LINEAR_REPLAY_FAIL" in capsys.readouterr().err


def test_unknown_candidate_is_refused_before_any_solve():
    with pytest.raises(ValueError, match="bogus"):
        replay.replay(GOLDEN, ["auto", "bogus"], ctx=object())
