"""Shared pytest setup.

* registers the ``gpu`` marker (tests that need a B200);
* makes the in-tree library, the plain-C oracle and the reference build
  available, building them when their sources are present and the binaries
  are not (the reference build only where the reference tree exists).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# the reference source tree (read only); override with CFDX_REFERENCE_ROOT
REF_SRC = Path(os.environ.get("CFDX_REFERENCE_ROOT", "/root/reference"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    lib = ROOT / "cfdx_dev_b200" / "_lib" / "libcfdxg.so"
    if not lib.exists():
        from cfdx_dev_b200 import build as b
        b.build()
    ref_lib = ROOT / "oracle" / "_ref" / "libcfdx_ref.so"
    demo = ROOT / "oracle" / "_ref" / "cfdx_adapter_demo"
    if (not ref_lib.exists() or not demo.exists()) and REF_SRC.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", "oracle", "adapter", f"REF_ROOT={REF_SRC}"],
                       check=True)
    c_lib = ROOT / "oracle" / "_build" / "libcfdx_oracle.so"
    if not c_lib.exists() and (ROOT / "oracle" / "cfdx_oracle.c").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def ctx():
    from cfdx_dev_b200 import Context
    c = Context(int(os.environ.get("CFDXG_TEST_DEVICE", "0")))
    yield c
    c.close()


@pytest.fixture(scope="session")
def oracle():
    """The plain-C restatement (oracle/cfdx_oracle.c), built with gcc on first use."""
    from oracle import cfdx_oracle as co
    co.lib()
    return co


@pytest.fixture(scope="session")
def ref():
    from oracle import ref as r
    if not r.available():
        pytest.skip("reference oracle library not built")
    return r
