"""Shared test setup: import paths, the `gpu` marker and oracle fixtures."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "ssm-simulators_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"
REF_DIR = ROOT / "oracle" / "_ref"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running statistical test")


@pytest.fixture(scope="session")
def oracle():
    import ssm_oracle

    ssm_oracle.build()
    return ssm_oracle


@pytest.fixture(scope="session")
def reference_cssm():
    """The reference simulators compiled by oracle/build_ref.py, if present."""
    if not (REF_DIR / "cssm").is_dir():
        pytest.skip("reference oracle build (oracle/_ref) not present")
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    try:
        import cssm.ddm_models  # noqa: F401
    except ImportError as e:  # pragma: no cover
        pytest.skip(f"reference oracle build not importable: {e}")
    import cssm

    return cssm


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
