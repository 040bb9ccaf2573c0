"""Test configuration: import paths, the `gpu` marker, and the built libraries."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "threejs-fire-pro_b200", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import fp_oracle

    fp_oracle.build()
    return fp_oracle.lib()


@pytest.fixture(scope="session")
def cuda_lib_path():
    import importlib.util

    spec = importlib.util.spec_from_file_location("fp_build", ROOT / "threejs-fire-pro_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()
