"""Test configuration: GPU tests carry @pytest.mark.gpu; CPU runs use
-m "not gpu".  The repository root is put on sys.path so `practice_b200` and
the test-only `oracle` package import without installation."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
