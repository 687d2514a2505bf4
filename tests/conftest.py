"""pytest configuration: the `gpu` marker and import paths for the package and the oracle."""
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent
for p in (ROOT / "arcane-benchs_b200", ROOT / "oracle", ROOT, ROOT / "tests" / "golden", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built sm_100a library")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")
