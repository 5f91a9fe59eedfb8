import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "maquis-dmrg_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # the oracle's OpenMP team: keep CPU tests light when many run at once
    os.environ.setdefault("ORACLE_THREADS", str(min(8, os.cpu_count() or 1)))
