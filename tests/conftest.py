import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

GOLDEN = REPO / "tests" / "golden" / "reference_fixtures.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    z = np.load(GOLDEN)
    out = {}
    for name in z["names"]:
        name = str(name)
        n, b, seed, mode = (int(x) for x in z[f"{name}/meta"])
        rec = dict(n=n, batch=b, seed=seed, mode="nearid" if mode else "random",
                   sha_H=z[f"{name}/sha_H"].tobytes(), sha_S=z[f"{name}/sha_S"].tobytes(), W=z[f"{name}/W"])
        if f"{name}/U2" in z.files:
            rec["U2"] = z[f"{name}/U2"]
        out[name] = rec
    return out


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sunny_gen_eigensolver_b200 import _native
    _native.load()          # raises when the library is missing: no fallback
    return torch.device("cuda:0")
