import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from jax_fluid_sim_b200.meshgen import MeshSource  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"
GOLDEN_CASES = ["smoke_p1", "smoke_p2", "smoke_p3", "box_p2", "box_p3", "mixed_p2", "species_p2", "curved_p2"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")


_cache = {}


def load_golden(case):
    if case not in _cache:
        with np.load(GOLDEN / f"{case}.npz", allow_pickle=False) as z:
            data = {k: z[k] for k in z.files}
        data["source"] = MeshSource.from_arrays(data)
        data["block_names"] = [str(n) for n in data["block_names"]]
        _cache[case] = data
    return _cache[case]


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="needs a CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def native_library():
    """Plan set-up calls the host routines of libdgb200.so (no GPU needed): build the library once
    when it is missing (nvcc cross-compiles for sm_100a without a GPU).  An existing library is
    used as it is."""
    from jax_fluid_sim_b200 import build
    if not build.LIB.exists():
        build.build()
    yield
