import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def small_case():
    """A jittered cylinder (~3.6k nodes) with its oracle FEM matrices."""
    from dogpup_b200.meshgen import cylinder_mesh
    from oracle.fem import gen_fwdmat, prepare_mesh
    m = cylinder_mesh(12, 20, 1.5, jitter=0.2, seed=3)
    geo = prepare_mesh(m.node, m.elem, 1.4)
    rng = np.random.default_rng(11)
    mua = 0.01 * (1 + 0.2 * rng.standard_normal(m.nn))
    musp = np.full(m.nn, 1.0)
    K, M = gen_fwdmat(m.node, m.elem, geo, mua, musp)
    return dict(mesh=m, geo=geo, mua=mua, musp=musp, K=K, M=M)
