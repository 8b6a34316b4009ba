import functools
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@functools.lru_cache(maxsize=None)
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


@functools.lru_cache(maxsize=None)
def system(name: str, **kw):
    from miniafqmc_b200.synthetic import CONFIGS, make_system
    import dataclasses
    cfg = dataclasses.replace(CONFIGS[name], **kw) if kw else CONFIGS[name]
    return make_system(cfg)


@functools.lru_cache(maxsize=None)
def tiny_system(complex_trial: bool = True, complex_chol: bool = True, nmo: int = 12,
                nel: int = 3, nchol: int = 20, density: float = 0.3, seed: int = 7):
    from miniafqmc_b200.synthetic import Config, make_system
    cfg = Config(nmo, nel, nchol, density, seed, dt=0.01, nwalk=4, complex_trial=complex_trial,
                 complex_chol=complex_chol)
    return make_system(cfg)
