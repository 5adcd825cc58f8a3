import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


class Golden:
    """Reference outputs recorded by tests/golden/make_golden.py."""

    def __init__(self, name):
        self.name = name
        self.data = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
        with open(os.path.join(GOLDEN, "manifest.json")) as f:
            self.meta = json.load(f)[name]

    def __getitem__(self, k):
        return self.data[k]

    def models(self):
        from oracle.pyoracle import Models
        d = self.data
        return Models(d["gp_nz"], d["gp_nt"], d["gp_coef"], d["ring_ndisk"], d["ring_param"], d["ring_disk"])

    def config_path(self, tmpdir=None):
        """Path of the system's Config.txt: stored, or regenerated from its seed and hash-checked."""
        if self.meta["stored"]:
            return os.path.join(GOLDEN, "systems", self.name, "Config.txt")
        from ephemeris_b200 import synth
        from tests.golden.make_golden import system_hash
        d = os.path.join(str(tmpdir), self.name)
        cfg = synth.write_workload(self.meta["generator"], d, **self.meta["kwargs"])
        assert system_hash(d) == self.meta["sha256"], "regenerated system differs from the recorded one"
        return cfg


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = Golden(name)
        return cache[name]
    return get


@pytest.fixture(scope="session")
def oracle():
    from oracle.pyoracle import Oracle
    return Oracle()
