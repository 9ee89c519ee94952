import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmupsi_gpu.so")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "libmupsi_oracle.so")
    srcs = [os.path.join(ROOT, "oracle", f) for f in ("mupsi_oracle.c", "mupsi_mlp_oracle.c", "mupsi_oracle.h")]
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(f) for f in srcs):
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "libmupsi_oracle.so"], check=True, env=env,
                       capture_output=True)


@pytest.fixture(scope="session")
def port():
    _ensure_oracle()
    from oracle import bind
    return bind.PortOracle()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture(scope="session")
def gpu():
    """The GPU library; the GPU tests fail (not skip) if it cannot run."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device not available for a gpu-marked test")
    from mupsi_b200 import build
    build.build()
    from mupsi_b200 import lib
    return lib.load()
