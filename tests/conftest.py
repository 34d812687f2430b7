import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device and the built library")


def load_case(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        c = {k: z[k] for k in z.files}
    for k in ("nz", "nx", "nabc", "nt"):
        c[k] = int(c[k])
    for k in ("dt", "dx", "f0"):
        c[k] = float(c[k])
    c["free_surface"] = bool(c["free_surface"])
    if "src_v" not in c:
        c["src_v"] = np.tile(c["wavelet"], (len(c["src_x"]), 1)).astype(np.float32)
    return c


def oracle_kwargs(c: dict) -> dict:
    return dict(nz=c["nz"], nx=c["nx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
                free_surface=c["free_surface"], src_x=c["src_x"], src_z=c["src_z"], src_v=c["src_v"],
                rcv_x=c["rcv_x"], rcv_z=c["rcv_z"], damp=c["damp"], vp=c["vp"], rho=c["rho"])


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is present")
    from geobrain_b200 import build
    build.build()
    return torch.device("cuda:0")
