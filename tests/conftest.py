import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and libnwgpu.so")
    config.addinivalue_line("markers", "slow: larger inputs (seconds of CPU oracle time)")


@pytest.fixture(scope="session")
def karate():
    return dict(np.load(os.path.join(GOLDEN, "karate.npz")))


@pytest.fixture(scope="session")
def small_graphs():
    z = np.load(os.path.join(GOLDEN, "small_graphs.npz"))
    out = {}
    for key in z.files:
        name, field = key.split("/", 1)
        out.setdefault(name, {})[field] = z[key]
    return out


@pytest.fixture(scope="session")
def refdata():
    """The reference's own test matrices (test/data/*.mtx) as its driver loads
    them, with NWGraph's outputs: {name: {"row_ptr", "col", "deg", "v10_20", ...}}."""
    z = np.load(os.path.join(GOLDEN, "refdata.npz"))
    out = {}
    for key in z.files:
        if key == "names":
            continue
        name, field = key.split("/", 1)
        out.setdefault(name, {})[field] = z[key]
    return out


REFDATA_NAMES = [str(x) for x in np.load(os.path.join(GOLDEN, "refdata.npz"))["names"]]


@pytest.fixture(scope="session")
def csr_golden():
    """Edge lists and the reference's CSRs for each clean-up flag set:
    {name: {"src", "dst", "n", flags: {"row_ptr", "col", "deg"}}}."""
    z = np.load(os.path.join(GOLDEN, "csr_build.npz"))
    out = {}
    for key in z.files:
        parts = key.split("/")
        g = out.setdefault(parts[0], {})
        if len(parts) == 2:
            g[parts[1]] = z[key] if parts[1] != "n" else int(z[key][0])
        else:
            g.setdefault(int(parts[1]), {})[parts[2]] = z[key]
    return out


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """GPU tests fail (never skip) without a device: `-m gpu` runs on a B200."""
    if not has_gpu():
        pytest.fail("no CUDA device visible to a `gpu`-marked test")
    import nwgraph_b200._native as N
    N.lib()
    return True


@pytest.fixture
def nccl_one_rank(gpu):
    """A one-rank NCCL process group on cuda:0 (the torch.distributed code paths
    of the sharded entry points, with nothing to wait for), destroyed after the test."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    yield dist.group.WORLD
    dist.destroy_process_group()
