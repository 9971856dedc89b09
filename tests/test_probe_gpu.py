"""The random-gather ceiling probe (nwgraph_b200/libnwprobe.so) that bench.py
reports beside the HBM roofline: it runs, gives a plausible B200 rate, and
rejects bad arguments."""
import ctypes as C
import os

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gather_probe(gpu):
    import torch
    torch.cuda.init()
    lib = C.CDLL(os.path.join(ROOT, "nwgraph_b200", "libnwprobe.so"))
    rate, ms = C.c_double(), C.c_double()
    assert lib.nwprobe_gather_rate(C.c_uint32(24), C.c_uint32(64), C.c_uint32(3), C.byref(rate), C.byref(ms)) == 0
    assert 20e9 < rate.value < 5e12 and ms.value > 0
    assert lib.nwprobe_gather_rate(C.c_uint32(40), C.c_uint32(64), C.c_uint32(3), C.byref(rate), C.byref(ms)) != 0
    assert lib.nwprobe_gather_rate(C.c_uint32(24), C.c_uint32(0), C.c_uint32(3), C.byref(rate), C.byref(ms)) != 0
