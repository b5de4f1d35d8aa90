"""sph_cell_offsets_static -- the cell-offset scan with its scratch in a
fixed device array -- against the cell offsets the handle API builds in a
step (sph_get_sort), called twice in a row through the C ABI."""
import ctypes as C

import numpy
import pytest
import torch

from sphere_b200 import _abi, scenes
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

EMPTY = 0xFFFFFFFF
SCAN_STATIC_MAX = 16777216     # SPH_SCAN_STATIC_MAX
UNSUPPORTED = 8                # SPH_ERR_UNSUPPORTED


def _static_scan(lib, counts, dev):
    d_counts = torch.from_numpy(counts.view(numpy.int32)).to(dev)
    d_off = torch.full((counts.size + 1,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = lib.sph_cell_offsets_static(C.c_void_p(d_counts.data_ptr()), counts.size,
                                     C.c_void_p(d_off.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    torch.cuda.synchronize(dev)
    return d_off.cpu().numpy().view(numpy.uint32)


def test_static_scan_matches_the_step_cell_offsets_twice():
    s = scenes.gravity_settling(n=10000, seed=3)
    st = Stepper([s], device=0)
    st.upload()
    st.step(1)
    _, _, cs, ce = st.sort_products()
    st.close()
    assert cs.size > 4096          # several scan tiles
    full = cs != EMPTY
    counts = numpy.where(full, ce - cs, 0).astype(numpy.uint32)
    lib = _abi.load_library()
    dev = torch.device("cuda", 0)
    for _ in range(2):
        off = _static_scan(lib, counts, dev)
        assert numpy.array_equal(off[:-1][full], cs[full])
        assert numpy.array_equal(off[1:][full], ce[full])
        assert int(off[-1]) == int(s.np[0])


def test_static_scan_large_random_counts_twice():
    rng = numpy.random.default_rng(11)
    counts = rng.integers(0, 9, SCAN_STATIC_MAX - 12345).astype(numpy.uint32)
    want = numpy.zeros(counts.size + 1, dtype=numpy.uint64)
    numpy.cumsum(counts, out=want[1:])
    lib = _abi.load_library()
    dev = torch.device("cuda", 0)
    for _ in range(2):
        off = _static_scan(lib, counts, dev)
        assert numpy.array_equal(off.astype(numpy.uint64), want)


def test_static_scan_rejects_sizes_beyond_its_scratch():
    # buffers sized for the n + 1 words the call would touch, so that the
    # call stays inside them even if the size check were wrong
    lib = _abi.load_library()
    dev = torch.device("cuda", 0)
    n = SCAN_STATIC_MAX + 1
    d_counts = torch.zeros(n, dtype=torch.int32, device=dev)
    d_off = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    rc = lib.sph_cell_offsets_static(C.c_void_p(d_counts.data_ptr()), n,
                                     C.c_void_p(d_off.data_ptr()), None)
    assert rc == UNSUPPORTED
    torch.cuda.synchronize(dev)
    assert int(d_off.abs().sum().item()) == 0   # nothing written


def test_static_scan_warm_call_allocates_no_device_memory():
    """After a first call, a call on 16 million counts leaves the device's
    free memory unchanged (the caller's buffers are made beforehand)."""
    lib = _abi.load_library()
    dev = torch.device("cuda", 0)
    counts = numpy.ones(SCAN_STATIC_MAX, dtype=numpy.uint32)
    d_counts = torch.from_numpy(counts.view(numpy.int32)).to(dev)
    d_off = torch.empty(counts.size + 1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def call():
        rc = lib.sph_cell_offsets_static(C.c_void_p(d_counts.data_ptr()), counts.size,
                                         C.c_void_p(d_off.data_ptr()),
                                         C.c_void_p(stream.cuda_stream))
        assert rc == 0, rc
        torch.cuda.synchronize(dev)

    call()
    free0, _ = torch.cuda.mem_get_info(dev)
    call()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert int(d_off[-1].item()) == SCAN_STATIC_MAX

