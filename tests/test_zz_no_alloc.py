"""The allocation-free operator entry point (hx_apply_stiffness_noalloc).

It serves callers that cannot let the library allocate device memory
(cudaMalloc/cudaFree synchronize the device; a pooling host runtime such as
CUDA.jl may hold most of it).  The test owns the input and output buffers;
the entry point itself uses only its static scratch array.  Its results are
compared with hx_apply_stiffness on two calls in a row (different grids, so
the shared scratch is reused), at the 1e-12 relative tolerance of the other
operator tests.  This file is collected last so that a failure here does not
hide the other GPU tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(hx, dims, x, fac):
    import torch
    L = hx.load()
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    fd = torch.from_numpy(fac).to(dev)
    yd = torch.empty_like(xd)
    sd = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = L.hx_apply_stiffness_noalloc(*dims, 1.0, 1.0, 1.0, 0.3, xd.data_ptr(), fd.data_ptr(),
                                      yd.data_ptr(), sd.data_ptr(),
                                      ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize(dev)
    return st, yd.cpu().numpy(), float(sd.item())


@pytest.mark.parametrize("calls", [[(13, 7, 5), (40, 9, 17)]])
def test_noalloc_matches_apply_stiffness(hx, calls):
    rng = np.random.default_rng(2024)
    for dims in calls:  # two calls in a row on different grids
        nn = (dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1)
        x = rng.standard_normal(3 * nn)
        fac = rng.uniform(0.0, 1.0, dims[0] * dims[1] * dims[2])
        st, y, xkx = _noalloc(hx, dims, x, fac)
        assert st == 0
        with hx.Context(0) as ctx:
            ctx.set_grid(*dims)
            ctx.set_material(1.0, 0.3)
            yref = ctx.apply_stiffness(x, fac)
        assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
        want = float(np.dot(x, yref))
        assert abs(xkx - want) <= 1e-12 * abs(want)


def test_noalloc_rejects_oversized_grid(hx):
    x = np.zeros(3 * 8)
    fac = np.zeros(1)
    import torch
    L = hx.load()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    # ~3226 x 1429 CTA columns: far beyond HX_NOALLOC_MAX_BLOCKS; rejected
    # before any launch, so the small buffers are never touched
    st = L.hx_apply_stiffness_noalloc(100000, 10000, 1, 1.0, 1.0, 1.0, 0.3, buf.data_ptr(),
                                      buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert st == 6  # HX_BAD_ARG
    # a misaligned array is refused before any launch (it would otherwise be a
    # misaligned-address fault in the caller's context): x needs 16 bytes,
    # the others 8
    p = buf.data_ptr()
    assert p % 16 == 0
    for k, off in ((0, 8), (1, 4), (2, 4), (3, 4)):
        args = [p, p + 32, p + 64, p + 96]
        args[k] += off
        st = L.hx_apply_stiffness_noalloc(1, 1, 1, 1.0, 1.0, 1.0, 0.3, *args, None)
        assert st == 6, k
    del x, fac
