"""nuc3d_reconstruct_crweno5_noalloc: the CRWENO5 reconstruction for callers
that cannot let a library allocate device memory (the scratch of the line
solve lives in a fixed 4 MiB array inside the library instead of coming from
cudaMallocAsync).  Checked through the C ABI against the allocating entry
point nuc3d_reconstruct on two calls in a row, so that a second call sees
the array holding the first call's contents.  This file is collected last.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the per-operator tolerance of tests/test_gpu_ops.py


def _noalloc_fn():
    import nuc3d_b200 as nb
    fn = nb.lib().nuc3d_reconstruct_crweno5_noalloc
    fn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import nuc3d_b200 as nb
    assert torch.cuda.is_available()
    fn = _noalloc_fn()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(77)
    # second call: different shape, direction and data, so stale scratch
    # contents from the first call would show
    for (nz, ny, nx), up in (((6, 9, 40), 1), ((5, 7, 64), -1)):
        f = torch.from_numpy(rng.standard_normal((nz, ny, nx))).cuda()
        hl = torch.from_numpy(rng.standard_normal((nz, ny, 3))).cuda()
        hr = torch.from_numpy(rng.standard_normal((nz, ny, 3))).cuda()
        ref = torch.zeros((nz, ny, nx + 1), dtype=torch.float64, device="cuda")
        got = torch.full((nz, ny, nx + 1), np.nan, dtype=torch.float64, device="cuda")
        nb.reconstruct(nb.CRWENO5, up, nb.QUIRKS_REFERENCE, f, hl, hr, ref, stream)
        rc = fn(up, nx, ny, nz, f.data_ptr(), hl.data_ptr(), hr.data_ptr(), got.data_ptr(),
                stream.cuda_stream)
        assert rc == nb.OK, nb.lib().nuc3d_last_error()
        torch.cuda.synchronize()
        assert _rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    import nuc3d_b200 as nb
    fn = _noalloc_fn()
    nz, ny, nx = 64, 64, 128  # 2*nx*ny*nz = 1048576 > 524288
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    assert fn(1, nx, ny, nz, p, p, p, p, None) == nb.ERR_INVALID
    assert b"static scratch" in nb.lib().nuc3d_last_error()
    # the allocating entry point's line-length rule holds here too: nx = 4097
    # fits the scratch (2*4097 doubles) but is refused by both entry points
    assert fn(1, 4097, 1, 1, p, p, p, p, None) == nb.ERR_INVALID
    assert b"nx <= 4096" in nb.lib().nuc3d_last_error()
    assert nb.lib().nuc3d_reconstruct(nb.CRWENO5, 1, 0, 4097, 1, 1, C.c_void_p(p),
                                      C.c_void_p(p), C.c_void_p(p), C.c_void_p(p),
                                      None) == nb.ERR_INVALID
