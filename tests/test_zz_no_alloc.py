"""Allocation-free SPD inverse (cf_spd_inverse_static) against cf_spd_inverse.

Some callers of this library must not allocate device memory at the point
where they need an inverse: an allocator hook, or a plugin whose host
application owns the memory pool and forbids new allocations after start-up.
``cf_spd_inverse_static`` serves them from a fixed scratch array compiled into
the library.  This test calls it through the C ABI twice in a row (different
sizes, so the second call runs on the stale scratch contents of the first) and
once more at the first size, and compares each result with the
workspace-taking ``cf_spd_inverse`` on the same matrix, at the 1e-12 tolerance
used for the FP64 inverse.  After a warm-up call it checks that a call leaves
the device's free memory unchanged, and that sizes above the stated maximum
are refused.

The file name sorts last so that a ``-x`` run reaches it after every other test.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _spd(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    return A @ A.T / n + np.diag(rng.uniform(0.5, 2.0, n))


def _inverse_with_workspace(lib, M):
    n = M.shape[0]
    A = torch.from_numpy(M).cuda()
    work = torch.empty(lib.cf_spd_inverse_workspace(n, 1) // 8 + 1, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.cf_spd_inverse(n, A.data_ptr(), n, n * n, 1, work.data_ptr(), info.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    return A.cpu().numpy()


def _inverse_static(lib, M):
    n = M.shape[0]
    A = torch.from_numpy(M).cuda()
    info = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    rc = lib.cf_spd_inverse_static(n, A.data_ptr(), n, info.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    return A.cpu().numpy()


def test_static_scratch_inverse_matches_workspace_inverse():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    for n, seed in ((768, 1), (300, 2), (768, 3)):
        M = _spd(n, seed)
        ref = _inverse_with_workspace(lib, M)
        got = _inverse_static(lib, M)
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= 1e-12
        assert np.allclose(got @ M, np.eye(n), atol=1e-9)


def test_static_scratch_rejects_oversized_problems():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    nmax = lib.cf_spd_inverse_static_max_n()
    assert nmax >= 1024
    A = torch.zeros(1, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.cf_spd_inverse_static(nmax + 1, A.data_ptr(), nmax + 1, info.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.CF_ERR_TOO_LARGE


def test_static_scratch_inverse_allocates_nothing():
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n = 512
    M = _spd(n, 4)
    A = torch.from_numpy(M).cuda()
    A0 = A.clone()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    # warm-up: module load, scratch address look-up, kernel attributes
    assert lib.cf_spd_inverse_static(n, A.data_ptr(), n, info.data_ptr(), st) == 0
    torch.cuda.synchronize()
    A.copy_(A0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert lib.cf_spd_inverse_static(n, A.data_ptr(), n, info.data_ptr(), st) == 0
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0
    assert int(info.item()) == 0
    assert np.allclose(A.cpu().numpy() @ M, np.eye(n), atol=1e-9)
