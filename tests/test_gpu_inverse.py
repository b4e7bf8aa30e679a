"""SPD inverse of single large matrices (order > 1024) against the same matrix
in a batch of two and against torch's FP64 inverse; LAPACK-numbered info for
bad pivots in either half."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _spd(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    R = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    return R @ R.T / n + 0.5 * torch.eye(n, dtype=torch.float64, device="cuda")


def _inverse(lib, A, batch):
    n = A.shape[-1]
    A = A.clone().contiguous()
    work = torch.empty(lib.cf_spd_inverse_workspace(n, batch) // 8 + 1, dtype=torch.float64, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    rc = lib.cf_spd_inverse(n, A.data_ptr(), n, n * n, batch, work.data_ptr(), info.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    return A, info


@pytest.mark.parametrize("n", [1100, 1500, 3000])
def test_large_inverse_matches_batched_and_torch(n):
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    C = _spd(n, n)
    rec, i1 = _inverse(lib, C, 1)
    blk, i2 = _inverse(lib, torch.stack([C, C]), 2)
    assert int(i1.abs().max()) == 0 and int(i2.abs().max()) == 0
    ref = torch.linalg.inv(C)
    e_rec = float((rec - ref).abs().max() / ref.abs().max())
    e_blk = float((rec - blk[0]).abs().max() / blk[0].abs().max())
    print(f"n={n}: vs torch {e_rec:.1e}, vs batch of two {e_blk:.1e}")
    assert e_rec <= 1e-11 and e_blk <= 1e-11
    assert torch.equal(rec, rec.T)


@pytest.mark.parametrize("bad", [700, 1301])
def test_large_inverse_reports_pivot(bad):
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n = 1500
    C = _spd(n, 7)
    C[bad, :] = 0.0
    C[:, bad] = 0.0
    C[bad, bad] = -1.0
    _, info = _inverse(lib, C, 1)
    assert int(info.item()) == bad + 1


def test_large_inverse_in_a_cuda_graph():
    """Above order 1024 the factorisation forks a side stream for its
    look-ahead and joins it back; the call must capture into a CUDA graph and
    replay to the eager result bit for bit."""
    from cosmoforge_b200 import _lib

    lib = _lib.lib()
    n = 1500
    C = _spd(n, 11)
    eager, _ = _inverse(lib, C, 1)
    A = C.clone()
    work = torch.empty(lib.cf_spd_inverse_workspace(n, 1) // 8 + 1, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            rc = lib.cf_spd_inverse(n, A.data_ptr(), n, n * n, 1, work.data_ptr(), info.data_ptr(), s.cuda_stream)
    assert rc == 0
    for _ in range(2):
        A.copy_(C)
        g.replay()
        torch.cuda.synchronize()
        assert int(info.item()) == 0
        assert torch.equal(A, eager)
