"""tcgen05 BF16 GEMM core (the engine of the learned warm start's convolutions) against torch."""

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mn_major", [0, 1])
@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (256, 32, 128), (136, 64, 72), (384, 128, 200), (128, 64, 1728)])
def test_tc_gemm_matches_torch(backend, M, N, K, mn_major):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    a = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.full((M, N), float("nan"), device="cuda")
    if mn_major:
        backend.call("clb_tc_test_gemm", a.t().contiguous(), b.t().contiguous(), c, M, N, K, 1)
    else:
        backend.call("clb_tc_test_gemm", a, b, c, M, N, K, 0)
    ref = a.float() @ b.float().t()
    torch.cuda.synchronize()
    assert backend.device_error() == 0
    torch.testing.assert_close(c, ref, rtol=1e-4, atol=1e-3 * K ** 0.5)
