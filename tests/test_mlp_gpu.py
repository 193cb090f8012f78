"""GPU: the tensor-core dense layer (csv_gemm_bf16, tcgen05 with the accumulator in tensor memory).

Compared with an fp32 product of the same bf16 inputs on the CPU; the tolerance covers fp32
accumulation in a different order (relative 1e-5 of the row's absolute sum) and one bf16 rounding
for the bf16 outputs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16(shape, rng, scale=1.0):
    import torch
    return torch.from_numpy(rng.standard_normal(shape).astype(np.float32) * scale).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (128, 16, 64), (256, 256, 128), (384, 48, 192), (128, 512, 64)])
def test_gemm_matches_fp32_reference(codec, M, N, K):
    import torch
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A, B = _bf16((M, K), rng), _bf16((N, K), rng)
    C = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    codec.gemm_bf16(A, B, C=C, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float().cpu() @ B.float().cpu().T
    scale = (A.float().abs().cpu() @ B.float().abs().cpu().T) + 1e-6
    assert torch.all((C.cpu() - ref).abs() <= 1e-5 * scale + 1e-6), float(((C.cpu() - ref).abs() / scale).max())


def test_gemm_epilogue_bias_relu_mask_and_transposed_outputs(codec):
    import torch
    rng = np.random.default_rng(5)
    M, N, K = 256, 64, 128
    A, B = _bf16((M, K), rng), _bf16((N, K), rng)
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32)).cuda()
    mask = _bf16((M, N), rng)
    C = torch.empty((M, N), device="cuda")
    Cb = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    CbT = torch.empty((N, M), dtype=torch.bfloat16, device="cuda")
    CT = torch.empty((N, M), device="cuda")
    codec.gemm_bf16(A, B, bias=bias, mask=mask, relu=True, C=C, Cb=Cb, CbT=CbT, CT=CT)
    torch.cuda.synchronize()
    ref = torch.relu(A.float().cpu() @ B.float().cpu().T + bias.cpu()) * (mask.float().cpu() > 0)
    scale = (A.float().abs().cpu() @ B.float().abs().cpu().T) + bias.abs().cpu() + 1e-6
    assert torch.all((C.cpu() - ref).abs() <= 1e-5 * scale + 1e-6)
    assert torch.equal(CT.cpu(), C.cpu().T)
    assert torch.equal(Cb.cpu(), C.cpu().to(torch.bfloat16))
    assert torch.equal(CbT.cpu(), C.cpu().T.contiguous().to(torch.bfloat16))


def test_gemm_rejects_unaligned_shapes(codec):
    import torch
    from csvb200 import CsvError
    A = torch.zeros((100, 64), dtype=torch.bfloat16, device="cuda")
    B = torch.zeros((32, 64), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(CsvError):
        codec.gemm_bf16(A, B, C=torch.empty((100, 32), device="cuda"))
