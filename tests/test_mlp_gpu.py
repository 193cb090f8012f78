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


@pytest.mark.parametrize("count", [1, 200, 128 * 148 + 77, 70000])
def test_fused_forward_equals_layer_by_layer_gemms(codec, count):
    """csv_mlp_forward runs the whole network in one persistent kernel (activations stay in tensor memory and
    shared memory, the 256 x 256 weight streams through a two-slot ring).  It issues the MMAs of the three
    layer GEMMs in the same shapes and K order, so its logits equal, bit for bit, those of three csv_gemm_bf16
    launches with the same bf16 rounding points; its choice is the argmax of each head (ties: the lower
    index).  Counts cover one partial tile, more tiles than SMs, and several tiles per CTA."""
    import torch
    from csvb200 import SelectorNet
    p = SelectorNet.init_params(5)
    p[256 * 64:256 * 64 + 256] = np.random.default_rng(1).normal(0, 0.1, 256)  # non-zero b1
    net = SelectorNet(codec, p)
    g = torch.Generator(device="cuda")
    g.manual_seed(count)
    feat = torch.rand((count, 32), device="cuda", generator=g)
    logits = torch.empty((count, 32), device="cuda")
    sel = torch.empty(count, dtype=torch.uint8, device="cuda")
    net.forward(feat, d_logits=logits, d_sel=sel)
    # the layer-by-layer reference on the same tensor cores
    rows = (count + 127) // 128 * 128
    P = torch.from_numpy(p).cuda()
    o = 0
    W1 = P[o:o + 256 * 64].view(256, 64).to(torch.bfloat16).contiguous(); o += 256 * 64
    b1 = P[o:o + 256].contiguous(); o += 256
    W2 = P[o:o + 256 * 256].view(256, 256).to(torch.bfloat16).contiguous(); o += 256 * 256
    b2 = P[o:o + 256].contiguous(); o += 256
    W3 = P[o:o + 32 * 256].view(32, 256).to(torch.bfloat16).contiguous(); o += 32 * 256
    b3 = P[o:o + 32].contiguous()
    X = torch.zeros((rows, 64), dtype=torch.bfloat16, device="cuda")
    X[:count, :32] = feat.to(torch.bfloat16)
    H1 = torch.empty((rows, 256), dtype=torch.bfloat16, device="cuda")
    H2 = torch.empty((rows, 256), dtype=torch.bfloat16, device="cuda")
    Z = torch.empty((rows, 32), dtype=torch.float32, device="cuda")
    codec.gemm_bf16(X, W1, bias=b1, relu=True, Cb=H1)
    codec.gemm_bf16(H1, W2, bias=b2, relu=True, Cb=H2)
    codec.gemm_bf16(H2, W3, bias=b3, C=Z)
    torch.cuda.synchronize()
    assert torch.equal(logits, Z[:count])
    zm, zt = Z[:count, :12], Z[:count, 12:28]
    ref_sel = (torch.argmax(zm, 1) | (torch.argmax(zt, 1) << 4)).to(torch.uint8)
    # torch.argmax returns the first maximal index, as the kernel's strict comparison does
    assert torch.equal(sel, ref_sel)
    assert net.status() == 0
    net.close()
