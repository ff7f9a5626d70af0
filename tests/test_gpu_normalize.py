"""GPU: vp_normalize_accumulator, the replacement of the reference's one plain C-ABI kernel
launch_normalize_accumulator_kernel (device/kernels/normalize_accumulator.cu:16-35):
out[i] = accumulator[i] * normalization_factor for image_size float4 pixels, device pointers,
asynchronous on the given stream (the context's stream when it is NULL).

The product is one FP32 multiplication per component, so the result must equal numpy's float32
product bit for bit.
"""
import numpy as np
import pytest

from volprim_b200._capi import check, lib

pytestmark = pytest.mark.gpu


def _launch(ctx, out, acc, n, scale, stream):
    check(lib.vp_normalize_accumulator(ctx.handle, out.data_ptr(), acc.data_ptr(), n, float(scale), stream))


@pytest.mark.parametrize("n", [1, 255, 256, 257, 262_144, 1024 * 1024 + 3])
def test_normalize_matches_float32_product_on_context_stream(vp_ctx, n):
    import torch
    rng = np.random.default_rng(n)
    acc = rng.normal(size=(n, 4)).astype(np.float32) * 7.0
    scale = np.float32(1.0 / 3.0)
    a = torch.from_numpy(acc).cuda()
    out = torch.full_like(a, float("nan"))
    torch.cuda.synchronize()
    _launch(vp_ctx, out, a, n, scale, None)  # NULL stream: the context's stream
    vp_ctx.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), (acc * scale).view(np.uint32))


def test_normalize_on_caller_stream(vp_ctx):
    import torch
    n = 500_000
    rng = np.random.default_rng(7)
    acc = rng.uniform(0, 100, size=(n, 4)).astype(np.float32)
    a = torch.from_numpy(acc).cuda()
    out = torch.empty_like(a)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        _launch(vp_ctx, out, a, n, np.float32(0.0625), s.cuda_stream)
    s.synchronize()
    assert np.array_equal(out.cpu().numpy(), acc * np.float32(0.0625))


def test_normalize_empty_and_null(vp_ctx):
    import torch
    a = torch.zeros(4, 4, device="cuda")
    _launch(vp_ctx, a, a, 0, 2.0, None)  # nothing to do
    vp_ctx.synchronize()
    assert lib.vp_normalize_accumulator(vp_ctx.handle, None, a.data_ptr(), 4, 1.0, None) != 0
