"""Target smoothing and the loss reductions against FP64 references."""
import numpy as np
import pytest
import torch

from deepcharacters_b200.losses import image_l1_loss, smooth_image, sum_squares_loss

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def smooth_fp64(img, size, mean, std):
    """Depthwise 'SAME' convolution with the normalised outer product of the
    sampled normal density (GaussianSmoothingGpu.py:20-33), FP64."""
    x = np.asarray(img, np.float64)
    k = np.arange(-size, size + 1, dtype=np.float64)
    v = np.exp(-0.5 * ((k - mean) / std) ** 2)
    K2 = np.outer(v, v)
    K2 /= K2.sum()
    H, W = x.shape[-3], x.shape[-2]
    pad = np.zeros(x.shape[:-3] + (H + 2 * size, W + 2 * size, x.shape[-1]))
    pad[..., size:size + H, size:size + W, :] = x
    out = np.zeros_like(x)
    for j in range(2 * size + 1):
        for i in range(2 * size + 1):
            out += K2[j, i] * pad[..., j:j + H, i:i + W, :]
    return out


@pytest.mark.parametrize("size,mean,std", [(1, 0.0, 1.0), (3, 0.0, 1.5), (7, 0.3, 2.0), (15, 0.0, 4.0)])
def test_smooth_matches_fp64(size, mean, std):
    rng = np.random.default_rng(size)
    img = rng.uniform(0, 1, size=(2, 3, 45, 70, 3)).astype(np.float32)
    ours = smooth_image(torch.from_numpy(img).to(DEV), size, mean, std).cpu().numpy()
    ref = smooth_fp64(img, size, mean, std)
    assert np.abs(ours - ref).max() < 2e-6


def test_smooth_identity_cases():
    x = torch.rand((1, 2, 8, 9, 3), device=DEV)
    assert smooth_image(x, 0, 0.0, 1.0) is x and smooth_image(x, 2, 0.0, 0.0) is x


def test_l1_and_sum_squares():
    rng = np.random.default_rng(4)
    r = rng.uniform(0, 1, size=(2, 3, 16, 16, 3)).astype(np.float32)
    t = rng.uniform(0, 1, size=r.shape).astype(np.float32)
    face = rng.integers(-1, 5, size=r.shape[:-1]).astype(np.int32)
    loss, grad = image_l1_loss(torch.from_numpy(r).to(DEV), torch.from_numpy(t).to(DEV), torch.from_numpy(face).to(DEV))
    m = (face >= 0)[..., None]
    d = 255.0 * (r.astype(np.float64) - t) * m
    cnt = np.count_nonzero(d)
    assert abs(float(loss) - np.abs(d).sum() / cnt) < 1e-4 * np.abs(d).sum() / cnt
    assert np.allclose(grad.cpu().numpy(), 255.0 * np.sign(d) / cnt, rtol=1e-6, atol=1e-9)
    x = rng.normal(size=(1000,)).astype(np.float32)
    l2, g2 = sum_squares_loss(torch.from_numpy(x).to(DEV), 0.5)
    assert abs(float(l2) - 0.5 * (x.astype(np.float64) ** 2).sum()) < 1e-5 * (x.astype(np.float64) ** 2).sum()
    assert torch.allclose(g2.cpu(), torch.from_numpy(x), rtol=1e-6)


def test_u8_images_widen_to_the_host_values():
    """hc_image_u8_to_f32 gives byte / 255 exactly as float32 division on the
    host does (every byte value; a length that is not a multiple of 4)."""
    from deepcharacters_b200 import _lib
    rng = np.random.default_rng(4)
    for n in (256, 1000003):
        src = np.arange(n, dtype=np.int64) % 256 if n == 256 else rng.integers(0, 256, n)
        src = src.astype(np.uint8)
        s = torch.from_numpy(src).to(DEV)
        d = torch.empty(n, dtype=torch.float32, device=DEV)
        _lib.call("hc_image_u8_to_f32", torch.cuda.current_stream().cuda_stream, n, s.data_ptr(), d.data_ptr())
        want = src.astype(np.float32) / np.float32(255.0)
        assert np.array_equal(d.cpu().numpy(), want)
