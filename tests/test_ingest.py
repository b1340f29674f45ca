"""Colour ingest (Image::from_file's load_grayscale + gaussian_blur_5x5,
src/image.rs:450-534): the oracle's restatement pinned against OpenCV's
5 x 5 Gaussian blur (the reference documents its blur as matching
cv2.GaussianBlur(ksize=(5, 5), sigmaX=1.1), BORDER_REFLECT_101), and the
device ingest against the oracle, bit for bit.
"""
import numpy as np
import pytest


def _rgb(h, w, seed=3):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    # smooth structure plus noise, and saturated corners to exercise the clamp
    y, x = np.mgrid[0:h, 0:w]
    ramp = ((np.sin(x / 7.0) + np.cos(y / 5.0)) * 60 + 128).astype(np.int32)
    img = np.clip(base.astype(np.int32) // 3 + ramp[..., None], 0, 255).astype(np.uint8)
    img[:2, :2] = 255
    img[-2:, -2:] = 0
    return img


def test_grey_level_formula(oracle):
    rgb = np.array([[[255, 0, 0], [0, 255, 0], [0, 0, 255]], [[10, 20, 30], [255, 255, 255], [1, 2, 3]],
                    [[7, 7, 7], [100, 150, 200], [0, 0, 0]]], np.uint8)
    # a constant image is unchanged by the blur: check the grey formula on constant 3 x 3 images
    for r, g, b in rgb.reshape(-1, 3):
        img = np.broadcast_to(np.array([r, g, b], np.uint8), (5, 6, 3)).copy()
        want = (2126 * int(r) + 7152 * int(g) + 722 * int(b) + 5000) // 10000
        assert np.all(oracle.ingest_rgb8(img) == want)


def test_blur_matches_opencv(oracle):
    cv2 = pytest.importorskip("cv2")
    grey = np.random.default_rng(5).integers(0, 256, (61, 77), dtype=np.uint8)
    rgb = np.repeat(grey[..., None], 3, axis=2)  # R = G = B: the grey formula returns the level itself
    ours = oracle.ingest_rgb8(rgb)
    # OpenCV's floating-point blur, rounded: identical
    ref = cv2.GaussianBlur(grey.astype(np.float64), ksize=(5, 5), sigmaX=1.1, sigmaY=1.1)
    assert np.array_equal(ours, np.clip(np.round(ref), 0, 255).astype(np.uint8))
    # its 8-bit path works in fixed point: within one grey level
    ref8 = cv2.GaussianBlur(grey, ksize=(5, 5), sigmaX=1.1, sigmaY=1.1)
    assert np.abs(ours.astype(int) - ref8.astype(int)).max() <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(3, 3), (37, 53), (257, 300), (1024, 768)])
def test_device_ingest_equals_oracle(gpv_mod, oracle, shape):
    rgb = _rgb(*shape)
    img = gpv_mod.Image(image_rgb=rgb, border=20)
    grey = img.image_gs.astype(np.uint8)
    assert np.array_equal(grey, oracle.ingest_rgb8(rgb))
    # and the coefficients are those of the grey image
    ref = gpv_mod.Image(image_gs=grey, border=20)
    assert np.array_equal(img.coef(), ref.coef())
    img.update_rgb(rgb[::-1].copy())
    assert np.array_equal(img.image_gs.astype(np.uint8), oracle.ingest_rgb8(rgb[::-1].copy()))


@pytest.mark.gpu
def test_ingest_rejects_tiny_images(gpv_mod):
    with pytest.raises(gpv_mod.GpvError, match="3 x 3"):
        gpv_mod.Image(image_rgb=np.zeros((2, 5, 3), np.uint8))
