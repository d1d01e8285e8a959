"""read_png / read_pnm / read_image on the GPU (stereonet.py:265-324,
3499-3612): host decode, raw samples to the device, FP64 gray and RGB
formed by k_raw_to_float -- bit-identical to the reference's outputs
(tests/golden/images.npz) in every output container."""

import numpy as np
import pytest
import torch

from conftest import bits, golden
from test_image import CASES, ERRORS, check_against_golden

pytestmark = pytest.mark.gpu

G = golden("images.npz")


@pytest.fixture(scope="module")
def image(svb):
    from importlib import import_module
    return import_module(svb.__name__ + ".image")


@pytest.mark.parametrize("name", CASES)
def test_read_image_matches_reference(image, tmp_path, name):
    data = G[name + "_file"].tobytes()
    path = tmp_path / name
    path.write_bytes(data)
    reader = image.read_png if data[:8] == image.PNG_SIGNATURE else image.read_pnm
    for fn in (reader, image.read_image):
        g, c, W, H = fn(str(path))
        assert isinstance(g, list) and isinstance(c, list)
        check_against_golden(name, g, c, W, H)
    g, c, W, H = image.read_image(str(path), out="cuda")
    assert g.is_cuda and c.is_cuda and g.dtype == torch.float64
    check_against_golden(name, g.cpu().numpy(), c.cpu().numpy(), W, H)
    g, c, W, H = image.decode_image(data, out="numpy")
    check_against_golden(name, g, c, W, H)


@pytest.mark.parametrize("name", sorted(ERRORS))
def test_rejects_what_the_reference_rejects(image, tmp_path, name):
    path = tmp_path / name
    path.write_bytes(G["err_" + name + "_file"].tobytes())
    with pytest.raises(ValueError):
        image.read_image(str(path))


def test_wrong_reader_raises(image, tmp_path):
    png = tmp_path / "a.png"
    png.write_bytes(G["rgb8_dyn_file"].tobytes())
    pgm = tmp_path / "a.pgm"
    pgm.write_bytes(G["p5_8_file"].tobytes())
    with pytest.raises(ValueError):
        image.read_pnm(str(png))
    with pytest.raises(ValueError):
        image.read_png(str(pgm))


def test_feeds_the_device_path(svb, image, tmp_path):
    """Decoded CUDA tensors go straight into the disparity path: a pair
    read from PNG files as device tensors gives the same refine_fullres
    output as the same files read as the reference's lists."""
    from importlib import import_module
    refine = import_module(svb.__name__ + ".refine")
    pair = svb.synth.make_pair(4242, 96, 64, 2.0, 12.0)
    files = []
    for k, view in enumerate((pair.left, pair.right)):
        data, _ = svb.synth.make_png(96, 64, 8, 0, view.astype(int).tolist(), (0, 1, 2, 3, 4), 9)
        p = tmp_path / ("v%d.png" % k)
        p.write_bytes(data)
        files.append(str(p))
    lg, _, W, H = image.read_image(files[0], out="cuda")
    rg, _, _, _ = image.read_image(files[1], out="cuda")
    ll, _, _, _ = image.read_image(files[0])
    rl, _, _, _ = image.read_image(files[1])
    d0 = np.round(pair.disp.reshape(-1))
    a = refine.refine_fullres(lg, rg, torch.tensor(d0, device="cuda"), W, H)
    b = refine.refine_fullres(ll, rl, d0.tolist(), W, H)
    assert a.is_cuda and isinstance(b, list)
    assert np.array_equal(bits(a.cpu().numpy()), bits(b))


def test_read_images_batch(image, tmp_path):
    paths = []
    for nm in CASES:
        p = tmp_path / nm
        p.write_bytes(G[nm + "_file"].tobytes())
        paths.append(str(p))
    for out in ("list", "numpy", "cuda"):
        res = image.read_images(paths, out=out, threads=3)
        for nm, (g, c, W, H) in zip(CASES, res):
            if out == "cuda":
                g, c = g.cpu().numpy(), c.cpu().numpy()
            check_against_golden(nm, g, c, W, H)
