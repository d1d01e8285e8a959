"""Input images on the CPU: the image oracle and the library's host decoder
(inflate, PNG row filters, Netpbm payloads) against the reference's own
read_png / read_pnm outputs (tests/golden/images.npz), and the error cases
the reference rejects (stereonet.py:244-324, 3421-3612)."""

import hashlib
import json
import sys

import numpy as np
import pytest

from conftest import REPO, bits, golden

sys.path.insert(0, REPO)
from oracle import image_oracle as io_orc  # noqa: E402

G = golden("images.npz")
CASES = sorted(k[:-5] for k in G.files if k.endswith("_file") and not k.startswith("err_"))
ERRORS = json.loads(str(G["err_kinds"]))


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes()).hexdigest()


def check_against_golden(name, gray, rgb, W, H):
    assert [W, H] == G[name + "_wh"].tolist()
    if name + "_gray" in G.files:
        assert np.array_equal(bits(gray), bits(G[name + "_gray"]))
        assert np.array_equal(bits(rgb), bits(G[name + "_rgb"]))
    else:
        assert _sha(gray) == str(G[name + "_gray_sha"])
        assert _sha(rgb) == str(G[name + "_rgb_sha"])


def test_fixture_coverage():
    """Every PNG colour type and depth, stored / fixed / dynamic blocks,
    all five filters and the four Netpbm formats are present."""
    assert len(CASES) >= 26 and len(ERRORS) >= 11
    assert all(v == "ValueError" for v in ERRORS.values())
    kinds = set()
    for name in CASES:
        data = G[name + "_file"].tobytes()
        if data[:8] == io_orc.PNG_SIGNATURE:
            kinds.add(("png", data[24], data[25]))
        else:
            kinds.add(("pnm", data[:2]))
    for ct, depths in ((0, (1, 2, 4, 8, 16)), (2, (8, 16)), (3, (1, 2, 4, 8)), (4, (8, 16)),
                       (6, (8, 16))):
        for d in depths:
            assert ("png", d, ct) in kinds, (d, ct)
    for m in (b"P2", b"P3", b"P5", b"P6"):
        assert ("pnm", m) in kinds


@pytest.mark.parametrize("name", CASES)
def test_oracle_vs_reference(name):
    gray, rgb, W, H = io_orc.read_image_bytes(G[name + "_file"].tobytes())
    check_against_golden(name, gray, rgb, W, H)


@pytest.mark.parametrize("name", sorted(ERRORS))
def test_oracle_rejects(name):
    with pytest.raises(ValueError):
        io_orc.read_image_bytes(G["err_" + name + "_file"].tobytes())


@pytest.mark.parametrize("name", CASES)
def test_host_decoder_vs_reference(svb, name):
    """The library's host half (no GPU): raw samples from sv_image_decode_raw,
    converted by the oracle's FP64 step, match the reference bit for bit."""
    from importlib import import_module
    image = import_module(svb.__name__ + ".image")
    raw, desc = image.decode_raw(G[name + "_file"].tobytes())
    gray, rgb = io_orc.raw_to_float(raw, desc)
    check_against_golden(name, gray, rgb, desc.width, desc.height)


@pytest.mark.parametrize("name", sorted(ERRORS))
def test_host_decoder_rejects(svb, name):
    from importlib import import_module
    image = import_module(svb.__name__ + ".image")
    with pytest.raises(ValueError):
        image.decode_raw(G["err_" + name + "_file"].tobytes())


def test_host_decoder_truncations_and_corruption(svb):
    """Cut or corrupted files either decode or raise ValueError; a file cut
    inside its pixel data is rejected."""
    from importlib import import_module
    image = import_module(svb.__name__ + ".image")
    rng = np.random.default_rng(31337)
    for name in ("rgb8_dyn", "gray8_rle", "pal4", "rgb16_fixed", "p6_8", "p2_15"):
        data = G[name + "_file"].tobytes()
        for cut in sorted(set(rng.integers(0, len(data), size=40).tolist())):
            try:
                image.decode_raw(data[:cut])
            except ValueError:
                pass
        for _ in range(60):
            b = bytearray(data)
            for _ in range(3):
                b[int(rng.integers(0, len(b)))] ^= 1 << int(rng.integers(0, 8))
            try:
                image.decode_raw(bytes(b))
            except ValueError:
                pass
    data = G["rgb8_dyn_file"].tobytes()
    with pytest.raises(ValueError):
        image.decode_raw(data[:len(data) // 2])


def test_host_decoder_large_stored_and_dynamic(svb):
    """A 640x480 RGB image (the largest input size the path is measured
    on) through stored and dynamic-Huffman streams decodes to the same
    samples the oracle's unfilter gives."""
    from importlib import import_module
    image = import_module(svb.__name__ + ".image")
    rng = np.random.default_rng(77)
    W, H = 640, 480
    yy, xx = np.mgrid[0:H, 0:W * 3]
    v = ((np.sin(xx / 9.0) + np.cos(yy / 13.0) + 2) / 4 * 255 + rng.integers(0, 4, (H, W * 3)))
    samples = np.clip(v, 0, 255).astype(int).tolist()
    for level in (0, 9):
        data, filtered = svb.synth.make_png(W, H, 8, 2, samples, (0, 1, 2, 3, 4), level)
        raw, desc = image.decode_raw(data)
        want = io_orc.unfilter(filtered, H, 3, 3 * W)
        assert np.array_equal(raw, want)
        assert np.array_equal(raw, np.array(samples, dtype=np.uint8))


def test_batch_decode_threads(svb):
    """sv_image_decode_batch on 4 threads gives each file's samples exactly
    as the single-file call does, and reports the failing file."""
    import ctypes
    from importlib import import_module
    image = import_module(svb.__name__ + ".image")
    lib = svb._lib.load()
    names = CASES + CASES
    blobs = [G[nm + "_file"].tobytes() for nm in names]
    blobs[5] = G["err_filter5_file"].tobytes()
    n = len(blobs)
    descs = (svb._lib.RawImage * n)()
    sizes = []
    for i, b in enumerate(blobs):
        assert lib.sv_image_info(b, len(b), ctypes.byref(descs[i])) == 0
        sizes.append(descs[i].stride * descs[i].height)
    raws = [np.zeros(max(s, 1), dtype=np.uint8) for s in sizes]
    st = (ctypes.c_int * n)()
    rc = lib.sv_image_decode_batch(
        n, (ctypes.c_char_p * n)(*blobs), (ctypes.c_size_t * n)(*[len(b) for b in blobs]),
        (ctypes.c_void_p * n)(*[r.ctypes.data for r in raws]), (ctypes.c_size_t * n)(*sizes),
        descs, st, 4)
    assert rc == svb._lib.SV_ERR_PARAM and list(st).count(0) == n - 1 and st[5] != 0
    assert lib.sv_last_error().decode().startswith("file 5: unknown PNG filter type 5")
    for i, b in enumerate(blobs):
        if i == 5:
            continue
        want, _ = image.decode_raw(b)
        assert np.array_equal(raws[i][:sizes[i]].reshape(want.shape), want)
