"""The denoiser's checker and host logic, without a GPU.

  * the oracle (oracle/denoise.py) against OIDN's own output on the
    reference's desk fixture (crates/denoise/tests/oidn.rs: 1e-3 x (1 + |v|)
    per channel; the reference measures 2.2e-6);
  * the product's tile split (denoise.cu, through a test hook) against the
    oracle's and the reference's own tile tests (tile.rs:98-131);
  * the product's weights parser: a valid blob is refused only for want of a
    device, a bad one with the reference's messages (tza.rs:51-118)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import denoise as D
from pfx_b200 import abi
from pfx_b200.denoise import DEFAULT_WEIGHTS, write_tza

GOLDEN = Path(__file__).parent / "golden" / "denoise_desk.npz"


def oidn_layers():
    if not DEFAULT_WEIGHTS.exists():
        pytest.skip("OIDN weights not fetched (pfx_b200/weights/fetch_oidn_weights.py)")
    return D.build_net(D.parse_tza(DEFAULT_WEIGHTS.read_bytes()))


def test_the_oracle_matches_oidn_on_the_desk():
    d = np.load(GOLDEN)
    out = D.denoise(d["color"], d["albedo"], d["normal"], oidn_layers())
    oidn = d["oidn"]
    gap = np.abs(out[..., :3] - oidn[..., :3]) / (1.0 + np.abs(oidn[..., :3]))
    assert gap.max() <= 1e-5, gap.max()
    assert np.array_equal(out[..., 3], d["color"][..., 3])


def test_the_shipped_weights_have_the_reference_layers():
    t = D.parse_tza(DEFAULT_WEIGHTS.read_bytes()) if DEFAULT_WEIGHTS.exists() else pytest.skip("no weights")
    assert t["enc_conv0.weight"].shape == (32, 9, 3, 3) and t["dec_conv0.bias"].shape == (3,)
    assert len(t) == 32
    layers = D.build_net(t)
    assert [l.out for l in layers] == [32, 32, 48, 64, 80, 96, 96, 112, 112, 96, 96, 64, 64, 64, 32, 3]


def test_halves_widen_exactly():
    # tza.rs:141-149
    bits = np.array([0x3c00, 0xc000, 0x7bff, 0x0001, 0x03ff, 0x3555, 0x7c00], np.uint16)
    v = D.half_to_float(bits)
    assert v[0] == 1.0 and v[1] == -2.0 and v[2] == 65504.0
    assert v[3] == np.float32(2.0 ** -24) and v[4] == np.float32(1023 * 2.0 ** -24)
    assert v[5] == np.float32(0.333_251_95) and np.isinf(v[6])


def product_plan(h, w, max_pixels=D.DEFAULT_MAX_TILE_PIXELS):
    lib = abi.load()
    head = np.zeros(4, np.uint32)
    tiles = np.zeros(12 * 64, np.uint32)
    abi.check(lib.pfxt_debug_denoise_plan(h, w, max_pixels, tiles.ctypes.data, 64, head.ctypes.data))
    return head, tiles[:12 * head[3]].reshape(-1, 6, 2)


def covered(tiles, h, w):
    hits = np.zeros((h, w), np.int32)
    for t in tiles:
        (oy, ox), (sh, sw) = t[4], t[5]
        hits[oy:oy + sh, ox:ox + sw] += 1
    return (hits == 1).all()


@pytest.mark.parametrize("h, w, max_pixels", [(1080, 1920, D.DEFAULT_MAX_TILE_PIXELS), (24, 32, D.DEFAULT_MAX_TILE_PIXELS),
                                              (2160, 3840, D.DEFAULT_MAX_TILE_PIXELS), (1000, 3000, 1 << 20),
                                              (777, 1333, 600_000), (5000, 4000, 2160 * 2160),
                                              (2880, 5120, 2160 * 2160), (800, 1000, 600_000)])
def test_the_tile_split_is_the_reference_split(h, w, max_pixels):
    head, tiles = product_plan(h, w, max_pixels)
    p = D.plan(h, w, max_pixels)
    assert (head[0], head[1], head[2], head[3]) == (p.tile_h, p.tile_w, p.overlap, len(p.tiles))
    for t, q in zip(tiles, p.tiles):
        assert [tuple(x) for x in t] == [q.src, q.dst, q.size, q.out_src, q.out_dst, q.out_size]
    assert covered(tiles, h, w)
    if (h, w) == (1080, 1920):
        assert (head[0], head[1], head[3]) == (1088, 1920, 1)
    if (h, w) == (2160, 3840):
        assert (head[0], head[1], head[3]) == (2160, 2016, 2)
    if (h, w) == (2880, 5120):
        assert head[3] == 4
    if max_pixels < D.DEFAULT_MAX_TILE_PIXELS or (h, w) == (5000, 4000):
        assert head[3] > 1


def random_weights(seed=0, scale=1.0, out_scale=0.1):
    """Seeded FP16 weights with the shapes of OIDN's RT network: He-scaled
    layers, and an output layer scaled by `out_scale` so that the network's
    output stays in the range a trained one gives (PU-encoded colour below
    ~1), where the inverse transfer does not amplify rounding exponentially."""
    rng = np.random.default_rng(seed)
    shapes = [("enc_conv0", 32, 9), ("enc_conv1", 32, 32), ("enc_conv2", 48, 32), ("enc_conv3", 64, 48),
              ("enc_conv4", 80, 64), ("enc_conv5a", 96, 80), ("enc_conv5b", 96, 96), ("dec_conv4a", 112, 160),
              ("dec_conv4b", 112, 112), ("dec_conv3a", 96, 160), ("dec_conv3b", 96, 96), ("dec_conv2a", 64, 128),
              ("dec_conv2b", 64, 64), ("dec_conv1a", 64, 73), ("dec_conv1b", 32, 64), ("dec_conv0", 3, 32)]
    t = {}
    for name, o, i in shapes:
        std = scale * np.sqrt(2.0 / (9 * i)) * (out_scale if name == "dec_conv0" else 1.0)
        t[f"{name}.weight"] = rng.normal(0.0, std, (o, i, 3, 3)).astype(np.float16)
        t[f"{name}.bias"] = rng.normal(0.25 if name == "dec_conv0" else 0.0, 0.02, o).astype(np.float16)
    return t


def create(blob: bytes):
    h = C.c_void_p()
    rc = abi.load().pfxt_denoiser_create(blob, len(blob), C.byref(h))
    msg = abi.load().pfxt_last_error().decode()
    if rc == abi.OK:
        abi.load().pfxt_denoiser_destroy(h)
    return rc, msg


def test_the_weights_parser_refuses_bad_blobs_with_the_reference_messages():
    good = write_tza(random_weights())
    rc, msg = create(good)
    assert rc in (abi.OK, abi.ERR_REFUSED), msg  # no GPU here: refused for want of a device only
    if rc == abi.ERR_REFUSED:
        assert "device" in msg
    assert create(good[:100]) == (abi.ERR_INVALID, "invalid or corrupted weights blob")
    assert create(b"\x00" * 64) == (abi.ERR_INVALID, "invalid or corrupted weights blob")
    bad_version = bytearray(good)
    bad_version[2] = 3
    assert create(bytes(bad_version)) == (abi.ERR_INVALID, "unsupported weights blob version")
    t = random_weights()
    t["dec_conv2b.weight"] = t["dec_conv2b.weight"][:, :60]
    rc, msg = create(write_tza(t))
    assert rc == abi.ERR_INVALID and msg == "dec_conv2b: the weights do not match the network"
    t = random_weights()
    del t["enc_conv3.bias"]
    assert create(write_tza(t)) == (abi.ERR_INVALID, "invalid or corrupted weights blob")
    t = random_weights()
    t["dec_conv0.weight"] = np.zeros((4, 32, 3, 3), np.float16)
    t["dec_conv0.bias"] = np.zeros(4, np.float16)
    assert create(write_tza(t)) == (abi.ERR_INVALID, "the network does not end in three channels")
