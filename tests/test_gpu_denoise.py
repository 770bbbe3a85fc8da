"""The denoiser on the GPU (pfx_b200/csrc/denoise.cu) against OIDN's output
and the oracle (oracle/denoise.py).

  * OIDN's weights on the reference's desk fixture: within 1e-3 x (1 + |v|)
    of OIDN 2.5.1's own output, the bar of crates/denoise/tests/oidn.rs;
  * seeded random FP16 weights on ragged sizes, on a frame split into tiles,
    and on colour with NaN and infinite values: within TOL x (1 + |v|) of
    the oracle's FP64 network.  The tensor cores sum the FP16 products in
    their FP32 accumulator with their own rounding, ~1e-5 relative on a
    layer's output; the inverse transfer function multiplies an error of the
    network's output by up to ~15 (its exponential branch);
  * a tracer's films through pfxt_denoise_trace equal the host path on the
    same films; two runs are equal bit for bit;
  * a convolution whose bounded wait runs out fails the call with
    PFXT_ERR_DEVICE and leaves the denoiser usable (no GPU fault)."""
import numpy as np
import pytest

from oracle import denoise as D
from pfx_b200 import abi
from pfx_b200.denoise import DEFAULT_WEIGHTS, Denoiser, write_tza

from test_denoise_oracle import GOLDEN, random_weights

pytestmark = pytest.mark.gpu
TOL = 2e-4


def gap(a, b):
    return float((np.abs(a[..., :3].astype(np.float64) - b[..., :3]) / (1.0 + np.abs(b[..., :3]))).max())


def images(h, w, seed):
    rng = np.random.default_rng(seed)
    color = np.ones((h, w, 4), np.float32)
    color[..., :3] = rng.gamma(1.5, 0.4, (h, w, 3))
    color[..., 3] = rng.uniform(0.0, 1.0, (h, w))
    albedo = np.ones((h, w, 4), np.float32)
    albedo[..., :3] = rng.uniform(0.05, 0.95, (h, w, 3))
    n = rng.normal(size=(h, w, 3))
    normal = np.zeros((h, w, 4), np.float32)
    normal[..., :3] = n / np.linalg.norm(n, axis=2, keepdims=True)
    return color, albedo, normal


def test_the_oidn_weights_match_oidn_on_the_desk(gpu):
    if not DEFAULT_WEIGHTS.exists():
        pytest.skip("OIDN weights not fetched (pfx_b200/weights/fetch_oidn_weights.py)")
    d = np.load(GOLDEN)
    den = Denoiser()
    out = den.denoise(d["color"], d["albedo"], d["normal"])
    assert gap(out, d["oidn"]) <= 1e-3
    layers = D.build_net(D.parse_tza(DEFAULT_WEIGHTS.read_bytes()))
    assert gap(out, D.denoise(d["color"], d["albedo"], d["normal"], layers)) <= TOL
    assert np.array_equal(out[..., 3], d["color"][..., 3])
    assert den.tiles() == (32, 32, 1)
    again = den.denoise(d["color"], d["albedo"], d["normal"])
    assert np.array_equal(again.view(np.uint32), out.view(np.uint32))
    print(f"desk: worst gap to OIDN {gap(out, d['oidn']):.2e}")


@pytest.mark.parametrize("h, w", [(24, 32), (29, 37), (211, 300), (64, 520)])
def test_random_weights_match_the_oracle(gpu, h, w):
    t = random_weights(seed=h + w)
    blob = write_tza(t)
    den = Denoiser(blob)
    layers = D.build_net(D.parse_tza(blob))
    color, albedo, normal = images(h, w, seed=h * w)
    out = den.denoise(color, albedo, normal)
    want = D.denoise(color, albedo, normal, layers)
    assert np.isfinite(out).all()
    assert gap(out, want) <= TOL, gap(out, want)
    assert np.array_equal(out[..., 3], color[..., 3])


def test_a_frame_split_into_tiles_matches_the_oracle(gpu):
    h, w = 800, 1000
    blob = write_tza(random_weights(seed=11))
    den = Denoiser(blob)
    den.set_max_tile_pixels(600_000)
    color, albedo, normal = images(h, w, seed=5)
    out = den.denoise(color, albedo, normal)
    tiles = den.tiles()
    assert tiles is not None and tiles[2] > 1
    want = D.denoise(color, albedo, normal, D.build_net(D.parse_tza(blob)), 600_000)
    assert gap(out, want) <= TOL, gap(out, want)


def test_nan_and_infinite_colour_match_the_oracle(gpu):
    h, w = 48, 64
    blob = write_tza(random_weights(seed=2))
    den = Denoiser(blob)
    color, albedo, normal = images(h, w, seed=9)
    color[3, 5, 0] = np.nan
    color[10, 20, :3] = np.inf
    color[11, 21, 1] = -np.inf
    albedo[7, 7, 2] = np.nan
    normal[8, 9, 0] = np.nan
    out = den.denoise(color, albedo, normal)
    want = D.denoise(color, albedo, normal, D.build_net(D.parse_tza(blob)))
    assert np.isfinite(out[..., :3]).all()
    assert gap(out, want) <= TOL, gap(out, want)


def test_the_tracer_films_through_the_device_path(gpu):
    import torch

    from pfx_b200 import synth
    from pfx_b200.trace import Trace

    w = synth.small("plain_512", (96, 64), sampler="sobol")
    trace = Trace(w.scene, w.settings, w.width, w.height)
    trace.sample(4, 3)
    films = trace.readback()
    blob = write_tza(random_weights(seed=7))
    den = Denoiser(blob)
    out = torch.empty((w.height, w.width, 4), dtype=torch.float32, device="cuda")
    den.denoise_trace(trace, out.data_ptr())
    ms, macs = den.last()
    assert ms > 0.0 and macs > 0
    host = den.denoise(films.color, films.albedo, films.normal)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), host.view(np.uint32))
    want = D.denoise(films.color, films.albedo, films.normal, D.build_net(D.parse_tza(blob)))
    assert gap(host, want) <= TOL, gap(host, want)
    trace.close()


def test_a_wait_that_runs_out_fails_the_call_and_the_denoiser_recovers(gpu):
    blob = write_tza(random_weights(seed=1))
    den = Denoiser(blob)
    color, albedo, normal = images(32, 48, seed=1)
    good = den.denoise(color, albedo, normal)
    den.set_wait_limit(0)
    with pytest.raises(abi.TraceError) as e:
        den.denoise(color, albedo, normal)
    assert e.value.code == abi.ERR_DEVICE and "ran out" in e.value.message
    den.set_wait_limit(1 << 26)
    again = den.denoise(color, albedo, normal)
    assert np.array_equal(again.view(np.uint32), good.view(np.uint32))


@pytest.mark.parametrize("shape", [1, 2, 3, 4, 5, 6, 7, 8, 9])
def test_every_conv_shape_matches_the_oracle(gpu, shape):
    """Every conv CTA shape (rows per CTA, stages, CTAs per SM), forced on
    the layers whose outputs it fits, gives the oracle's image."""
    h, w = 130, 270
    blob = write_tza(random_weights(seed=21))
    den = Denoiser(blob)
    assert den._lib.pfxt_debug_denoiser_shape(den.handle, shape) == abi.OK
    color, albedo, normal = images(h, w, seed=22)
    out = den.denoise(color, albedo, normal)
    want = D.denoise(color, albedo, normal, D.build_net(D.parse_tza(blob)))
    assert gap(out, want) <= TOL, gap(out, want)
