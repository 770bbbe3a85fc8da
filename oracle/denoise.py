"""CPU restatement of the reference's denoiser (test infrastructure only: the
checker of the sm_100a denoiser in pfx_b200/csrc/denoise.cu, never part of
the product path).

The reference's `pfx-denoise` crate is OIDN 2.5.1's RT filter ported to
Rust/WGSL; this module restates what decides its output, from the crate's
source:
  * the weights blob (crates/denoise/src/tza.rs:51-118): OIDN's tensor archive;
  * the network (net.rs:193-232): OIDN's U-Net, 3x3 convolutions with zero
    padding, bias and ReLU, 2x2 max pooling after enc_conv1-4, nearest
    upsampling of the deeper source concatenated before the skip source;
  * autoexposure (process.wgsl:108-157): mean luminance of ~16x16 bins,
    geometric mean of the bins above 1e-8, 0.18 over it;
  * input and output processing (process.wgsl:57-106): the PU transfer
    function and its inverse, normalised by norm_scales (lib.rs:75-78);
  * the tiling (tile.rs:30-95): tiles of at most 2160x2160 pixels overlapping
    by 96, aligned to 16.
Convolutions are evaluated in float64 (the reference sums in f32 in its own
order; OIDN's CPU device in another), so the oracle is as exact as either.
It is pinned against OIDN's own output on the reference's desk fixture
(tests/golden/denoise_desk.npz; tests/test_denoise_oracle.py).
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

RECEPTIVE_FIELD = 174          # net.rs:3
MIN_TILE_ALIGNMENT = 16        # tile.rs:1
DEFAULT_MAX_TILE_PIXELS = 2160 * 2160  # tile.rs:2
FLT_MAX = np.float32(3.4028234663852886e38)


# ------------------------------------------------------------------ weights
def half_to_float(bits: np.ndarray) -> np.ndarray:
    """IEEE binary16 -> binary32, exact (tza.rs:120-137)."""
    return bits.astype(np.uint16).view(np.float16).astype(np.float32)


def parse_tza(blob: bytes) -> dict:
    """OIDN tensor archive, version 2 (tza.rs:51-118): magic 0x41D7, major 2,
    then a table offset; the table lists name, dims, layout ("x" or "oihw"),
    type ('f' or 'h') and data offset of every tensor."""
    if len(blob) < 12 or struct.unpack_from("<H", blob, 0)[0] != 0x41D7:
        raise ValueError("invalid or corrupted weights blob")
    if blob[2] != 2:
        raise ValueError("unsupported weights blob version")
    at = struct.unpack_from("<Q", blob, 4)[0]
    count = struct.unpack_from("<I", blob, at)[0]
    at += 4
    tensors = {}
    for _ in range(count):
        n = struct.unpack_from("<H", blob, at)[0]
        at += 2
        name = blob[at:at + n].decode()
        at += n
        rank = blob[at]
        at += 1
        dims = list(struct.unpack_from(f"<{rank}I", blob, at))
        at += 4 * rank
        layout = blob[at:at + rank]
        at += rank
        if layout not in (b"x", b"oihw"):
            raise ValueError("invalid tensor layout")
        kind = chr(blob[at])
        at += 1
        offset = struct.unpack_from("<Q", blob, at)[0]
        at += 8
        elements = int(np.prod(dims))
        if kind == "f":
            data = np.frombuffer(blob, "<f4", elements, offset).astype(np.float32)
        elif kind == "h":
            data = half_to_float(np.frombuffer(blob, "<u2", elements, offset))
        else:
            raise ValueError("invalid tensor data type")
        tensors[name] = data.reshape(dims)
    return tensors


# ------------------------------------------------------------------ network
@dataclass
class Layer:
    name: str
    src0: int            # -1: the input tensor, else the index of a layer
    src1: int | None     # the skip source of an upsample+concat layer
    pool: bool
    level: int           # resolution level of the layer's input (0 = full)
    in0: int
    in1: int
    out: int
    weight: np.ndarray = field(repr=False)  # (out, in0 + in1, 3, 3)
    bias: np.ndarray = field(repr=False)

    @property
    def out_level(self) -> int:
        return self.level + (1 if self.pool else 0)


def build_net(tensors: dict, input_channels: int = 9) -> list[Layer]:
    """The U-Net of net.rs:193-232 (OIDN's UNetFilter::addUNet)."""
    layers: list[Layer] = []

    def channels(src):
        return input_channels if src == -1 else layers[src].out

    def level(src):
        return 0 if src == -1 else layers[src].out_level

    def push(name, src0, src1=None, pool=False):
        w, b = tensors[f"{name}.weight"], tensors[f"{name}.bias"]
        in0, in1 = channels(src0), (0 if src1 is None else channels(src1))
        lv = level(src1) if src1 is not None else level(src0)
        if src1 is not None and level(src0) != lv + 1:
            raise ValueError(f"{name}: the upsampled source is not one level down")
        if w.shape[1:] != (in0 + in1, 3, 3) or b.shape != (w.shape[0],):
            raise ValueError(f"{name}: the weights do not match the network")
        layers.append(Layer(name, src0, src1, pool, lv, in0, in1, w.shape[0], w, b))
        return len(layers) - 1

    x = push("enc_conv0", -1)
    pool1 = push("enc_conv1", x, pool=True)
    pool2 = push("enc_conv2", pool1, pool=True)
    pool3 = push("enc_conv3", pool2, pool=True)
    pool4 = push("enc_conv4", pool3, pool=True)
    x = push("enc_conv5a", pool4)
    x = push("enc_conv5b", x)
    x = push("dec_conv4a", x, pool3)
    x = push("dec_conv4b", x)
    x = push("dec_conv3a", x, pool2)
    x = push("dec_conv3b", x)
    x = push("dec_conv2a", x, pool1)
    x = push("dec_conv2b", x)
    x = push("dec_conv1a", x, -1)
    x = push("dec_conv1b", x)
    push("dec_conv0", x)
    if layers[-1].out != 3:
        raise ValueError("the network does not end in three channels")
    return layers


def conv3x3(x: np.ndarray, weight: np.ndarray, bias: np.ndarray) -> np.ndarray:
    """Zero-padded 3x3 convolution of x (H, W, C) in float64, then ReLU."""
    h, w, c = x.shape
    xp = np.zeros((h + 2, w + 2, c), np.float64)
    xp[1:-1, 1:-1] = x
    out = np.broadcast_to(bias.astype(np.float64), (h, w, weight.shape[0])).copy()
    wt = weight.astype(np.float64)
    for ky in range(3):
        for kx in range(3):
            out += xp[ky:ky + h, kx:kx + w] @ wt[:, :, ky, kx].T
    return np.maximum(out, 0.0)


def forward(layers: list[Layer], x: np.ndarray) -> np.ndarray:
    """The network on one tile tensor (H, W, 9), H and W multiples of 16."""
    outs = []
    for layer in layers:
        a = x if layer.src0 == -1 else outs[layer.src0]
        if layer.src1 is not None:
            skip = x if layer.src1 == -1 else outs[layer.src1]
            a = np.concatenate([np.repeat(np.repeat(a, 2, axis=0), 2, axis=1), skip], axis=2)
        y = conv3x3(a, layer.weight, layer.bias)
        if layer.pool:
            h, w = y.shape[0] // 2, y.shape[1] // 2
            y = y[:2 * h, :2 * w].reshape(h, 2, w, 2, -1).max(axis=(1, 3))
        outs.append(y)
    return outs[-1]


# ------------------------------------------------------------------ tiling
def _round_up(a: int, b: int) -> int:
    return -(-a // b) * b


def _round_up_rem(a: int, b: int, c: int) -> int:
    return (a + b - c - 1) // b * b + c


@dataclass
class Tile:
    src: tuple      # (y, x) of the tile's first image pixel
    dst: tuple      # (y, x) where that pixel lands in the tile buffer
    size: tuple     # (h, w) of image pixels in the tile
    out_src: tuple  # (y, x) in the tile buffer of the first pixel kept
    out_dst: tuple  # (y, x) in the image of the first pixel kept
    out_size: tuple  # (h, w) kept


@dataclass
class Plan:
    tile_h: int
    tile_w: int
    overlap: int
    tiles: list


def plan(height: int, width: int, max_tile_pixels: int = DEFAULT_MAX_TILE_PIXELS) -> Plan:
    """OIDN's tile split as tile.rs:30-95 restates it (UNetFilter::init)."""
    al = MIN_TILE_ALIGNMENT
    overlap = _round_up(RECEPTIVE_FIELD // 2, al)
    h, w = height, width
    tile_h, tile_w = _round_up(h, al), _round_up(w, al)
    pad_h, pad_w = tile_h % al, tile_w % al
    count_h = count_w = 1
    min_dim = max(4 * overlap, 768)
    min_tile_h, min_tile_w = _round_up_rem(min_dim, al, pad_h), _round_up_rem(min_dim, al, pad_w)
    span_h, span_w = 2 * overlap + pad_h, 2 * overlap + pad_w
    while tile_h * tile_w > max_tile_pixels:
        if tile_h > min_tile_h and tile_h > tile_w:
            nxt = -(-(h + span_h * count_h) // (count_h + 1))
            tile_h = min(max(_round_up_rem(nxt, al, pad_h), min_tile_h), tile_h - al)
            count_h = max(-(-max(h - span_h, 0) // (tile_h - span_h)), 1)
        elif tile_w > min_tile_w:
            nxt = -(-(w + span_w * count_w) // (count_w + 1))
            tile_w = min(max(_round_up_rem(nxt, al, pad_w), min_tile_w), tile_w - al)
            count_w = max(-(-max(w - span_w, 0) // (tile_w - span_w)), 1)
        else:
            break
    tiles = []
    for i in range(count_h):
        y = i * max(tile_h - span_h, 0)
        begin_h = overlap if i > 0 else 0
        end_h = overlap + pad_h if i < count_h - 1 else 0
        th1 = min(h - y, tile_h)
        th2 = th1 - begin_h - end_h
        align_h = tile_h - _round_up(th1, al)
        for j in range(count_w):
            x = j * max(tile_w - span_w, 0)
            begin_w = overlap if j > 0 else 0
            end_w = overlap + pad_w if j < count_w - 1 else 0
            tw1 = min(w - x, tile_w)
            tw2 = tw1 - begin_w - end_w
            align_w = tile_w - _round_up(tw1, al)
            tiles.append(Tile((y, x), (align_h, align_w), (th1, tw1), (align_h + begin_h, align_w + begin_w),
                              (y + begin_h, x + begin_w), (th2, tw2)))
    return Plan(tile_h, tile_w, overlap, tiles)


# ------------------------------------------------------------------ transfer
def pu_forward(y: np.ndarray) -> np.ndarray:
    y = y.astype(np.float64)
    return np.where(y <= 1.57945760e-06, 1.41283765e+03 * y,
                    np.where(y <= 3.22087631e-02, 1.64593172e+00 * np.power(np.maximum(y, 0.0), 4.31384981e-01)
                             - 2.94139609e-03,
                             1.92653254e-01 * np.log(y + 6.26026094e-03) + 9.98620152e-01))


def pu_inverse(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.float64)
    return np.where(x <= 2.23151711e-03, x / 1.41283765e+03,
                    np.where(x <= 3.70974749e-01,
                             np.power(np.maximum((x + 2.94139609e-03) / 1.64593172e+00, 0.0), 1.0 / 4.31384981e-01),
                             np.exp((x - 9.98620152e-01) / 1.92653254e-01) - 6.26026094e-03))


def norm_scales() -> tuple[float, float]:
    """(1 / max, max): max is the PU value of 65504 (lib.rs:75-78)."""
    m = float(np.float32(np.float32(1.926_532_5e-1) * np.float32(math.log(np.float32(65504.0) + np.float32(6.260_261e-3)))
                         + np.float32(9.986_201_5e-1)))
    return float(np.float32(1.0 / m)), m


def _clean(v: np.ndarray, lo, hi) -> np.ndarray:
    v = np.where(np.isnan(v), 0.0, v)
    return np.clip(v, lo, hi)


def autoexposure(color: np.ndarray) -> float:
    """process.wgsl:108-157 over the whole image (H, W, 4)."""
    h, w = color.shape[:2]
    gx, gy = -(-w // 16), -(-h // 16)
    c = _clean(color[..., :3].astype(np.float64), 0.0, float(FLT_MAX))
    lum = 0.212671 * c[..., 0] + 0.715160 * c[..., 1] + 0.072169 * c[..., 2]
    total, count = 0.0, 0
    for j in range(gy):
        y0, y1 = j * h // gy, (j + 1) * h // gy
        for i in range(gx):
            x0, x1 = i * w // gx, (i + 1) * w // gx
            mean = lum[y0:y1, x0:x1].sum() / ((y1 - y0) * (x1 - x0))
            if mean > 1e-8:
                total += math.log2(mean)
                count += 1
    return 0.18 / 2.0 ** (total / count) if count else 1.0


def denoise(color: np.ndarray, albedo: np.ndarray, normal: np.ndarray, layers: list[Layer],
            max_tile_pixels: int = DEFAULT_MAX_TILE_PIXELS) -> np.ndarray:
    """Denoised RGBA (alpha from `color`), as Denoiser::denoise computes it."""
    h, w = color.shape[:2]
    scale = autoexposure(color)
    norm, rcp_norm = norm_scales()
    p = plan(h, w, max_tile_pixels)
    out = np.zeros((h, w, 4), np.float32)
    out[..., 3] = color[..., 3]
    c = pu_forward(_clean(color[..., :3].astype(np.float64) * scale, 0.0, float(FLT_MAX))) * norm
    a = _clean(albedo[..., :3].astype(np.float64), 0.0, 1.0)
    n = _clean(normal[..., :3].astype(np.float64), -1.0, 1.0) * 0.5 + 0.5
    image = np.concatenate([c, a, n], axis=2)
    for t in p.tiles:
        x = np.zeros((p.tile_h, p.tile_w, 9), np.float64)
        x[t.dst[0]:t.dst[0] + t.size[0], t.dst[1]:t.dst[1] + t.size[1]] = \
            image[t.src[0]:t.src[0] + t.size[0], t.src[1]:t.src[1] + t.size[1]]
        y = forward(layers, x)
        y = y[t.out_src[0]:t.out_src[0] + t.out_size[0], t.out_src[1]:t.out_src[1] + t.out_size[1]]
        v = pu_inverse(_clean(y, 0.0, float(FLT_MAX)) * rcp_norm) * ((1.0 / scale) if scale != 0.0 else 0.0)
        out[t.out_dst[0]:t.out_dst[0] + t.out_size[0], t.out_dst[1]:t.out_dst[1] + t.out_size[1], :3] = v
    return out
