"""Output stage: png.writePng (src/png.zig:10-117) and Image.toRgb8 on the
device.

CPU tests pin the host encoder to the oracle's restatement of png.zig (byte
for byte) and to Python's zlib (inflate round trip, chunk CRCs), as
png.zig's own round-trip tests do.  GPU tests check the device-assembled
PNG against the host encoder byte for byte, the device 8-bit encode against
the host one (equal except where the two math libraries' pow() round a value
to opposite sides of a u8 boundary: at most 1 LSB), and the fused
render-to-PNG entry point against the staged path.
"""
import struct
import zlib

import numpy as np
import pytest

import zigtrace_b200 as zt
from oracle import png as OPNG

SIZES = [(1, 1), (2, 1), (3, 2), (37, 23), (200, 150), (1456, 15), (1456, 30), (21845, 1)]


def _rgb(w, h, seed=0):
    return np.random.default_rng(seed).integers(0, 256, w * h * 3, dtype=np.uint8)


def _chunks(png: bytes):
    assert png[:8] == OPNG.SIGNATURE
    pos, out = 8, []
    while pos < len(png):
        (n,) = struct.unpack(">I", png[pos:pos + 4])
        kind, data = png[pos + 4:pos + 8], png[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", png[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(kind + data)
        out.append((kind, data))
        pos += 12 + n
    return out


def _decode(png: bytes):
    ch = _chunks(png)
    assert [k for k, _ in ch] == [b"IHDR", b"IDAT", b"IEND"]
    w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", ch[0][1])
    assert (depth, ctype, comp, filt, inter) == (8, 2, 0, 0, 0)
    raw = zlib.decompress(ch[1][1])
    rows = np.frombuffer(raw, np.uint8).reshape(h, 3 * w + 1)
    assert (rows[:, 0] == 0).all()
    return w, h, rows[:, 1:].reshape(-1)


def test_oracle_png_matches_zlib_checksums():
    data = bytes(_rgb(50, 7))
    assert OPNG.crc32(data) == zlib.crc32(data)
    assert OPNG.adler32(data) == zlib.adler32(data)


@pytest.mark.parametrize("w,h", SIZES)
def test_host_png_is_the_reference_stream(native_lib, w, h):
    rgb = _rgb(w, h, w + h)
    got = zt.encode_png(rgb, w, h)
    assert len(got) == zt.png_size(w, h)
    assert got == OPNG.write_png(w, h, bytes(rgb))
    ww, hh, back = _decode(got)
    assert (ww, hh) == (w, h) and back.tobytes() == rgb.tobytes()


def test_png_block_split(native_lib):
    # (3w+1)h = 65535 is one full stored block; twice that is two
    one = zt.encode_png(_rgb(1456, 15), 1456, 15)
    two = zt.encode_png(_rgb(1456, 30), 1456, 30)
    assert len(one) == 8 + 25 + 12 + (2 + 65535 + 5 + 4) + 12
    assert len(two) == 8 + 25 + 12 + (2 + 131070 + 10 + 4) + 12


def test_png_errors(native_lib):
    for w, h in ((0, 4), (4, 0), (2**31, 1), (1, 2**31)):
        with pytest.raises(zt.ZigtraceError, match="InvalidDimensions"):
            zt.png_size(w, h)
    with pytest.raises(zt.ZigtraceError, match="ImageTooLarge"):
        zt.png_size(2**31 - 1, 1)
    with pytest.raises(zt.ZigtraceError):
        zt.encode_png(np.zeros(5, np.uint8), 2, 1)


def test_write_png_file(native_lib, tmp_path):
    rgb = _rgb(5, 3)
    p = tmp_path / "x.png"
    with open(p, "wb") as f:
        zt.write_png(f, 5, 3, rgb)
    assert p.read_bytes() == OPNG.write_png(5, 3, bytes(rgb))


# ----------------------------------------------------------------- device --
@pytest.mark.gpu
@pytest.mark.parametrize("w,h", SIZES + [(1920, 1080), (4096, 2160)])
def test_device_png_equals_host_png(w, h):
    import torch
    rgb = _rgb(w, h, 3 * w + h)
    want = zt.encode_png(rgb, w, h)
    n = zt.png_size(w, h)
    d_rgb = torch.from_numpy(rgb).cuda()
    for offset in (0, 3):  # the PNG buffer at an odd address too
        d_out = torch.full((n + offset,), 0xAB, dtype=torch.uint8, device="cuda")
        zt.encode_png_device(d_rgb.data_ptr(), w, h, d_out.data_ptr() + offset, n,
                             torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert d_out[offset:].cpu().numpy().tobytes() == want


@pytest.mark.gpu
@pytest.mark.parametrize("tonemap", ["none", "reinhard", "aces"])
def test_device_rgb8_matches_host_encode(tonemap):
    import torch
    rng = np.random.default_rng(7)
    px = np.concatenate([rng.uniform(-1, 8, 3 * 400_000 - 9), rng.exponential(0.3, 3),
                         [np.nan, np.inf, -np.inf, 0.0, -0.0, 1e300]])
    n_pix = px.size // 3
    for gamma, exposure in ((2.2, 1.0), (1.0, 0.5), (2.4, 1.7)):
        out = zt.Output(tonemap=tonemap, gamma=gamma, exposure=exposure)
        want = zt.Image(n_pix, 1, px.reshape(-1, 3)).to_rgb8(out)
        for off_px, off_out in ((0, 0), (1, 1)):  # aligned (vector) and unaligned (scalar) paths
            d_px = torch.from_numpy(np.concatenate([np.zeros(off_px), px])).cuda()
            d_out = torch.zeros(px.size + off_out, dtype=torch.uint8, device="cuda")
            zt.image_to_rgb8_device(d_px.data_ptr() + 8 * off_px, n_pix, d_out.data_ptr() + off_out, out,
                                    torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            got = d_out[off_out:].cpu().numpy()
            diff = np.abs(got.astype(int) - want.astype(int))
            assert diff.max() <= 1
            assert (diff != 0).sum() <= 3, f"{(diff != 0).sum()} values differ by 1 LSB"


@pytest.mark.gpu
def test_render_png_matches_staged_path():
    from zigtrace_b200 import scenes
    scene = scenes.cornell().build()
    o = zt.Options(96, 64, 4, 16)
    out = zt.Output(tonemap="aces", gamma=2.2, exposure=1.0)
    hdr = zt.render(scene, o)
    rgb_host = hdr.to_rgb8(out)
    rgb_dev = zt.render_rgb8(scene, o, out)
    assert np.abs(rgb_dev.astype(int) - rgb_host.astype(int)).max() <= 1
    png = zt.render_png(scene, o, out)
    assert png == zt.encode_png(rgb_dev, 96, 64)
    w, h, back = _decode(png)
    assert (w, h) == (96, 64) and back.tobytes() == rgb_dev.tobytes()
    for mode in (zt.MODE_WAVEFRONT, zt.MODE_MEGAKERNEL_REGEN):
        assert zt.render_png(scene, o, out, zt.GpuConfig(mode)) == png
