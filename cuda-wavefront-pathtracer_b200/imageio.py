"""Image output and comparison: the display transform and writers of io/image.cpp (clip to [0, 1], sRGB OETF,
exposure 0; 8-bit PNG with stored deflate; little-endian PFM with bottom-to-top rows) and the PSNR of
tools/psnr.py (tone-mapped sRGB space)."""
import struct
import zlib

import numpy as np


def srgb(lin):
    x = np.clip(np.asarray(lin, np.float32), 0.0, 1.0)
    return np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1.0 / 2.4) - 0.055).astype(np.float32)


def tonemap_srgb8(lin):
    """Linear radiance -> 8-bit sRGB (io/image.cpp:45-50)."""
    return (srgb(lin) * 255.0 + 0.5).astype(np.uint8)


def accum_to_image(accum, w, h, spp):
    """w*h float4 radiance sums -> (h, w, 3) float32 mean radiance."""
    return (np.asarray(accum, np.float32).reshape(h, w, 4)[:, :, :3] / np.float32(spp)).astype(np.float32)


def psnr(a, b, space="srgb"):
    """PSNR in dB between two linear images: 'srgb' compares clip + sRGB OETF values (tools/psnr.py); 'srgb8'
    compares the 8-bit images; 'linear' uses the peak of b."""
    if space == "srgb":
        x, y, peak = srgb(a), srgb(b), 1.0
    elif space == "srgb8":
        x, y, peak = tonemap_srgb8(a).astype(np.float64), tonemap_srgb8(b).astype(np.float64), 255.0
    else:
        x, y, peak = np.asarray(a, np.float64), np.asarray(b, np.float64), float(np.max(b))
    mse = float(np.mean((np.asarray(x, np.float64) - np.asarray(y, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)


def write_pfm(path, img):
    img = np.asarray(img, np.float32); h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.0\n" % (w, h))
        f.write(np.ascontiguousarray(img[::-1]).astype("<f4").tobytes())


def read_pfm(path):
    with open(path, "rb") as f:
        kind = f.readline().strip()
        w, h = map(int, f.readline().split())
        scale = float(f.readline())
        ch = 3 if kind == b"PF" else 1
        data = np.frombuffer(f.read(w * h * ch * 4), "<f4" if scale < 0 else ">f4").astype(np.float32)
    return data.reshape(h, w, ch)[::-1].copy()


def write_png(path, rgb8):
    rgb8 = np.ascontiguousarray(rgb8, np.uint8); h, w = rgb8.shape[:2]
    raw = b"".join(b"\x00" + rgb8[y].tobytes() for y in range(h))
    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) + chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))
