"""Readers for the image files the library writes (test checkers): PFM and Radiance RGBE, and the
reference's image error restated in NumPy."""
from __future__ import annotations

import numpy as np


def read_pfm(path: str) -> np.ndarray:
    """[H, W, 3] float32, row 0 = top (PFM stores rows bottom to top; scale < 0: little-endian)."""
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(b"\n", 3)
    assert parts[0] == b"PF"
    w, h = (int(x) for x in parts[1].split())
    scale = float(parts[2])
    dt = "<f4" if scale < 0 else ">f4"
    px = np.frombuffer(parts[3], dtype=dt, count=3 * w * h).reshape(h, w, 3)
    return px[::-1].astype(np.float32)


def _read_scanline(buf: bytes, pos: int, w: int) -> tuple[np.ndarray, int]:
    if w >= 8 and w <= 0x7FFF and buf[pos] == 2 and buf[pos + 1] == 2 and (buf[pos + 2] << 8 | buf[pos + 3]) == w:
        pos += 4
        line = np.zeros((w, 4), np.uint8)
        for c in range(4):
            x = 0
            while x < w:
                n = buf[pos]
                pos += 1
                if n > 128:  # run
                    n -= 128
                    line[x:x + n, c] = buf[pos]
                    pos += 1
                else:  # literal
                    line[x:x + n, c] = np.frombuffer(buf, np.uint8, n, pos)
                    pos += n
                x += n
        return line, pos
    line = np.frombuffer(buf, np.uint8, 4 * w, pos).reshape(w, 4)
    return line, pos + 4 * w


def read_hdr(path: str) -> np.ndarray:
    """[H, W, 3] float32 from a Radiance RGBE file with a -Y H +X W resolution line."""
    with open(path, "rb") as f:
        buf = f.read()
    assert buf.startswith(b"#?RADIANCE")
    head_end = buf.index(b"\n\n") + 2
    res_end = buf.index(b"\n", head_end)
    tok = buf[head_end:res_end].split()
    assert tok[0] == b"-Y" and tok[2] == b"+X"
    h, w = int(tok[1]), int(tok[3])
    pos = res_end + 1
    out = np.zeros((h, w, 3), np.float32)
    for y in range(h):
        line, pos = _read_scanline(buf, pos, w)
        e = line[:, 3].astype(np.int32)
        f = np.where(e > 0, np.ldexp(1.0, e - (128 + 8)), 0.0)
        out[y] = (line[:, :3].astype(np.float64) * f[:, None]).astype(np.float32)
    return out


def reference_error(ref: np.ndarray, img: np.ndarray, as_written: bool = True) -> tuple[float, np.ndarray]:
    """CReferenceImage::GetError (CReferenceImage.cpp:28-51): per channel the square root of the
    mean of min(100, d^2), d = ref - img in FP32; returns 1/3 (e_r e_g + e_b) as written, or the
    mean of the three."""
    d = (np.asarray(ref, np.float32)[..., :3] - np.asarray(img, np.float32)[..., :3]).reshape(-1, 3)
    sq = np.minimum(np.float32(100.0), d * d).astype(np.float64)
    e = np.sqrt(sq.sum(0) / d.shape[0])
    return ((e[0] * e[1] + e[2]) / 3.0 if as_written else e.mean()), e
