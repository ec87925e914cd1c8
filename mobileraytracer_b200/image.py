"""Headless output of a render: the ARGB8888 bitmap of Renderer::renderFrame (red in the low byte,
Utils.cpp:48-70) as an RGB array or a binary PPM file, in place of the reference's GTK / GLES
display (GTK_Interface.cpp:61-102), which needs a graphics stack."""
from __future__ import annotations

import numpy as np


def to_rgb(bitmap, width: int | None = None, height: int | None = None) -> np.ndarray:
    """(H, W, 3) uint8 from a bitmap (numpy or CUDA tensor, shape (H, W) or flat with width/height)."""
    if hasattr(bitmap, "cpu"):
        bitmap = bitmap.cpu().numpy()
    b = np.ascontiguousarray(bitmap).view(np.uint32)
    if b.ndim == 1:
        b = b.reshape(height, width)
    return np.stack([b & 0xFF, (b >> 8) & 0xFF, (b >> 16) & 0xFF], -1).astype(np.uint8)


def write_ppm(path: str, bitmap, width: int | None = None, height: int | None = None) -> None:
    rgb = to_rgb(bitmap, width, height)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (rgb.shape[1], rgb.shape[0]))
        f.write(rgb.tobytes())
