"""Headless image output (no GPU)."""
import numpy as np

from mobileraytracer_b200 import image


def test_ppm_round_trip(tmp_path):
    bm = np.array([[0xFF0000FF, 0xFF00FF00], [0xFFFF0000, 0xFF102030]], np.uint32)
    rgb = image.to_rgb(bm)
    assert rgb[0, 0].tolist() == [255, 0, 0] and rgb[0, 1].tolist() == [0, 255, 0]
    assert rgb[1, 0].tolist() == [0, 0, 255] and rgb[1, 1].tolist() == [0x30, 0x20, 0x10]
    p = tmp_path / "x.ppm"
    image.write_ppm(str(p), bm.reshape(-1), 2, 2)
    data = p.read_bytes()
    assert data.startswith(b"P6\n2 2\n255\n") and data[len(b"P6\n2 2\n255\n"):] == rgb.tobytes()
