"""Frame output on the host: the PNG encoder and the CPU renderer's geometry."""
import numpy as np


def test_png_round_trip(tmp_path):
    from mpm_snow_sim2d_b200 import image
    rgb = (np.random.default_rng(1).random((9, 13, 3)) * 255).astype(np.uint8)
    image.write_png(tmp_path / "f.png", rgb)
    data = (tmp_path / "f.png").read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    assert np.array_equal(image.decode_png(data), rgb)


def test_reference_renderer_geometry():
    from oracle import render_ref
    # one particle at the centre of a 2D 100 x 50 domain on a 200 x 100 image
    img = render_ref.render(np.array([[50.0, 25.0]]), 2, 100, 50, 0, 3, 200, 100, point_size=3.0)
    # x = 50 -> pixel column 100, y = 25 -> row 100 - 50 = 50 (rows top first)
    lit = np.argwhere(img[..., 0] == img[..., 0].max())
    assert img[..., 0].max() == 255
    assert abs(lit[:, 0].mean() - 49.5) <= 0.5 and abs(lit[:, 1].mean() - 99.5) <= 0.5
    assert (img == 128).any()  # the border
    # 3D: a particle at the grid centre projects to the image centre
    img3 = render_ref.render(np.array([[16.0, 16.0, 16.0]]), 3, 32, 32, 32, 2, 200, 100, point_size=3.0,
                             distance=60.0)
    ys, xs = np.nonzero(img3[..., 0] == 255)
    assert abs(xs.mean() - 100) < 1.5 and abs(ys.mean() - 50) < 1.5
