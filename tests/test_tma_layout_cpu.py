"""Host-side check of the TMA plane loads' alignment rules for the Cartesian
interior tile (waveqlab3d_q_gpu_b200/csrc/wql3d_device.cuh,
interior_split_tile and SplitSmem; csrc/wql3d_api.cu, the padded layout of
setup_block).  The arithmetic is restated here so that it can be checked over
many block sizes.  Over every tile of every block from 13 to 300 points per
axis, in FP64 and FP32, it checks three things:
* the box's innermost coordinate is a multiple of 16 bytes;
* every field plane's shared-memory destination sits on a 128-byte boundary;
* the box fits the tensor-map limits (at most 256 per dimension, inner extent a
  multiple of 16 bytes).
No GPU is involved."""
import pytest

NB = 3


def tma_plane_width(w, h, esz, vec):
    while (h * w * esz) % 128:
        w += vec
    return w


def layout(nq, nr, esz):
    xoff = 32 // esz
    row = 128 // esz
    px = ((xoff + nq + NB + row - 1) // row) * row
    py = nr + 2 * NB
    sy, sz = px, px * py
    o1 = xoff + sy * NB + sz * NB
    return sy, sz, o1


@pytest.mark.parametrize("esz", [8, 4])
def test_plane_boxes_keep_the_tma_rules(esz):
    vec = 16 // esz
    ty = 4
    h = ty + 6
    w = tma_plane_width(((38 + vec - 1 + vec - 1) // vec) * vec, h, esz, vec)
    assert w <= 256 and h <= 256 and (w * esz) % 16 == 0
    plane_bytes = 8 * h * w * esz
    for buf in (0, 1):
        for f in range(8):
            assert (buf * plane_bytes + f * h * w * esz) % 128 == 0
    for nq in list(range(13, 80)) + [101, 128, 129, 201, 256, 300]:
        for nr in (13, 23, 101):
            sy, sz, o1 = layout(nq, nr, esz)
            assert (sy * esz) % 16 == 0 and (sz * esz) % 16 == 0
            lo, hi = 7, nq - 6
            for x0 in range(lo, hi + 1, 32):
                for y0 in range(7, nr - 5, ty):
                    for zs in (7, 8, 20):
                        row0 = o1 + (x0 - 3 - 1) + sy * (y0 - 3 - 1) + sz * (zs - 1)
                        base0 = row0 - row0 % vec
                        for k in range(3):
                            plane0 = base0 + k * sz
                            cx = (plane0 % sz) % sy
                            cy = (plane0 % sz) // sy
                            assert cx % vec == 0 and cx >= 0 and cy >= 0, (nq, nr, x0, y0)
