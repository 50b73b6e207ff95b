"""The burst generator of the median-stack workload (CPU): frame count and
size, near-identity homographies within the stated translation and rotation,
and the share of pixels under outlier rectangles."""
import math

import numpy as np

from image360_b200 import synth


def test_burst_generator_shapes_and_motion():
    cfg = synth.scaled_stack(synth.C2, 0.03)
    st = synth.make_stack(cfg)
    assert len(st.cfa) == cfg.frames == 16
    for c in st.cfa:
        assert tuple(c.shape) == (cfg.frame_h, cfg.frame_w)
        a = c.numpy().view(np.uint16) if c.dtype != np.uint16 else c
        assert int(np.asarray(a).max()) <= (1 << cfg.bits) - 1
    for H in st.to_ref:
        rot = math.degrees(math.atan2(H[1, 0], H[0, 0]))
        assert abs(rot) <= cfg.max_rot_deg + 1e-9
        cx, cy = (cfg.frame_w - 1) / 2.0, (cfg.frame_h - 1) / 2.0
        moved = H @ np.array([cx, cy, 1.0])
        assert abs(moved[0] - cx) <= cfg.max_shift + 1e-9 and abs(moved[1] - cy) <= cfg.max_shift + 1e-9
    assert all(0.05 <= f < 0.2 for f in st.outlier_frac)
    assert len({round(float(H[0, 2]), 6) for H in st.to_ref}) == cfg.frames  # distinct motions
