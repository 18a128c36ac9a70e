"""numpy mirrors of the C structs in include/aprict_b200.h.

``proj_spec`` is byte-identical to the reference's ``proj_spec``
(src/aprict/data/cusrc/geometry.h:1-13; Python mirror
src/aprict/cuda/structs/geometry.py), so a reference user's packed view array
can be passed unchanged. The layouts are fixed here instead of being probed on
the GPU at import time as the reference does (src/aprict/cuda/kern_structs.py:355-409);
``aprict_b200_struct_size`` in the library cross-checks them.
"""

from __future__ import annotations

import numpy as np

fvec3 = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4")])

proj_spec = np.dtype(
    {
        "names": ["source_pos", "det_pos", "det_u", "det_v", "nu", "nv", "type"],
        "formats": [fvec3, fvec3, fvec3, fvec3, "<u4", "<u4", "u1"],
        "offsets": [0, 12, 24, 36, 48, 52, 56],
        "itemsize": 60,
    }
)

vol_desc = np.dtype(
    {
        "names": ["nx", "ny", "nz", "order", "voxwid", "corner"],
        "formats": ["<u4", "<u4", "<u4", "<u4", "<f4", fvec3],
        "offsets": [0, 4, 8, 12, 16, 20],
        "itemsize": 32,
    }
)

proj_desc = np.dtype(
    {
        "names": ["n_views", "nu", "nv", "stride_view", "stride_u", "stride_v"],
        "formats": ["<u4", "<u4", "<u4", "<i8", "<i8", "<i8"],
        "offsets": [0, 4, 8, 16, 24, 32],
        "itemsize": 40,
    }
)

project_config = np.dtype(
    [("shrink_volume_factor", "<f4"), ("multiply_before_adding", "<f4"), ("ssu", "<u4"), ("ssv", "<u4")]
)

backproject_config = np.dtype(
    [
        ("exact", "<u4"),
        ("backproject_all_1s", "<u4"),
        ("mask_to_cylinder", "<u4"),
        ("mask_to_cyl_rad", "<f4"),
        ("apply_summand_multiplier", "<u4"),
        ("soften_edge_proportion", "<f4"),
        ("Z_on_L_factor_power", "<i4"),
        ("Z_on_val_factor_power", "<i4"),
        ("Z_on_val_factor_val", "<f4"),
        ("approx_mode_direct_raycast", "<u4"),
        ("approx_mode_linear_interpolate", "<u4"),
        ("weighting_preset", "<u4"),
        ("ssx", "<u4"),
        ("ssy", "<u4"),
        ("ssz", "<u4"),
        ("soft_vartheta_v", "<f4"),
        ("soft_vartheta_v_softspan", "<f4"),
        ("soft_vartheta_h", "<f4"),
        ("soft_vartheta_h_softspan", "<f4"),
    ]
)

forbild_clip = np.dtype(
    {"names": ["axis", "dotprod", "mode"], "formats": [fvec3, "<f4", "u1"], "offsets": [0, 12, 16], "itemsize": 20}
)

# Byte-identical to the reference's FORBILD_Shape (FORBILD_volumes.h:1395-1415).
forbild_shape = np.dtype(
    {
        "names": ["type", "rho", "cas1", "cas2", "cas3", "x", "y", "z", "dx", "dy", "dz", "r", "r1", "r2", "l",
                  "a_x", "a_y", "a_z", "axis"],
        "formats": ["u1", "<f4", forbild_clip, forbild_clip, forbild_clip] + ["<f4"] * 10 + [fvec3] * 4,
        "offsets": [0, 4, 8, 28, 48, 68, 72, 76, 80, 84, 88, 92, 96, 100, 104, 108, 120, 132, 144],
        "itemsize": 156,
    }
)

quadric = np.dtype(
    [
        ("kind", "<i4"),
        ("n_clip", "<i4"),
        ("rho", "<f8"),
        ("c", "<f8", (3,)),
        ("M", "<f8", (9,)),
        ("h", "<f8"),
        ("alpha", "<f8"),
        ("beta", "<f8"),
        ("clip", "<f8", (3, 4)),
        ("bb_half", "<f8", (3,)),
    ]
)

# One scan of a batch (aprict_scan): the arguments of one one-scan call.
scan = np.dtype(
    {
        "names": ["specs_dev", "projs", "projs_dev", "base_dev", "vol", "vol_dev", "multiplier_dev", "status_dev"],
        "formats": ["<u8", proj_desc, "<u8", "<u8", vol_desc, "<u8", "<u8", "<u8"],
        "offsets": [0, 8, 48, 56, 64, 96, 104, 112],
        "itemsize": 120,
    }
)

# name in the C library -> numpy dtype, checked against sizeof() in tests.
ABI_STRUCTS = {
    "aprict_proj_spec": proj_spec,
    "aprict_vol_desc": vol_desc,
    "aprict_proj_desc": proj_desc,
    "aprict_project_config": project_config,
    "aprict_backproject_config": backproject_config,
    "aprict_forbild_shape": forbild_shape,
    "aprict_quadric": quadric,
    "aprict_scan": scan,
}
