"""Reference API surface beyond the operators, on the GPU: Volume slicing and
axis sums (Volume.as_cupy_slice / sum_to_cupy_array, volume.py:260-275, torch
forms here), the ramp filter's bulk stream / concat forms
(ramp_filter.py:242-305), the no-op filterer (cb/noop_filter.py) and the
overflow counter alias."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from aprict_b200 import Volume
from aprict_b200.cb import NoOpFilterer, RampFilterer
from aprict_b200.cb import flatpanel as fp
from helpers import circular

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", ["C", "F"])
def test_volume_slices_and_axis_sums(order: str) -> None:
    rng = np.random.default_rng(3)
    x = rng.random((9, 7, 5)).astype(np.float32)
    v = Volume(x, voxwid=1.0, order=order)
    for axis, sl, want in [(0, slice(2, 5), x[2:5]), (1, slice(None, 3), x[:, :3]), (2, slice(4, 99), x[:, :, 4:])]:
        got = v.slice_axis(axis, sl)
        assert got.is_contiguous()
        np.testing.assert_array_equal(got.cpu().numpy(), want)
    for axis in range(3):
        np.testing.assert_allclose(v.sum_axis(axis).cpu().numpy(), x.astype(np.float64).sum(axis), rtol=1e-6)
    with pytest.raises(ValueError):
        v.slice_axis(0, slice(9, 12))
    with pytest.raises(NotImplementedError):
        v.slice_axis(0, slice(0, 4, 2))


def test_ramp_bulk_forms_equal_one_call() -> None:
    rng = np.random.default_rng(4)
    data = torch.from_numpy(rng.random((7, 40, 6)).astype(np.float32)).cuda()
    rf = RampFilterer(physpixwid=0.5, proj_2d_shape=(40, 6), projs_per_batch=3)
    (whole,) = rf.filter(data)
    (cat,), _ = rf.filter_bulk_axis1_concat(data)
    parts = [o[0] for o, _ in rf.filter_bulk_axis1_stream(data)]
    assert [p.shape[0] for p in parts] == [3, 3, 1]
    assert torch.equal(cat, whole) and torch.equal(torch.cat(parts), whole)
    nf = NoOpFilterer(proj_2d_shape=(40, 6), projs_per_batch=3)
    (copy,), _ = nf.filter_bulk_axis1_concat(data)
    assert torch.equal(copy, data) and copy.data_ptr() != data.data_ptr()
    assert torch.equal(torch.cat([o[0] for o, _ in nf.filter_bulk_axis1_stream(data)]), data)


def test_overflow_counter_alias() -> None:
    ps = fp.ProjectionSet(circular(2, 50.0, 50.0, 1.0, 4, 4), data=None)
    assert ps.out_of_mem_counter_cp is ps.out_of_mem_counter and ps.out_of_mem_count == 0
