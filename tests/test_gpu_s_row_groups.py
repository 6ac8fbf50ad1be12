"""The row-group FP32 y = S v kernel (one warp per group of up to 8 rows sharing a column segment) against the
one-warp-per-row-segment kernel and the FP64 apply, through the allocating A^-1 entry point.  Scenes: a small
hex cantilever, the heterogeneous tet block of the bench, and a 24^3 hex block (rows of up to 2048-value
segments, groups whose rows end at different columns)."""
import numpy as np
import pytest

from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu


def _scenes():
    return [("cantilever", lambda: scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=1)),
            ("nh_tet_block", lambda: scenes.nh_tet_block()),
            ("contact_drop", lambda: scenes.contact_drop())]


@pytest.mark.parametrize("name,make", _scenes(), ids=[s[0] for s in _scenes()])
def test_row_group_s_pass_matches_row_kernel_and_fp64(name, make):
    sc = make()
    d = core.from_scene(sc)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(sc.dofs)
    x64 = d.debug_ainv(b, sc.dt, fp32=False)
    d.set_s_kernel(row_groups=True)
    xs = d.debug_ainv(b, sc.dt, fp32=True)
    xs2 = d.debug_ainv(b, sc.dt, fp32=True)
    d.set_s_kernel(row_groups=False)
    xr = d.debug_ainv(b, sc.dt, fp32=True)
    d.set_s_kernel(row_groups=True)
    scale = np.abs(x64).max()
    assert np.array_equal(xs, xs2)  # deterministic
    e_reg = np.abs(xs - xr).max() / scale
    e_64 = np.abs(xs - x64).max() / scale
    print(f"{name}: row groups vs one row per warp {e_reg:.2e}, vs FP64 {e_64:.2e}")
    assert e_reg == 0.0, e_reg  # the two kernels sum in the same per-lane order
    assert e_64 < 5e-5, e_64
