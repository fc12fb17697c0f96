"""Tolerance of the raycast against the oracle's.

The library marches the reference's rays (GenerateDepthKernel /
GenerateRgbKernel, tsdf.cu:471-526) in voxel units with fused
multiply-adds, and steps through free space (cells whose voxels are all
unobserved or saturated) without interpolating; the oracle evaluates the
reference's expressions with IEEE rounding at every sample.  Both take the
same steps up to rounding, so depths agree to rounding almost everywhere;
where a rounding difference flips a discrete choice (a sample's voxel at a
half-voxel tie, the last step before the stop test) the hit moves by at most
about a voxel.  Bars: hit / miss agreement on at least 99.5 % of pixels;
over pixels both hit, the median difference within 1 % of a voxel and the
99th percentile within a voxel; colours within 2 units on 99 % of them.
"""
import numpy as np


def assert_raycast_close(gd, od, voxel_size, max_depth, grgb=None, orgb=None):
    hit_g, hit_o = gd < max_depth, od < max_depth
    agree = float(np.mean(hit_g == hit_o))
    assert agree >= 0.995, f"hit/miss agreement {agree}"
    both = hit_g & hit_o
    assert both.sum() > 0.1 * both.size
    err = np.abs(gd[both].astype(np.float64) - od[both])
    med, p99 = float(np.median(err)), float(np.quantile(err, 0.99))
    assert med <= 0.01 * voxel_size, f"median {med}"
    assert p99 <= voxel_size, f"p99 {p99}"
    if grgb is not None:
        dc = np.abs(grgb[both].astype(np.int32) - orgb[both].astype(np.int32)).max(axis=-1)
        assert float(np.mean(dc <= 2)) >= 0.99, f"colour within 2 on {np.mean(dc <= 2)}"
    return {"agree": agree, "median": med, "p99": p99}
