"""The bench line's roofline.traffic comes from the committed ncu summaries
(profiles/<pass>_pass_512.md, a line traffic_bytes_per_launch_<waves>_waves):
the default workload's 1024-wave launches of both passes must find theirs,
and each figure must lie below the algorithmic bytes of its launch (24 N per
wave, N = 512^2) -- traffic far above that would mean re-reads."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("kind", ["column", "row"])
def test_traffic_figures_for_the_default_workload(kind):
    sys.path.insert(0, ROOT)
    import bench

    t = bench.traffic_from_profiles(kind, 1024)
    assert t is not None, kind
    algo = 1024 * 24 * 512 * 512
    assert 0.2 * algo < t < algo, (kind, t, algo)
