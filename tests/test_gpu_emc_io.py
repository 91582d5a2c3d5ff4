"""Native .emc ingest (dfg_load_emc / dfg_save_emc) against the Python mirror
of the reference's reader and writer (emcfile.pyx) and against dfg_set_frames."""
import os

import numpy as np
import pytest

from common import load_case
from dragonfly_b200.emcfile import read_emc, write_emc


@pytest.mark.gpu
def test_gpu_emc_load_save_round_trip(tmp_path):
    from dragonfly_b200._lib import Context
    prob, _ = load_case("edge")   # ragged frames, empty frames, a count above 1023
    n = prob.num_data
    half = n // 2
    o1 = np.concatenate([[0], np.cumsum(prob.ones)])
    om = np.concatenate([[0], np.cumsum(prob.multi)])
    f1, f2 = str(tmp_path / "a.emc"), str(tmp_path / "b.emc")
    write_emc(f1, prob.num_pix, prob.ones[:half], prob.multi[:half], prob.place_ones[:o1[half]],
              prob.place_multi[:om[half]], prob.count_multi[:om[half]])
    write_emc(f2, prob.num_pix, prob.ones[half:], prob.multi[half:], prob.place_ones[o1[half]:],
              prob.place_multi[om[half]:], prob.count_multi[om[half]:])

    ref = Context(0)
    ref.set_detector(prob.qvals, prob.corr, prob.mask)
    ref.set_frames(prob.ones, prob.multi, prob.place_ones, prob.place_multi, prob.count_multi)
    c = Context(0)
    c.set_detector(prob.qvals, prob.corr, prob.mask)
    c.load_emc([f1, f2])
    assert c.num_data == n
    a, b = c.frame_params(), ref.frame_params()
    np.testing.assert_array_equal(a["fcounts"], b["fcounts"])
    np.testing.assert_array_equal(a["sum_fact"], b["sum_fact"])

    out = str(tmp_path / "c.emc")
    c.save_emc(out)
    num_pix, ones, multi, po, pm, cm = read_emc(out)
    assert num_pix == prob.num_pix
    for x, y in ((ones, prob.ones), (multi, prob.multi), (po, prob.place_ones), (pm, prob.place_multi),
                 (cm, prob.count_multi)):
        np.testing.assert_array_equal(x, y)

    # dense integer frames (type 1) are read as the same sparse frames
    dense = np.zeros((n, prob.num_pix), np.int32)
    for d in range(n):
        dense[d, prob.place_ones[o1[d]:o1[d + 1]]] = 1
        dense[d, prob.place_multi[om[d]:om[d + 1]]] = prob.count_multi[om[d]:om[d + 1]]
    fd = str(tmp_path / "d.emc")
    with open(fd, "wb") as f:
        head = np.zeros(256, np.int32)
        head[:3] = [n, prob.num_pix, 1]
        head.tofile(f)
        dense.tofile(f)
    c.load_emc(fd)
    np.testing.assert_array_equal(c.frame_params()["fcounts"], b["fcounts"])

    with pytest.raises(Exception):
        c.load_emc(str(tmp_path / "missing.emc"))
    c.close()
    ref.close()
