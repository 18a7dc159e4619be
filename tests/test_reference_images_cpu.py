"""Round trips of the reference's own test images (128x128 crops of
tests/images/*.png) through the oracle, for every case of the reference's PSNR
tests (tests/metrics.rs:255-526): the quality is what the encoders should give
(floors per format, BC7 at least as good as BC1/BC3 on the same image, the
slowest preset of a family at least as good as its fastest), BC1/BC3 agree
with the independent numpy transcription, and the PSNR table that the GPU
test checks against is the oracle's. CPU only."""
import json

import numpy as np
import pytest

import reference_images as ri

FLOOR = {0: 35.0, 2: 40.0, 5: 38.0, 6: 40.0}


@pytest.fixture(scope="module")
def table(bcn, oracle_lib):
    return ri.oracle_psnr_table(bcn, oracle_lib)


def test_quality_floors_and_ordering(table):
    for case in ri.CASES:
        assert table[ri.case_id(case)] >= FLOOR[case[1]], ri.case_id(case)
    for im in ri.OPAQUE:
        bc1 = table["%s-bc1" % im]
        assert all(table["%s-bc7-%s" % (im, p)] > bc1 for p in ri.BC7_OPAQUE)
        assert table["%s-bc7-opaque_slow" % im] >= table["%s-bc7-opaque_ultra_fast" % im] - 0.01
        assert table["%s-bc6h-very_slow" % im] >= table["%s-bc6h-very_fast" % im] - 0.01
    for im in ri.ALPHA:
        bc3 = table["%s-bc3" % im]
        assert all(table["%s-bc7-%s" % (im, p)] > bc3 for p in ri.BC7_ALPHA)
        assert table["%s-bc7-alpha_slow" % im] >= table["%s-bc7-alpha_ultrafast" % im] - 0.01


def test_committed_table_is_the_oracles(table):
    committed = json.load(open(ri.TABLE))
    assert set(committed) == set(table)
    for k, v in table.items():
        assert committed[k] == pytest.approx(v, abs=1e-9), k


@pytest.mark.parametrize("name", ri.OPAQUE + ri.ALPHA)
def test_bc1_bc3_second_transcription_on_reference_images(oracle_lib, name):
    from oracle import numpy_restatement as nr
    img = ri.load(name)
    for vid in (0, 1, 2, 3, 4):
        assert np.array_equal(nr.compress_bc15(vid, img), oracle_lib.compress_rgba8(vid, img, 128, 128)), (name, vid)
