"""CPU tests of the code layer: the shipped reference tables, the QC and IRA
generators (structure, 4-cycle freedom, rank) and both encoders (zero syndrome)."""
import numpy as np
import pytest

import fast_ldpc_decoder_for_gpu_fixed_b200 as fl
from fast_ldpc_decoder_for_gpu_fixed_b200.codes import (Encoder, IRAEncoder, ira, qc_irregular, qc_regular)

# (N, checks, edges, groups) of src/matrix/<code>/constantes_gpu.h
REFERENCE = {
    "4000x2000": (4000, 2000, 12000, [(6, 2000)]),
    "576x288": (576, 288, 1824, [(7, 96), (6, 192)]),
    "1944x972": (1944, 972, 6966, [(8, 162), (7, 810)]),
    "2048x384": (2048, 384, 12288, [(32, 384)]),
    "64800x32400": (64800, 32400, 226799, [(7, 32399), (6, 1)]),
}


def test_all_reference_tables_shipped():
    assert len(fl.reference_tables()) == 14


@pytest.mark.parametrize("name", sorted(REFERENCE))
def test_reference_table_contents(name):
    code = fl.load_table(name)
    n, m, e, groups = REFERENCE[name]
    assert (code.n, code.m, code.e) == (n, m, e)
    assert code.groups == groups
    d1, c1 = groups[0]
    assert (code.row_class[:c1] == 0).all() and (code.row_class[c1:] == 1).all()
    assert (code.degrees[:c1] == d1).all()


def test_first_row_of_default_table():
    # src/matrix/4000x2000/constantes_decoder.h:4
    assert fl.load_table("4000x2000").cols[:6].tolist() == [490, 694, 954, 999, 2407, 2908]


def _has_4cycle(code):
    h = code.dense().astype(np.int32)
    ov = h @ h.T
    np.fill_diagonal(ov, 0)
    return (ov > 1).any()


def test_qc_regular_structure():
    c = qc_regular(z=64, mb=8, nb=16, wc=3, seed=5)
    assert (c.n, c.m) == (1024, 512)
    assert set(c.degrees.tolist()) == {6}
    colw = np.bincount(c.cols, minlength=c.n)
    assert set(colw.tolist()) == {3}
    assert not _has_4cycle(c)
    enc = Encoder(c)
    cw = enc.encode(np.random.default_rng(0).integers(0, 2, size=(8, enc.k)))
    assert c.syndrome(cw).max() == 0


def test_qc_regular_is_deterministic():
    a = qc_regular(z=32, seed=9)
    b = qc_regular(z=32, seed=9)
    assert np.array_equal(a.cols, b.cols)


@pytest.mark.parametrize("z,rate", [(27, (1, 2)), (54, (2, 3)), (81, (3, 4)), (27, (5, 6))])
def test_qc_irregular(z, rate):
    c = qc_irregular(z=z, rate=rate)
    assert c.n == 24 * z and c.m == 24 * z * (rate[1] - rate[0]) // rate[1]
    assert not _has_4cycle(c)
    enc = Encoder(c)
    assert enc.rank == c.m
    cw = enc.encode(np.random.default_rng(1).integers(0, 2, size=(5, enc.k)))
    assert c.syndrome(cw).max() == 0


def test_ira_structure_and_encoder():
    c = ira(n=3600, k=1800, group=360, seed=3)
    assert (c.n, c.m) == (3600, 1800)
    colw = np.bincount(c.cols, minlength=c.n)
    assert set(colw[:1800].tolist()) <= {3, 8}
    assert (colw[1800:-1] == 2).all() and colw[-1] == 1     # dual-diagonal staircase
    enc = IRAEncoder(c)
    cw = enc.encode(np.random.default_rng(2).integers(0, 2, size=(6, enc.k)))
    assert c.syndrome(cw).max() == 0


def test_ira_default_degree_profile():
    c = ira()
    assert (c.n, c.m) == (64800, 32400)
    assert abs(c.degrees.mean() - 6.0) < 0.05
