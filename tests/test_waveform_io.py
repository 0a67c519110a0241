"""Waveform files: the writer reproduces the reference's hm*.dat rows byte
for byte, and QNM_Extraction's own loader reads what it writes."""
import glob
import os
import sys

import numpy as np
import pytest

import bh_ringdown_b200 as bhr

GOLD = os.path.join(os.path.dirname(__file__), "golden")
from oracle.build_ref import default_reference_root  # noqa: E402

REF = default_reference_root()


@pytest.mark.parametrize("fn,m", [("hm2_a0.7_thi000_thf090.0_n", 2.0), ("hmm1_a0.7_thi000_thf090.0_n", -1.0)])
def test_writer_reproduces_reference_rows_byte_for_byte(tmp_path, fn, m):
    path = os.path.join(GOLD, f"example_head_{fn}.txt")
    ref = open(path).read()
    d = np.loadtxt(path)
    bhr.write_waveform(str(tmp_path), "a0.7_thi000_thf090.0_n", m, d[:, 0], d[:, 1:])
    out = open(tmp_path / f"{fn}.dat").read()
    assert out == ref
    full = np.loadtxt(str(tmp_path / f"{fn}.dat.full"))
    assert np.allclose(full[:, :15], d, rtol=1e-6, atol=0)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "QNM_Extraction")), reason="reference tree not mounted")
def test_qnm_extraction_reads_written_files(tmp_path, monkeypatch):
    """QNM_Extraction/Library/ringdownlib.py:49-123 (loadwaveforms) on files
    written by bhr_write_waveform for m = 0..2 and -1, -2.  pandas 3 removed
    read_csv(delim_whitespace=...), so the harness maps it to sep=r'\\s+'."""
    import pandas
    orig = pandas.read_csv

    def read_csv(*a, **k):
        if k.pop("delim_whitespace", False):
            k["sep"] = r"\s+"
        return orig(*a, **k)
    monkeypatch.setattr(pandas, "read_csv", read_csv)
    sys.path.insert(0, os.path.join(REF, "QNM_Extraction", "Library"))
    try:
        import ringdownlib
    finally:
        sys.path.pop(0)
    rng = np.random.default_rng(7)
    t = 2000.0 + 0.1 * np.arange(200)
    files, expect = [], {}
    for m in (0, 1, 2, -1, -2):
        h = rng.standard_normal((len(t), 14))
        name = "a0.7_thi000_thf090.0_n"
        bhr.write_waveform(str(tmp_path), name, float(m), t, h)
        files.append(str(tmp_path / f"{'hmm' if m < 0 else 'hm'}{abs(m)}_{name}.dat"))
        expect[m] = h
    modes = [[2, 2], [3, 2], [2, 1], [2, -1], [3, -2], [2, 0]]
    res, (thf, thdot) = ringdownlib.loadwaveforms(files, modes, 4)
    assert thf == 90.0 and thdot == -1
    for (l, m), (tt, hp, hc) in zip(modes, res):
        col = 2 * (l - abs(m))
        h = expect[m]
        # the loader takes the first row as a header: data starts at row 1
        assert np.allclose(tt[:50], t[1:51], atol=1e-9)
        assert np.allclose(hp[:50], h[1:51, col], rtol=1e-5, atol=1e-12)
        assert np.allclose(hc[:50], h[1:51, col + 1], rtol=1e-5, atol=1e-12)
