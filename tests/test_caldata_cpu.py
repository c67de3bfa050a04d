"""GPU calibrations written in the reference's calibration-data file format
are read back by the reference's own reader, skyline lookup and lookup-cost
model (compiled from its sources into oracle/_ref/libdtlref_caldata.so)."""
import ctypes as C
import os

import numpy as np
import pytest

from dtlg.model import cost as CM
from dtlg.model.calibration import DEFAULT_PATH, CalibrationData
from dtlg.model.caldata import MAGIC, POW2, read_reference_file, write_reference_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libdtlref_caldata.so")

pytestmark = pytest.mark.skipif(not os.path.exists(DEFAULT_PATH), reason="no calibration data")


@pytest.fixture(scope="module")
def written(tmp_path_factory):
    model = CM.CostModel(CalibrationData.load())
    path = str(tmp_path_factory.mktemp("cal") / "dtl-filter.dat")
    info = write_reference_file(path, model, n_log2=range(10, 25, 2), tw_log2=range(4, 25, 4))
    return model, path, info


def test_round_trip(written):
    model, path, info = written
    d = read_reference_file(path)
    assert d["mem_levels"] == 2 and d["cache_sizes"] == [126 << 20]
    assert len(d["bloom"]) == 2 * 278 and len(d["cuckoo"]) == 2 * 6
    t = d["bloom"][(8, 8, 8, 8, MAGIC, 1)]
    assert t.shape == (2, 2) and t[0, 1] > 0            # dt_L2 in ns
    sky = d["skyline"]
    assert len(sky["entries"]) == len(sky["n"]) * len(sky["tw"])
    assert os.path.getsize(path) == info["bytes"]


def ref():
    L = C.CDLL(LIB)
    L.ref_cal_sizeof.restype = C.c_uint64
    L.ref_cal_open.restype = C.c_void_p
    L.ref_cal_open.argtypes = [C.c_char_p]
    L.ref_cal_close.argtypes = [C.c_void_p]
    for fn in ("ref_cal_mem_levels", "ref_cal_bbf_count"):
        getattr(L, fn).restype = C.c_uint64
        getattr(L, fn).argtypes = [C.c_void_p]
    for fn in ("ref_cal_cache_size", "ref_cal_filter_size"):
        getattr(L, fn).restype = C.c_uint64
        getattr(L, fn).argtypes = [C.c_void_p, C.c_uint32]
    L.ref_cal_bbf_timing.argtypes = [C.c_void_p] + [C.c_uint32] * 7 + [C.POINTER(C.c_double)] * 2
    L.ref_cal_lookup_cost.argtypes = [C.c_void_p] + [C.c_uint32] * 6 + [C.c_uint64] + [C.POINTER(C.c_double)] * 2
    L.ref_cal_skyline.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    return L


@pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref/libdtlref_caldata.so not built")
def test_reference_reader_takes_the_file(written):
    model, path, _ = written
    L = ref()
    assert [L.ref_cal_sizeof(i) for i in range(5)] == [24, 12, 16, 4, 48]
    h = L.ref_cal_open(path.encode())
    assert h
    try:
        assert L.ref_cal_mem_levels(h) == 2
        assert L.ref_cal_cache_size(h, 0) == 126 << 20
        m1, m2 = L.ref_cal_filter_size(h, 0), L.ref_cal_filter_size(h, 1)
        assert L.ref_cal_bbf_count(h) == 2 * 278
        d = read_reference_file(path)
        cyc, ns = C.c_double(), C.c_double()
        for key in [(8, 8, 8, 8, MAGIC, 1), (4, 4, 1, 1, POW2, 1), (8, 4, 16, 16, MAGIC, 2), (16, 8, 8, 8, MAGIC, 4)]:
            for level in (0, 1):
                assert L.ref_cal_bbf_timing(h, *key, level, C.byref(cyc), C.byref(ns)) == 1
                assert ns.value == d["bloom"][key][level, 1] and cyc.value == d["bloom"][key][level, 0]
            # the reference's cost model (filter size in bytes against the stored
            # cache size) reproduces the calibrated times at the two filter sizes
            ci = [c.name for c in model.candidates].index(
                f"bbf u{key[1] * 8} w={key[2]} s={key[3]} z={key[5]} k={key[0]}")
            for m in (m1, m2):
                assert L.ref_cal_lookup_cost(h, *key, m, C.byref(cyc), C.byref(ns)) == 1
                want = float(np.interp(np.log2(m / 8), model.calib.log2_bytes, model.calib.ns_per_key[ci]))
                assert abs(ns.value - want) <= 1e-9 * want, (key, m)
        # its skyline lookup returns the cheapest of the (up to four) entries
        # around the query point (skyline_matrix.hpp:119-157)
        cfg = (C.c_uint32 * 6)()
        m = C.c_uint64()
        sky = d["skyline"]
        nn, nt = len(sky["n"]), len(sky["tw"])
        for n, tw in [(1 << 10, 16), (1 << 16, 1 << 12), (1 << 24, 1 << 24), (3000, 100)]:
            assert L.ref_cal_skyline(h, n, tw, cfg, C.byref(m), C.byref(cyc)) == 1
            i_n = min(int(np.searchsorted(sky["n"], n)), nn - 1)
            i_t = min(int(np.searchsorted(sky["tw"], tw)), nt - 1)
            around = [sky["entries"][t * nn + k] for t in (i_t, i_t + 1) for k in (i_n, i_n + 1) if t < nt and k < nn]
            best = min(around, key=lambda e: e[7])
            assert tuple(cfg) == best[:6] and m.value == best[6] and cyc.value == best[7]
    finally:
        L.ref_cal_close(h)
