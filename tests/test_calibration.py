"""Calibration tables of the 3-D path (esrrf.calibration): the table as
GetSpatialCalibrationMFMdata_.java:293-308 assembles it, the text export round trip, the axial
offset regression of LinearRegressions.java:19-47 and what LiveSRRF_CL.initialise derives
(LiveSRRF_CL.java:207-240).  Host logic only."""
import numpy as np
import pytest

from esrrf import calibration as C
from esrrf import EsrrfError


def test_java_rounding_to_two_digits():
    # Math.round = floor(x + 1/2): halves go up, also for negative numbers
    got = C.round_to_n_digits([0.125, -0.125, 1.005, 2.675, -3.14159, 0.0], 2)
    want = [np.floor(v * 100 + 0.5) / 100 for v in [0.125, -0.125, 1.005, 2.675, -3.14159, 0.0]]
    np.testing.assert_array_equal(got, want)
    assert got[1] == -0.12 and got[4] == -3.14


def test_rank_gather_sort_quirk():
    # getSortedIndices gives ranks; sortArray gathers by them: out[i] = a[rank[i]], which is a
    # true sort only when the rank permutation is its own inverse
    nominal = [300.0, -300.0, 0.0, 600.0]          # ranks [2, 0, 1, 3]
    np.testing.assert_array_equal(C.sorted_indices(nominal), [2, 0, 1, 3])
    a = [10.0, 11.0, 12.0, 13.0]
    np.testing.assert_array_equal(C.sort_array(a, C.sorted_indices(nominal)), [12.0, 10.0, 11.0, 13.0])
    # an involution (a swap) does sort
    np.testing.assert_array_equal(C.sort_array([5.0, 4.0], C.sorted_indices([1.0, 0.0])), [4.0, 5.0])


def make_table():
    n = 9
    rng = np.random.default_rng(3)
    nominal = np.array([400, -400, 300, -300, 200, -200, 100, -100, 0], np.float64)
    return C.make_calibration_table(
        shift_x=rng.uniform(-2, 2, n), shift_y=rng.uniform(-2, 2, n), theta=rng.uniform(-1, 1, n),
        axial_positions=np.linspace(-400, 400, n) + rng.normal(0, 3, n), nominal_axial_positions=nominal,
        roi_locations=np.arange(n, dtype=np.float64), intensity_scaling=rng.uniform(0.8, 1.2, n),
        background_level=101.5)


def test_table_keys_order_and_contents():
    t = make_table()
    assert tuple(t) == C.CALIB_KEYS_ALL
    assert all(len(v) == 9 for v in t.values())
    np.testing.assert_array_equal(t["Background level (ADC)"], np.full(9, 101.5))
    for k, v in t.items():
        np.testing.assert_array_equal(v, np.round(v, 2))  # all rounded to 2 digits
    # axial positions are rounded, not reordered
    assert np.all(np.diff(t["Axial positions"]) > 0)
    with pytest.raises(EsrrfError):
        C.make_calibration_table([0.0], [0.0], [0.0], [0.0, 1.0], [0.0, 1.0], [0.0, 1.0], [1.0, 1.0], 0.0)


@pytest.mark.parametrize("row_numbers,decimals", [(True, None), (False, None), (True, 2)])
def test_text_round_trip(tmp_path, row_numbers, decimals):
    t = make_table()
    p = tmp_path / "cal - MFM_CalibrationTable.csv"
    C.save_calibration_table(p, t, row_numbers=row_numbers, decimals=decimals)
    back = C.load_calibration_table(p)
    assert tuple(back) == C.CALIB_KEYS_ALL
    for k in t:
        np.testing.assert_allclose(back[k], t[k], rtol=0, atol=0 if decimals is None else 5e-3)


def test_tab_separated_export_named_njt(tmp_path):
    t = make_table()
    p = tmp_path / "cal.njt"
    keys = list(t)
    lines = ["\t".join([" "] + keys)] + ["\t".join([str(i + 1)] + [f"{t[k][i]:.4f}" for k in keys]) for i in range(9)]
    p.write_text("\n".join(lines) + "\n")
    back = C.load_calibration_table(p)
    np.testing.assert_allclose(back["Theta (degrees)"], t["Theta (degrees)"], atol=1e-9)


def test_binary_and_broken_tables_are_refused(tmp_path):
    b = tmp_path / "cal.njt"
    b.write_bytes(b"\xac\xed\x00\x05sr\x00\x17java.util.LinkedHashMap")
    with pytest.raises(EsrrfError, match="binary NanoJ table"):
        C.load_calibration_table(b)
    m = tmp_path / "missing.csv"
    m.write_text("X-shift (pixels),Y-shift (pixels)\n1,2\n")
    with pytest.raises(EsrrfError, match="missing columns"):
        C.load_calibration_table(m)
    r = tmp_path / "ragged.csv"
    r.write_text(",".join(C.CALIB_KEYS_USED) + "\n1,2\n")
    with pytest.raises(EsrrfError, match="number of columns"):
        C.load_calibration_table(r)


def test_axial_offset_regression():
    # exact line through the plane closest to zero
    y = [-600.0, -300.0, 0.5, 300.5, 600.5]
    assert C.axial_offset(y) == pytest.approx((-2 * -600 + -1 * -300 + 300.5 + 2 * 600.5) / 10)
    # the first of two equally close entries anchors x = 0
    y2 = [-10.0, 10.0, 30.0]
    assert C.axial_offset(y2) == pytest.approx((0 * -10 + 1 * 10 + 2 * 30) / 5)


def test_table_geometry_matches_initialise():
    t = make_table()
    g = C.table_geometry(t, 384, 390, 3, 250.0, 0.106)
    assert (g["nPlanes"], g["widthS"], g["heightS"], g["nPlanesM"]) == (9, 128, 130, 27)
    assert g["backgroundLevel"] == 101.5
    off = np.float32(C.axial_offset(t["Axial positions"]))
    assert g["axialOffset"] == float(off)
    assert g["dimensionRatioXYvsZ"] == float(off / (np.float32(1000) * np.float32(0.106)))
    z = dict(t, **{"Axial positions": np.zeros(9)})
    assert C.table_geometry(z, 384, 384, 3, 250.0, 0.1)["axialOffset"] == 250.0
