"""MFM calibration tables: the inputs of the 3-D path (LiveSRRF_CL.initialise with a table,
LiveSRRF_CL.java:207-240).

The reference writes the table in gui/GetSpatialCalibrationMFMdata_.java:293-314 -- a
LinkedHashMap<String, double[]> with the keys of CALIB_KEYS_ALL, every entry rounded to 2 digits
and the per-ROI entries reordered by the nominal axial positions -- saves it with NanoJ-Core's
SaveNanoJTable (.njt) and shows it as the "Calibration-Table" ResultsTable window (:310; again on
loading, LiveSRRF_CL.java:222 and gui/ApplyCalibrationMFMdata_.java:59).  NanoJ-Core is not part
of the reference tree, so the binary .njt layout cannot be restated here; this module reads and
writes the table as ImageJ's ResultsTable text export of that window (comma- or tab-separated,
one row per plane, an optional leading row-number column), and a binary .njt is refused with an
explanation rather than guessed at.

Functions:
  make_calibration_table  the table exactly as GetSpatialCalibrationMFMdata_ assembles it
  load_calibration_table  text export -> {key: float64 array}
  save_calibration_table  {key: array} -> ImageJ-style CSV
  axial_offset            LinearRegressions.linearRegressionLeastSquareNoOffset(double[])
  table_geometry          what LiveSRRF_CL.initialise derives from a table
"""
from __future__ import annotations

import math
import os

import numpy as np

from ._lib import EsrrfError

# insertion order of GetSpatialCalibrationMFMdata_.java:296-308
CALIB_KEYS_ALL = ("X-shift (pixels)", "Y-shift (pixels)", "Theta (degrees)", "Axial positions",
                  "Nominal positions", "ROI #", "Intensity scaling", "Background level (ADC)")
# the entries LiveSRRF_CL.initialise reads (LiveSRRF_CL.java:213-220)
CALIB_KEYS_USED = ("X-shift (pixels)", "Y-shift (pixels)", "Theta (degrees)", "Axial positions",
                   "ROI #", "Intensity scaling", "Background level (ADC)")


def _java_round(x: float) -> float:
    """Math.round(double) as a double: floor(x + 1/2) (ties toward positive infinity)."""
    return float(math.floor(x + 0.5))


def round_to_n_digits(values, digits=2) -> np.ndarray:
    """GetSpatialCalibrationMFMdata_.roundToNdigits (:445-452): Math.round(v * 10^d) / 10^d."""
    R = math.pow(10, digits)
    return np.array([_java_round(float(v) * R) / R for v in values], np.float64)


def sorted_indices(values) -> np.ndarray:
    """GetSpatialCalibrationMFMdata_.getSortedIndices (:349-358): the rank of each entry (number
    of strictly smaller entries), which sortArray then uses as a gather index."""
    v = [float(x) for x in values]
    return np.array([sum(1 for u in v if u < vi) for vi in v], np.int64)


def sort_array(values, indices) -> np.ndarray:
    """GetSpatialCalibrationMFMdata_.sortArray (:361-367): out[i] = values[indices[i]]."""
    values = np.asarray(values, np.float64)
    return np.array([values[int(i)] for i in indices], np.float64)


def make_calibration_table(shift_x, shift_y, theta, axial_positions, nominal_axial_positions,
                           roi_locations, intensity_scaling, background_level, digits=2) -> dict:
    """The table as GetSpatialCalibrationMFMdata_.java:293-308 assembles it (axial positions
    already relative to the reference plane, :286-289): per-ROI entries rounded and reordered by
    the ranks of the nominal positions; the axial positions rounded but not reordered; the
    background level repeated for every plane."""
    idx = sorted_indices(nominal_axial_positions)
    n = len(idx)
    for name, a in (("shift_x", shift_x), ("shift_y", shift_y), ("theta", theta),
                    ("axial_positions", axial_positions), ("roi_locations", roi_locations),
                    ("intensity_scaling", intensity_scaling)):
        if len(a) != n:
            raise EsrrfError(f"{name} has {len(a)} entries, the nominal positions {n}")
    r = lambda a: round_to_n_digits(a, digits)  # noqa: E731
    return {
        "X-shift (pixels)": sort_array(r(shift_x), idx),
        "Y-shift (pixels)": sort_array(r(shift_y), idx),
        "Theta (degrees)": sort_array(r(theta), idx),
        "Axial positions": r(axial_positions),
        "Nominal positions": sort_array(r(nominal_axial_positions), idx),
        "ROI #": sort_array(r(roi_locations), idx),
        "Intensity scaling": sort_array(r(intensity_scaling), idx),
        "Background level (ADC)": np.full(n, float(background_level)),
    }


def _is_text(raw: bytes) -> bool:
    if not raw:
        return False
    if b"\x00" in raw[:4096]:
        return False
    try:
        raw[:4096].decode("utf-8")
    except UnicodeDecodeError:
        return False
    return True


def load_calibration_table(path) -> dict:
    """Read a calibration table saved as ImageJ's ResultsTable text export (the
    "Calibration-Table" window saved as .csv/.txt/.xls, or such a file named .njt).  Returns
    {column heading: float64 array} in file order.  Raises EsrrfError for a binary NanoJ-Core
    .njt file, a missing column LiveSRRF_CL.initialise reads, or ragged rows."""
    path = os.fspath(path)
    with open(path, "rb") as fh:
        raw = fh.read()
    if not _is_text(raw):
        raise EsrrfError(
            f"{path}: binary NanoJ table; its layout is defined by NanoJ-Core's SaveNanoJTable, "
            "which is not available here -- save the Calibration-Table window as CSV instead")
    lines = [ln for ln in raw.decode("utf-8").splitlines() if ln.strip()]
    if len(lines) < 2:
        raise EsrrfError(f"{path}: no table rows")
    sep = "\t" if "\t" in lines[0] else ","
    head = [h.strip().strip('"') for h in lines[0].split(sep)]
    rows = [[c.strip().strip('"') for c in ln.split(sep)] for ln in lines[1:]]
    if any(len(r) != len(head) for r in rows):
        raise EsrrfError(f"{path}: rows with a different number of columns than the heading")
    # ImageJ writes the row numbers as a first column headed " " (or empty)
    skip = 1 if head and head[0] in ("", " ") else 0
    out = {}
    for j in range(skip, len(head)):
        try:
            out[head[j]] = np.array([float(r[j]) for r in rows], np.float64)
        except ValueError as e:
            raise EsrrfError(f"{path}: column {head[j]!r} is not numeric ({e})") from None
    missing = [k for k in CALIB_KEYS_USED if k not in out]
    if missing:
        raise EsrrfError(f"{path}: missing columns {missing}")
    return out


def save_calibration_table(path, table: dict, row_numbers=True, decimals=None) -> None:
    """Write {key: array} as ImageJ's ResultsTable CSV export: a heading row (" " over the row
    numbers when row_numbers), one row per plane.  decimals=None writes shortest round-trip
    values."""
    keys = list(table)
    cols = [np.asarray(table[k], np.float64) for k in keys]
    n = len(cols[0]) if cols else 0
    if any(len(c) != n for c in cols):
        raise EsrrfError("table columns differ in length")
    fmt = (lambda v: repr(float(v))) if decimals is None else (lambda v: f"{v:.{decimals}f}")
    with open(os.fspath(path), "w") as fh:
        fh.write(",".join(([" "] if row_numbers else []) + keys) + "\n")
        for i in range(n):
            cells = ([str(i + 1)] if row_numbers else []) + [fmt(c[i]) for c in cols]
            fh.write(",".join(cells) + "\n")


def axial_offset(axial_positions) -> float:
    """LinearRegressions.linearRegressionLeastSquareNoOffset(double[]) (LinearRegressions.java:
    19-47): x_i = i - (index of the entry closest to zero, first on ties), slope = sum x y / sum
    x^2 in double."""
    y = [float(v) for v in axial_positions]
    d0, i0 = float("inf"), 0
    for i, v in enumerate(y):
        if abs(v) < d0:
            d0, i0 = abs(v), i
    XX = XY = 0.0
    for i, v in enumerate(y):
        x = float(i - i0)
        XX += x * x
        XY += x * v
    return XY / XX


def table_geometry(table: dict, width: int, height: int, magnification: int, axialOffset: float,
                   pixelSize: float) -> dict:
    """What LiveSRRF_CL.initialise derives from a table (LiveSRRF_CL.java:207-240): nPlanes,
    widthS/heightS (nSplits = 3), nPlanesM, the background level (first entry), the axial offset
    (the regression when the axial positions do not sum to zero, else the argument; Java float)
    and dimensionRatioXYvsZ = axialOffset / (1000 pixelSize) in float."""
    f32 = np.float32
    n_planes = len(table["X-shift (pixels)"])
    ap = np.asarray(table["Axial positions"], np.float64)
    off = f32(axialOffset)
    if float(ap.sum()) != 0.0:
        off = f32(axial_offset(ap))
    return {
        "nPlanes": n_planes, "widthS": int(width) // 3, "heightS": int(height) // 3,
        "nPlanesM": n_planes * int(magnification),
        "backgroundLevel": float(f32(np.asarray(table["Background level (ADC)"])[0])),
        "axialOffset": float(off),
        "dimensionRatioXYvsZ": float(off / (f32(1000) * f32(pixelSize))),
    }
