"""GPU parity tests of the 2-D bicubic path (liveSRRF.cl) and the 3-D MFM path (live3DSRRF.cl)
through the C ABI.  Same bar as the FHT path: every output slice within 1e-4 of its dynamic
range of the oracle (the FP32 restatement, pinned bit-exactly to the reference kernels)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4


def run(esrrf, frames, M, fwhm, S, intw=True, mp=True, fht=False, calib=None, drift=None,
        frames_per_launch=0, chunks=None, kernel="fused"):
    eng = esrrf.LiveSRRF_CL()
    n = frames.shape[0]
    eng.initialise(frames.shape[-1], frames.shape[-2], M, fwhm, S, n, n, intWeighting=intw,
                   doMPmapCorrection=mp, doFHTinterpolation=fht, calibTable3DSRRF=calib,
                   framesPerLaunch=frames_per_launch, kernel=kernel)
    try:
        eng.resetFramePosition()
        if drift is not None:
            eng.loadDriftXYGPUbuffer(*drift)
        if chunks is None:
            assert not eng.calculateSRRF(frames)
        else:
            s = 0
            for c in chunks:
                assert not eng.calculateSRRF(frames[s:s + c])
                s += c
        return eng.readSRRFbuffer().copy(), eng
    finally:
        eng.release()


def assert_close(got, ref, what):
    got = got.reshape(4, -1)
    ref = ref.reshape(4, -1)
    for k in range(4):
        e = rel_err(got[k], ref[k])
        assert e < TOL, f"{what} slice {k}: {e:.3g}"


def tile_planes(planes, roi):
    """Camera frames [n][3h][3w] holding plane z at the 3x3 tile `roi[z]`."""
    n, P, h, w = planes.shape
    cam = np.zeros((n, 3 * h, 3 * w), np.float32)
    for z in range(P):
        i, j = int(roi[z]) % 3, int(roi[z]) // 3
        cam[:, j * h:(j + 1) * h, i * w:(i + 1) * w] = planes[:, z]
    return cam


def calib(P, theta, sx, sy, roi, coeff=None, bg=0.0):
    return {"X-shift (pixels)": sx, "Y-shift (pixels)": sy, "Theta (degrees)": theta,
            "Axial positions": np.zeros(P, np.float32), "ROI #": roi,
            "Intensity scaling": np.ones(P, np.float32) if coeff is None else coeff,
            "Background level (ADC)": np.full(P, bg, np.float32)}


@pytest.mark.parametrize("name", golden_names("bic"))
def test_bic_golden(esrrf_mod, name):
    g = load_golden(name)
    drift = (g["drift_x"], g["drift_y"]) if "drift_x" in g else None
    got, _ = run(esrrf_mod, g["raw"], int(g["magnification"]), float(g["fwhm"]),
                 int(g["sensitivity"]), bool(g["int_weighting"]), bool(g["mp_correction"]),
                 drift=drift)
    assert_close(got, g["out"], name)


def test_bic_chunked_u16(esrrf_mod, oracle_mod):
    from esrrf import synth
    raw = synth.small_stack(41, 11, 28, 24)
    ref = oracle_mod.bic_block(raw.astype(np.float32), 3, 1.5, 2)
    got, _ = run(esrrf_mod, raw, 3, 1.5, 2, chunks=[4, 4, 3], frames_per_launch=3)
    assert_close(got, ref, "bic chunked")


@pytest.mark.parametrize("M,fwhm,S", [(2, 1.0, 1), (3, 2.5, 2), (4, 1.5, 2), (5, 2.0, 1),
                                      (8, 1.5, 1), (4, 4.0, 1)])
def test_bic_tabulated_taps_radii(esrrf_mod, oracle_mod, M, fwhm, S):
    """The tabulated bicubic kernel (launches without drift: per-phase tap lists, per-pixel sums
    of weights at the edges, slab staging, CTAs that overhang a 37 x 29 frame) across
    magnifications -- odd M, whose phase centres are not exact in FP32, included -- and radii,
    against the oracle and against the per-pixel kernel (kernel="plain")."""
    from esrrf import synth
    raw = synth.small_stack(60 + M, 6, 29, 37)
    ref = oracle_mod.bic_block(raw.astype(np.float32), M, fwhm, S)
    got, _ = run(esrrf_mod, raw, M, fwhm, S)
    assert_close(got, ref, f"bic tabulated M{M} r{fwhm}")
    plain, _ = run(esrrf_mod, raw, M, fwhm, S, kernel="plain")
    assert_close(got, plain, f"bic tabulated vs per-pixel M{M} r{fwhm}")


def test_bic_radius_beyond_the_tables_uses_per_pixel_kernel(esrrf_mod, oracle_mod):
    """A radius whose slab rows exceed the tabulated kernel's reach (fwhm 20: 138 positions per
    row) builds no tables: every launch takes the per-pixel kernel, against the oracle."""
    from esrrf import synth
    raw = synth.small_stack(88, 4, 40, 44).astype(np.float32)
    ref = oracle_mod.bic_block(raw, 2, 20.0, 1)
    got, _ = run(esrrf_mod, raw, 2, 20.0, 1)
    assert_close(got, ref, "bic fwhm 20")


def test_bic_drift_uses_per_pixel_kernel(esrrf_mod, oracle_mod):
    """A launch with drift takes the per-pixel kernel (the tap geometry then moves per frame);
    the launch without drift after it the tabulated one; both against the oracle."""
    from esrrf import synth
    raw = synth.small_stack(77, 8, 32, 40).astype(np.float32)
    dx = np.zeros(8, np.float32)
    dy = np.zeros(8, np.float32)
    dx[:4] = np.linspace(0.0, 0.3, 4)
    dy[:4] = np.linspace(0.1, -0.2, 4)
    ref = oracle_mod.bic_block(raw, 4, 1.5, 2, drift_x=dx, drift_y=dy)
    got, _ = run(esrrf_mod, raw, 4, 1.5, 2, drift=(dx, dy), frames_per_launch=4)
    assert_close(got, ref, "bic drift then none")


@pytest.mark.parametrize("name", golden_names("3d"))
def test_3d_golden(esrrf_mod, name):
    g = load_golden(name)
    P = g["raw"].shape[1]
    roi = np.array([4, 0, 8, 5][:P], np.float32)
    cam = tile_planes(g["raw"], roi)
    got, _ = run(esrrf_mod, cam, int(g["magnification"]), float(g["fwhm"]), int(g["sensitivity"]),
                 bool(g["int_weighting"]), bool(g["mp_correction"]),
                 calib=calib(P, g["theta"], g["shift_x"], g["shift_y"], roi))
    assert_close(got, g["out"], name)


def test_3d_mfm_normalisation_and_nine_planes(esrrf_mod, oracle_mod):
    """Nine planes read from a 3x3 camera frame with background and per-plane scaling, checked
    against the oracle's host-side reshape + 3-D block (the 9-plane MFM layout, at 48x48)."""
    from esrrf import synth
    P, h, w, n, M = 9, 48, 48, 5, 3
    planes = synth.small_stack(42, n, h, w, planes=P).astype(np.float32)
    roi = np.array([4, 0, 1, 2, 3, 5, 6, 7, 8], np.float32)
    coeff = np.linspace(0.8, 1.2, P).astype(np.float32)
    bg = 90.0
    cam = tile_planes(planes * coeff[None, :, None, None] + bg, roi)
    theta = np.linspace(-1.0, 1.0, P).astype(np.float32)
    sx = np.linspace(-0.3, 0.3, P).astype(np.float32)
    sy = np.linspace(0.2, -0.2, P).astype(np.float32)
    ref_planes = oracle_mod.mfm_reshape(cam, P, roi, coeff, bg)
    ref = oracle_mod.block3d(ref_planes, M, 1.5, 1, theta, sx, sy, mp_correction=False)
    got, _ = run(esrrf_mod, cam, M, 1.5, 1, mp=False, calib=calib(P, theta, sx, sy, roi, coeff, bg))
    assert got.shape == (4 * P * M, h * M, w * M)
    assert_close(got, ref, "mfm 9 planes")


@pytest.mark.parametrize("M,fwhm,S,form", [(2, 2.0, 2, "zblock"), (4, 1.0, 1, "zblock"),
                                            (3, 2.5, 1, "zblock"), (5, 1.5, 1, "zblock"),
                                            (3, 1.5, 2, "zb"), (2, 2.0, 2, "zb"),
                                            (3, 1.5, 2, "voxel"), (4, 1.0, 1, "voxel")])
def test_3d_tabulated_taps_radii(esrrf_mod, oracle_mod, monkeypatch, M, fwhm, S, form):
    """Blocks without drift take the tabulated-tap 3-D kernels (taps listed per sub-pixel phase,
    zero-halo unit-gradient field, tabulated sums of weights), z-blocked (the M z-phases of a
    cell in one thread; the field staged in shared memory one plane offset at a time, or read
    through the L1 cache with ESRRF_RGC3D=zb) or one voxel per thread (ESRRF_RGC3D=voxel):
    checked against the oracle at several magnifications and radii, on volumes where most voxels
    have taps beyond a face."""
    from esrrf import synth
    if form in ("voxel", "zb"):
        monkeypatch.setenv("ESRRF_RGC3D", form)
    else:
        monkeypatch.delenv("ESRRF_RGC3D", raising=False)
    P, h, w, n = (5, 40, 36, 3) if M < 5 else (3, 20, 18, 3)
    planes = synth.small_stack(7 + M, n, h, w, planes=P).astype(np.float32)
    roi = np.array([4, 0, 8, 5, 1], np.float32)
    zeros = np.zeros(P, np.float32)
    ref = oracle_mod.block3d(planes, M, fwhm, S, zeros, zeros, zeros, mp_correction=False)
    got, _ = run(esrrf_mod, tile_planes(planes, roi), M, fwhm, S, mp=False,
                 calib=calib(P, zeros, zeros, zeros, roi))
    assert_close(got, ref, f"3d M{M} fwhm{fwhm} {form}")


def test_3d_drift_per_voxel_kernel(esrrf_mod, oracle_mod):
    """Frames with drift keep the per-voxel 3-D kernel (the reference's arithmetic per tap)."""
    from esrrf import synth
    P, h, w, n, M = 3, 20, 18, 4, 3
    planes = synth.small_stack(31, n, h, w, planes=P).astype(np.float32)
    roi = np.array([4, 0, 8], np.float32)
    zeros = np.zeros(P, np.float32)
    rng = np.random.default_rng(5)
    dx = rng.uniform(-0.4, 0.4, n).astype(np.float32)
    dy = rng.uniform(-0.4, 0.4, n).astype(np.float32)
    ref = oracle_mod.block3d(planes, M, 1.5, 1, zeros, zeros, zeros, mp_correction=False,
                             drift_x=dx, drift_y=dy)
    got, _ = run(esrrf_mod, tile_planes(planes, roi), M, 1.5, 1, mp=False,
                 calib=calib(P, zeros, zeros, zeros, roi), drift=(dx, dy))
    assert_close(got, ref, "3d drift")


def test_3d_calibration_table_from_file(esrrf_mod, tmp_path):
    """The table read from its text export (the reference takes a path, LiveSRRF_CL.java:210-222)
    gives the same reconstruction as the same table passed as a mapping, and initialise derives
    the axial offset from the axial positions as the reference does."""
    from esrrf import calibration as C
    from esrrf import synth
    P, h, w, n, M = 9, 48, 48, 4, 2
    planes = synth.small_stack(7, n, h, w, planes=P).astype(np.float32)
    roi = np.array([4, 0, 1, 2, 3, 5, 6, 7, 8], np.float64)
    table = C.make_calibration_table(
        shift_x=np.linspace(-0.3, 0.3, P), shift_y=np.linspace(0.2, -0.2, P), theta=np.linspace(-1, 1, P),
        axial_positions=np.linspace(-400, 400, P) + 3.0, nominal_axial_positions=np.linspace(-400, 400, P),
        roi_locations=roi, intensity_scaling=np.linspace(0.8, 1.2, P), background_level=90.0)
    cam = tile_planes(planes * np.asarray(table["Intensity scaling"], np.float32)[None, :, None, None] + 90.0,
                      table["ROI #"].astype(np.float32))
    path = tmp_path / "beads - MFM_CalibrationTable.csv"
    C.save_calibration_table(path, table)
    a, _ = run(esrrf_mod, cam, M, 1.5, 1, mp=False, calib={k: table[k].astype(np.float32) for k in table})
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(cam.shape[-1], cam.shape[-2], M, 1.5, 1, n, n, doMPmapCorrection=False,
                   doFHTinterpolation=False, calibTable3DSRRF=str(path), axialOffset=250.0, pixelSize=0.1)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(cam)
        b = eng.readSRRFbuffer().copy()
        assert eng.axialOffset == float(np.float32(C.axial_offset(table["Axial positions"])))
        assert eng.nPlanes == P
    finally:
        eng.release()
    np.testing.assert_array_equal(a, b)


def test_3d_read_aligned_pixels(esrrf_mod, oracle_mod):
    """readAlignedPixels (LiveSRRF_CL.java:881-906): the aligned planes of the first frame of the
    last group on the GPU.  With no rotation they are the split, background-subtracted, scaled
    planes (the oracle's reshape), moved by the integer calibration shifts."""
    from esrrf import synth
    P, h, w, n, M = 9, 40, 48, 5, 2
    planes = synth.small_stack(5, n, h, w, planes=P).astype(np.float32)
    roi = np.array([4, 0, 1, 2, 3, 5, 6, 7, 8], np.float32)
    coeff = np.linspace(0.8, 1.2, P).astype(np.float32)
    bg = 90.0
    cam = tile_planes(planes * coeff[None, :, None, None] + bg, roi)
    ref = oracle_mod.mfm_reshape(cam, P, roi, coeff, bg)[0]
    zeros = np.zeros(P, np.float32)
    sx = np.array([0, 1, -2, 0, 3, 0, -1, 2, 0], np.float32)
    sy = np.array([0, 0, 1, -2, 0, 2, -1, 0, 1], np.float32)
    for shx, shy in ((zeros, zeros), (sx, sy)):
        eng = esrrf_mod.LiveSRRF_CL()
        eng.initialise(w * 3, h * 3, M, 1.5, 1, n, n, doMPmapCorrection=False,
                       doFHTinterpolation=False, calibTable3DSRRF=calib(P, zeros, shx, shy, roi, coeff, bg))
        try:
            eng.resetFramePosition()
            assert not eng.calculateSRRF(cam)
            got = eng.readAlignedPixels()
        finally:
            eng.release()
        assert got.shape == (P, h, w)
        for z in range(P):
            ix, iy = int(shx[z]), int(shy[z])
            # aligned(x, y) = plane(x - sx, y - sy); compare where the source stays 2 px inside
            ys = slice(max(iy, 0) + 2, h + min(iy, 0) - 2)
            xs = slice(max(ix, 0) + 2, w + min(ix, 0) - 2)
            src = np.roll(ref[z], (iy, ix), axis=(0, 1))
            np.testing.assert_allclose(got[z][ys, xs], src[ys, xs], rtol=1e-6, atol=1e-6 * np.abs(ref).max(),
                                       err_msg=f"plane {z}")


def test_2d_read_aligned_pixels_is_a_state_error(esrrf_mod):
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(32, 32, 2, 1.5, 1, 4, 4, doFHTinterpolation=False)
    try:
        with pytest.raises(esrrf_mod.EsrrfError):
            eng.readAlignedPixels()
    finally:
        eng.release()


@pytest.mark.parametrize("is3d", [False, True])
def test_read_mp_maps(esrrf_mod, is3d):
    """readMPmaps (LiveSRRF_CL.java:909-935): each cumulant's mean over the image at every
    sub-pixel phase of the uncorrected reconstruction; the corrected output is the uncorrected one
    divided by its phase's entry."""
    from esrrf import synth
    M, n = 3, 6
    if is3d:
        P, h, w = 4, 24, 32
        planes = synth.small_stack(11, n, h, w, planes=P).astype(np.float32)
        roi = np.array([0, 1, 2, 3], np.float32)
        zeros = np.zeros(P, np.float32)
        frames = tile_planes(planes, roi)
        cal = calib(P, np.linspace(-0.5, 0.5, P).astype(np.float32), zeros, zeros, roi)
    else:
        P, h, w = 1, 36, 44
        frames = synth.small_stack(11, n, h, w).astype(np.float32)
        cal = None
    raw, _ = run(esrrf_mod, frames, M, 1.5, 2, mp=False, calib=cal)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(frames.shape[-1], frames.shape[-2], M, 1.5, 2, n, n, doMPmapCorrection=True,
                   doFHTinterpolation=False, calibTable3DSRRF=cal)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(frames)
        corr = eng.readSRRFbuffer().copy()
        maps = eng.readMPmaps()
    finally:
        eng.release()
    PM = P * M if is3d else 1
    raw = raw.reshape(4, PM, h * M, w * M).astype(np.float64)
    corr = corr.reshape(4, PM, h * M, w * M)
    assert maps.shape == (3 * (M if is3d else 1), M, M)
    ref = np.empty((3, M if is3d else 1, M, M))
    for c in range(3):
        for pz in range(M if is3d else 1):
            for py in range(M):
                for px in range(M):
                    ref[c, pz, py, px] = raw[c, pz::M, py::M, px::M].mean()
    for c in range(3):
        np.testing.assert_allclose(maps.reshape(ref.shape)[c], ref[c], rtol=2e-5,
                                   atol=1e-5 * np.abs(ref[c]).max(), err_msg=f"map {c}")
    for c in range(3):
        m = ref[c][(np.arange(PM) % M)[:, None, None] if is3d else np.zeros((1, 1, 1), int),
                   (np.arange(h * M) % M)[None, :, None], (np.arange(w * M) % M)[None, None, :]]
        assert rel_err(corr[c], (raw[c] / m).astype(np.float32)) < TOL, f"cumulant {c}"


def test_fht_read_mp_maps_is_a_state_error(esrrf_mod):
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(32, 32, 2, 1.5, 1, 4, 4, doMPmapCorrection=True, doFHTinterpolation=True)
    try:
        with pytest.raises(esrrf_mod.EsrrfError):
            eng.readMPmaps()
    finally:
        eng.release()
