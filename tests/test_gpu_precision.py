"""Error of each cumulant against the FP64 oracle on the 512x512 M4 workload's settings
(radius 1.5, S2, AVG/VAR/TAC2/INT) over a 128x128 crop of its stack, next to the error of the
reference's own FP32 kernel arithmetic (the restatement, bit-exact to it) against the same FP64
oracle.  Writes the figures as JSON to the file named by ESRRF_PRECISION_JSON when it is set."""
import json
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_cumulant_errors_against_fp64(esrrf_mod, oracle_mod):
    from esrrf import synth
    raw = synth.make_stack("fht512", frames=20)[:, 192:320, 192:320]
    M, fwhm, S = 4, 1.5, 2
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(128, 128, M, fwhm, S, 20, 20)
    try:
        eng.resetFramePosition()
        eng.calculateSRRF(raw)
        gpu = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    interp = oracle_mod.fht_interpolate(raw.astype(np.float32), M)
    f64 = oracle_mod.fht_block(interp, M, fwhm, S, precision="f64")
    f32 = oracle_mod.fht_block(interp, M, fwhm, S, precision="f32")
    names = ["AVG", "VAR", "TAC2", "INT"]
    res = {n: {"gpu_vs_fp64": rel_err(gpu[k], f64[k]), "ref_fp32_vs_fp64": rel_err(f32[k], f64[k])}
           for k, n in enumerate(names)}
    out = os.environ.get("ESRRF_PRECISION_JSON")
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    for n in names:
        assert res[n]["gpu_vs_fp64"] < 1e-4, (n, res[n])
