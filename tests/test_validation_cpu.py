"""Argument validation of the C ABI without a device: every invalid call of
the reference library's recorded error cases (tests/golden/errors.json, made
by running the reference) returns the reference's code, and the calls that
return before any work (m = 0, n = 0, an sbs with k = 0) return success and
leave C untouched, on a host-processing-unit context and host buffers. The
order of the checks follows pgemm_ssb_host.cpp:151-171,
pgemm_sbs_host.cpp:171-193 and check_gemm_param.hpp:36-50; the cases that do
device work (the valid calls, and k = 0 with C to be scaled by beta) are left
to the GPU parity tests."""
import json

import numpy as np
import pytest

import golden_cases as gc
from capi import SplaCAPI

DEVICE_WORK = {"ssb ok", "sbs ok", "gemm ok", "gemm ldc small is accepted",
               "ssb null A k zero"}


@pytest.fixture(scope="module")
def ours():
    import spla_b200
    if not spla_b200.LIB_PATH.exists():
        pytest.skip("libspla.so not built")
    return SplaCAPI(spla_b200.LIB_PATH)


def test_error_codes_without_a_device(ours):
    cases = json.loads((gc.GOLDEN / "errors.json").read_text())
    ctx = ours.ctx(0)  # SPLA_PU_HOST
    _, dist = ours.block_cyclic(1, 1, 64, 64)
    A = np.ones(1000)
    ran = 0
    for c in cases:
        if c["name"] in DEVICE_WORK:
            continue
        a = c["args"]
        C = np.ones(1000)
        p = lambda key: A if a.get(key, 1) else None  # noqa: E731
        cp = C if a.get("C", 1) else None
        d = np.float64
        if c["call"] == "ssb":
            rc = ours.pgemm_ssb(d, a["m"], a["n"], a["k"], a["opA"], 1.0, p("A"), a["lda"], p("B"),
                                a["ldb"], 0.0, cp, a["ldc"], a["ro"], a["co"], dist, ctx)
        elif c["call"] == "sbs":
            rc = ours.pgemm_sbs(d, a["m"], a["n"], a["k"], 1.0, p("A"), a["lda"], p("B"), a["ldb"],
                                a["bro"], a["bco"], dist, 0.0, cp, a["ldc"], ctx)
        else:
            rc = ours.gemm(d, a["opA"], a["opB"], a["m"], a["n"], a["k"], 1.0, p("A"), a["lda"],
                           p("B"), a["ldb"], 0.0, cp, a["ldc"], ctx)
        assert rc == c["code"], c
        assert np.all(C == 1.0), c  # rejected or returned early: C untouched
        ran += 1
    assert ran >= 20
