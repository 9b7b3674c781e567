"""The precision study (tests/precision_study.py) at a small size, with bounds: float32, float16 and
bfloat16 storage against the FP64 oracle on noise with narrowband and zero-DM broadband RFI, rank 12
from 4096 channels, the benchmark's 5-tree layout, one beam, four chunks. The bounds hold the
measured errors with margin (at rank 16, 8 beams x 64 chunks, the same study gives 7.2e-3 sigma and
1.3e-3 relative for float16)."""

import pytest

import precision_study as PS

pytestmark = pytest.mark.gpu

# dtype: (max |err| in sigma on outputs within 10 sigma, max relative error, min token agreement)
BOUNDS = {"float32": (1e-4, 1e-5, 0.9999), "float16": (1e-2, 4e-3, 0.99), "bfloat16": (8e-2, 3e-2, 0.95)}


def test_precision_with_rfi(pb2lib):
    r = PS.run(rank=12, nfreq=4096, beams=1, chunks=4, workers=1, log=lambda s: None)
    print(PS.table(r))
    for dt, (tol_abs, tol_rel, min_agree) in BOUNDS.items():
        d = r["dtypes"][dt]
        assert d["nonfinite"] == 0, dt
        assert d["classes"][0]["max_abs_sigma"] <= tol_abs, (dt, d["classes"][0])
        assert d["max_rel"] <= tol_rel, (dt, d["max_rel"])
        assert d["token_agreement"] >= min_agree, (dt, d["token_agreement"])
        # every token disagreement is within the storage error of its magnitude class
        assert d["max_margin_over_bound"] <= 1.0, (dt, d["max_margin_over_bound"])
