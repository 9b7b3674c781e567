"""The CUDA path against pirate's OWN reference dedisperser, directly.

The committed fixtures (tests/golden/pirate_ref_fixtures.npz, written by tests/golden/make_ref_golden.py
from pirate's reference CPU sources compiled unmodified into oracle/_ref) hold sha256 digests of pirate's
float32 out_max and uint32 out_argmax for every (seq_id, tree) of the cases in
helpers.pirate_fixture_cases(). Here the same seeded inputs and weights go through the public
GpuDedisperser API (and so the C ABI and the sm_100a kernels) with float32 storage, and every output must
have exactly pirate's bytes. The cases include NaN inputs, a dispersed pulse, five primary trees run until
every delay line has wrapped (rank 12, 68 chunks), and rank 16 over 34 chunks of 2048 samples, so that the
2^16-sample delay lines wrap inside the compared run."""

import json
import os

import numpy as np
import pytest

import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pirate_ref_fixtures.npz")
CASES = H.pirate_fixture_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_gpu_matches_pirate_reference(pb2lib, case):
    z = np.load(FIX)
    meta = json.loads(bytes(z["meta_json"]).decode())[case["name"]]
    xs = H.fixture_inputs(case)
    assert H.inputs_digest(xs) == meta["inputs_sha256"]
    orc = O.OracleDedisperser(case["cfg"], 1, 32) if case["cfg"]["toplevel_tree_rank"] < 16 else None
    ws = H.fixture_weights(case, orc) if orc else _weights_from_meta(case, meta)
    _, _, gres = H.run_gpu(pb2lib, case["cfg"], xs, ws)
    bad = []
    for seq in range(len(xs)):
        for i in range(len(meta["trees"])):
            gm = gres[seq][0][i].astype(np.float32)
            ga = gres[seq][1][i]
            if H.output_digest(gm, ga) != meta["digests"][seq][i]:
                bad.append((seq, i))
    assert not bad, "%s: %d of %d (seq, tree) outputs differ from pirate's reference, first %s" % (
        case["name"], len(bad), len(xs) * len(meta["trees"]), bad[:5])


def _weights_from_meta(case, meta):
    """Weights of a case, shaped from the fixture's tree geometry (no oracle instance needed)."""
    class Shapes:
        pass
    s = Shapes()
    s.ntrees = len(meta["trees"])
    s.trees = meta["trees"]
    B = case["cfg"]["beams_per_batch"]
    s.wt_shape = lambda i: (B, s.trees[i]["ndm_wt"], s.trees[i]["nt_wt"], s.trees[i]["nprofiles"], s.trees[i]["N"])
    return H.fixture_weights(case, s)
