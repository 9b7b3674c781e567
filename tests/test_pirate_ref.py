"""Parity of the restated oracle (oracle/refdd.cpp) with pirate's OWN reference dedisperser.

pirate's reference CPU sources (src_lib/ReferenceDedisperser.cpp, ReferenceTree.cpp, ReferenceLagbuf.cpp,
ReferenceLaggedDownsamplingKernel.cpp, TreeGriddingKernel.cu, PeakFindingKernel.cu, DedispersionPlan.cpp,
MegaRingbuf.cpp and the rest listed in oracle/Makefile) were compiled unmodified into oracle/_ref and run
on the seeded cases of helpers.pirate_fixture_cases(); tests/golden/make_ref_golden.py committed their
outputs as sha256 digests per (seq_id, tree) (full arrays for the small cases). These tests require the
oracle's float32 outputs to have exactly those bytes: out_max bit for bit and every argmax token. Where
oracle/_ref is built, they also run pirate's own self-tests and compare on fresh random configurations.
"""

import json
import os

import numpy as np
import pytest

import helpers as H
import oracle as O
import pirate_ref as PR

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pirate_ref_fixtures.npz")


def _fixtures():
    z = np.load(FIX)
    meta = json.loads(bytes(z["meta_json"]).decode())
    return z, meta


CASES = H.pirate_fixture_cases()


def test_fixture_covers_every_case():
    _, meta = _fixtures()
    ded = sorted(k for k, v in meta.items() if v.get("kind") != "pulse")
    assert ded == sorted(c["name"] for c in CASES)
    assert sorted(k for k, v in meta.items() if v.get("kind") == "pulse") == sorted(c["name"] for c in H.pulse_fixture_cases())
    # The small cases were also checked equal across pirate's three reference sophistications.
    assert all(meta[c["name"]]["sophistication_equal"] == [0, 2] for c in CASES if c["cfg"]["toplevel_tree_rank"] <= 12)


CPU_CASES = [c for c in CASES if c.get("cpu", True)]


@pytest.mark.parametrize("case", CPU_CASES, ids=[c["name"] for c in CPU_CASES])
def test_oracle_matches_pirate_reference(case):
    z, meta = _fixtures()
    m = meta[case["name"]]
    xs = H.fixture_inputs(case)
    assert H.inputs_digest(xs) == m["inputs_sha256"], "the fixture's inputs are no longer reproduced"
    orc = O.OracleDedisperser(case["cfg"], 1, 32)
    assert [dict(t) for t in orc.trees] == m["trees"], "tree geometry differs from pirate's plan"
    ws = H.fixture_weights(case, orc)
    nb = case["cfg"]["beams_per_gpu"] // case["cfg"]["beams_per_batch"]
    for seq, x in enumerate(xs):
        om, oa = orc.dedisperse(seq % nb, x, [w[0] for w in ws])
        for i in range(orc.ntrees):
            got = H.output_digest(om[i].astype(np.float32), oa[i])
            if got == m["digests"][seq][i]:
                continue
            msg = "%s seq %d tree %d: oracle output differs from pirate's reference" % (case["name"], seq, i)
            if m["full"]:
                pm = z["%s/%d/%d/max" % (case["name"], seq, i)]
                pa = z["%s/%d/%d/arg" % (case["name"], seq, i)]
                msg += " (out_max differs at %d entries, tokens at %d)" % (
                    int((pm.astype(np.float64) != om[i]).sum()), int((pa != oa[i]).sum()))
            pytest.fail(msg)


needs_ref = pytest.mark.skipif(not PR.available(), reason="oracle/_ref not built (make -C oracle ref PIRATE_SRC=...)")


@needs_ref
def test_pirate_self_tests():
    """pirate's ReferenceTree::test_basics / test_subbands and ReferenceLagbuf::test_random."""
    PR.self_tests(3)


@needs_ref
@pytest.mark.parametrize("seed", range(4))
def test_oracle_matches_pirate_on_random_configs(seed):
    """Fresh random plans (ranks 5-11, up to 3 primary trees, early triggers, subbands, time
    downsampling, several beams and batches): the oracle's fp32 outputs equal pirate's bit for bit,
    for pirate's sophistications 1 and 2 (ring buffers), and for the oracle's sophistication 0."""
    rng = np.random.default_rng(1000 + seed)
    rank = int(rng.integers(5, 12))
    npri = int(rng.integers(1, 4))
    nt = int(2 ** rng.integers(7, 10)) * (2 ** (npri - 1))
    sb_len = int(rng.integers(1, min(rank // 2, 4) + 1))
    sb = [int(rng.integers(0, 3)) for _ in range(sb_len - 1)] + [1]
    pts = []
    for ip in range(npri):
        net = int(rng.integers(0, 2)) if rank - ip >= 6 else 0
        w = int(2 ** rng.integers(0, 6))
        pts.append((net, w, 0))
    bpb = int(rng.integers(1, 3))
    cfg = H.toy_config(rank=rank, nfreq=int(rng.integers(2 ** (rank - 2), 2 ** (rank + 1))), nt=nt, subbands=sb,
                       beams_per_gpu=bpb * int(rng.integers(1, 3)), beams_per_batch=bpb,
                       primary_trees=H._prim(rank, pts, 16))
    try:
        orc1 = O.OracleDedisperser(cfg, 1, 32)
    except RuntimeError as e:
        pytest.skip("configuration rejected: %s" % e)
    orc0 = O.OracleDedisperser(cfg, 0, 32)
    refs = [PR.PirateReferenceDedisperser(cfg, sophistication=s) for s in (1, 2)]
    ws = H.make_weights(orc1, seed=seed)
    nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
    xs = H.make_inputs(cfg, 4, seed=seed)
    for seq, x in enumerate(xs):
        outs = [orc1.dedisperse(seq % nb, x, [w[0] for w in ws]), orc0.dedisperse(seq % nb, x, [w[0] for w in ws])]
        outs += [r.dedisperse(x, [w[0] for w in ws]) for r in refs]
        for i in range(orc1.ntrees):
            d = [H.output_digest(np.asarray(o[0][i], dtype=np.float32), o[1][i]) for o in outs]
            assert len(set(d)) == 1, "seq %d tree %d: digests %s (oracle 1, oracle 0, pirate 1, pirate 2)" % (seq, i, d)
