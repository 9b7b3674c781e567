"""Generates tests/golden/pirate_ref_fixtures.npz: outputs of pirate's OWN reference CPU dedisperser
(src_lib/ReferenceDedisperser.cpp, compiled unmodified from pirate's source tree into oracle/_ref by
'make -C oracle ref') on the seeded cases of tests/helpers.pirate_fixture_cases().

    python tests/golden/make_ref_golden.py PIRATE_SRC

For every case it records:
  - the sha256 of the case's inputs (so a change of the input generator is detected),
  - per (seq_id, tree) the sha256 of pirate's out_max (float32) and out_argmax (uint32) bytes,
  - the full outputs of cases whose outputs are small, for diagnostics;
  - for the pulses of tests/helpers.pulse_fixture_cases(), pirate's SinglePulse sparse representation
    (src_lib/simpulse.cpp; MKL's complex-to-real DFT supplied by oracle/ksgpu_shim/mkl_dfti.h).
It runs sophistication 1 (two-stage trees with lagged downsampling, pirate's GPU algorithm) and checks
that sophistication 0 (one-stage trees on plainly downsampled input) and 2 (MegaRingbuf ring buffers)
give the same bytes on the smaller cases. Every tree's Dcore is min(time_downsampling, 8), the rule of
pirate's production kernel registry.
"""

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import helpers as H        # noqa: E402
import oracle as O         # noqa: E402
import pirate_ref as PR    # noqa: E402

OUT = os.path.join(HERE, "pirate_ref_fixtures.npz")
FULL_LIMIT = 400_000       # store full outputs of cases with at most this many output elements


def run_case(case, soph):
    cfg = case["cfg"]
    xs = H.fixture_inputs(case)
    orc = O.OracleDedisperser(cfg, 1, 32)     # shapes only
    ws = H.fixture_weights(case, orc)
    ref = PR.PirateReferenceDedisperser(cfg, sophistication=soph, dcore_max=8)
    digests, outs = [], []
    for x in xs:
        m, a = ref.dedisperse(x, [w[0] for w in ws])
        digests.append([H.output_digest(m[i], a[i]) for i in range(ref.ntrees)])
        outs.append((m, a))
    return H.inputs_digest(xs), digests, outs, ref


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_ref_golden.py PIRATE_SRC")
    PR.build(sys.argv[1])
    PR.self_tests(5)
    arrays, meta = {}, {}
    for case in H.pirate_fixture_cases():
        t0 = time.time()
        din, digests, outs, ref = run_case(case, 1)
        nelts = sum(m.size for m, _ in [(mm, aa) for s in outs for mm, aa in zip(*s)])
        soph_checked = []
        if case["cfg"]["toplevel_tree_rank"] <= 12:
            for soph in (0, 2):
                _, d2, _, _ = run_case(case, soph)
                assert d2 == digests, "%s: sophistication %d differs from sophistication 1" % (case["name"], soph)
                soph_checked.append(soph)
        meta[case["name"]] = dict(inputs_sha256=din, digests=digests, sophistication_equal=soph_checked,
                                  full=bool(nelts <= FULL_LIMIT), trees=ref.trees)
        if nelts <= FULL_LIMIT:
            for s, (m, a) in enumerate(outs):
                for i in range(len(m)):
                    arrays["%s/%d/%d/max" % (case["name"], s, i)] = m[i]
                    arrays["%s/%d/%d/arg" % (case["name"], s, i)] = a[i]
        print("%-20s %3d seqs, %d trees, %.1f s, sophistication 0/2 checked: %s" %
              (case["name"], len(digests), len(ref.trees), time.time() - t0, soph_checked), flush=True)
    # SinglePulse construction (src_lib/simpulse.cpp), MKL's c2r DFT supplied by oracle/ksgpu_shim/mkl_dfti.h.
    for pc in H.pulse_fixture_cases():
        sp = PR.PiratePulse(freq_edges_MHz=pc["edges"], freq_variances=pc["var"], **pc["params"])
        meta[pc["name"]] = dict(kind="pulse", it_start=int(sp.it_start), it_end=int(sp.it_end))
        for k in ("freq_it0", "freq_nt", "freq_sd_off", "sparse_data"):
            arrays["%s/%s" % (pc["name"], k)] = getattr(sp, k)
        print("%-20s %d samples in [%d, %d)" % (pc["name"], sp.sparse_data.size, sp.it_start, sp.it_end), flush=True)
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
