"""Black-box test of DedispersionPlan.decode_argmax (src_lib/DedispersionPlan.cpp:481-543), after
pirate's own test strategy (pirate_frb/tests/test_decode_argmax.py).

For a fixed token, the oracle's eval_tokens is a linear functional of the tree-domain input with
nonnegative coefficients (all weights 1). So for a nonnegative probe it is nonzero exactly when the
probe meets the trial's support. decode_argmax reports the support as channels [fmin, fmax] and
exclusive trailing edges tlo, thi (the last summed samples of channels fmin and fmax). Probes:
  membership: constant input on one channel f: every cell of every token of a subband is > 0 when
              fmin <= f <= fmax, and exactly 0 otherwise;
  P1 / P2:    one-hot at (fmin, tlo - 1) / (fmax, thi - 1): the decoded cell is > 0;
  P3:         indicator of {f < fmin} + {f > fmax} + {f = fmin, t >= tlo} + {f = fmax, t >= thi}:
              the decoded cell is exactly 0.
The probes go in as tree-domain input (ReferenceDedisperser's tree_domain_input), the space
decode_argmax reports in."""

import random
import zlib

import numpy as np
import pytest

import helpers as H
import oracle as O


def _pt(et, w, wt_dm, wt_t, dm_ds=0, t_ds=0):
    return dict(num_early_triggers=et, max_width=w, dm_downsampling=dm_ds, time_downsampling=t_ds,
                wt_dm_downsampling=wt_dm, wt_time_downsampling=wt_t)


CONFIGS = {
    "r6_et": H.toy_config(rank=6, nfreq=100, nt=256, subbands=[1, 1, 1], beams_per_gpu=6, beams_per_batch=6,
                          primary_trees=[_pt(1, 8, 8, 16), _pt(0, 4, 4, 16)]),
    "r7_three": H.toy_config(rank=7, nfreq=150, nt=512, subbands=[2, 2, 1], beams_per_gpu=6, beams_per_batch=6,
                             primary_trees=[_pt(0, 16, 16, 16), _pt(1, 8, 16, 16), _pt(0, 4, 8, 16)]),
    "r5_w32": H.toy_config(rank=5, nfreq=60, nt=256, subbands=[0, 1, 1], beams_per_gpu=6, beams_per_batch=6,
                           primary_trees=[_pt(2, 32, 8, 32)]),
    "r6_fp16": H.toy_config(rank=6, nfreq=90, nt=256, dtype="float16", subbands=[1, 2, 1], beams_per_gpu=6,
                            beams_per_batch=6, primary_trees=[_pt(1, 16, 16, 16), _pt(0, 2, 4, 16)]),
}


def _setup(pb, cfg):
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    orc = O.OracleDedisperser(cfg, 0, 32)
    rtop = cfg["toplevel_tree_rank"]
    nt = cfg["time_samples_per_chunk"]
    # Chunks enough to hold every trial's full support, ending in the chunk that is evaluated.
    depth = 0
    for t in orc.trees:
        w = t["max_width"]
        depth = max(depth, (2 ** (rtop - t["et_level"]) + 4 * w + max(2 * w, 4)) * 2 ** t["ipri"])
    return plan, orc, depth // nt + 2


def _run(orc, C, fill):
    """Dedisperses C chunks of tree-domain input; fill(c, x) writes chunk c into the zeroed x."""
    ws = [np.ones(orc.wt_shape(i), np.float32) for i in range(orc.ntrees)]
    for c in range(C):
        x = np.zeros((orc.B, 2 ** orc.rank, orc.nt_in), np.float32)
        fill(c, x)
        orc.dedisperse(0, x, ws, tree_domain=True)
    return ws


def _eval(orc, ws, itree, token_of_beam):
    t = orc.trees[itree]
    toks = np.zeros((orc.B, t["ndm_out"], t["nt_out"]), np.uint32)
    for b, tok in token_of_beam.items():
        toks[b] = tok
    return orc.eval_tokens(itree, toks, ws[itree])


def _kinfo(orc, i):
    t = orc.trees[i]
    return t["M"], t["nprofiles"], t["nt_ds"] // t["nt_out"], t["Dcore"]


def _dt(p, Dcore):
    return min(Dcore, 2 ** ((p - 1) // 3 if p else 0))


def _bands(plan, orc):
    """Per tree: (token, fmin, fmax) for the first multiplet of each decoded band, and the first and
    last multiplet of each band."""
    bands, edges = [], []
    for i in range(plan.ntrees):
        first, last = {}, {}
        for m in range(orc.trees[i]["M"]):
            fmin, fmax = plan.decode_argmax(m << 16, i, 0, 0)[:2]
            first.setdefault((fmin, fmax), m)
            last[(fmin, fmax)] = m
        bands.append([(m << 16, a, b) for (a, b), m in first.items()])
        edges.append(sorted(set(first.values()) | set(last.values())))
    return bands, edges


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_decode_argmax_bad_arguments(pb2lib, name):
    plan, orc, _ = _setup(pb2lib, CONFIGS[name])
    for i in range(plan.ntrees):
        M, P, Dout, Dcore = _kinfo(orc, i)
        t = plan.trees[i]
        bad = [(M << 16, i, 0, 0), (P << 8, i, 0, 0), (0, plan.ntrees, 0, 0), (0, i, t.ndm_out, 0),
               (0, i, 0, t.nt_out), (0, i, -1, 0)]
        if Dout < 256:
            bad.append((Dout, i, 0, 0))
        for p in range(P):
            if _dt(p, Dcore) > 1:
                bad.append(((p << 8) | 1, i, 0, 0))
                break
        for args in bad:
            with pytest.raises(RuntimeError):
                plan.decode_argmax(*args)
        for m in range(M):          # every well-formed token decodes
            for p in range(P):
                for tt in range(0, Dout, _dt(p, Dcore)):
                    fmin, fmax, tlo, thi, pp = plan.decode_argmax((m << 16) | (p << 8) | tt, i, t.ndm_out - 1, t.nt_out - 1)
                    assert 0 <= fmin <= fmax < 2 ** CONFIGS[name]["toplevel_tree_rank"] and tlo <= thi and pp == p


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_decode_argmax_membership(pb2lib, name):
    plan, orc, C = _setup(pb2lib, CONFIGS[name])
    nchan = 2 ** orc.rank
    bands, _ = _bands(plan, orc)
    chans = set()
    for tb in bands:
        for _, a, b in tb:
            chans.update(c for c in (a - 1, a, b, b + 1) if 0 <= c < nchan)
    rng = random.Random(zlib.crc32(name.encode()))
    chans.update(rng.sample(range(nchan), 4))
    chans = sorted(chans)
    for i0 in range(0, len(chans), orc.B):
        batch = chans[i0:i0 + orc.B]

        def fill(c, x):
            for b, f in enumerate(batch):
                x[b, f, :] = 1.0

        ws = _run(orc, C, fill)
        for i in range(plan.ntrees):
            for tok, a, b in bands[i]:
                out = _eval(orc, ws, i, {k: tok for k in range(len(batch))})
                for k, f in enumerate(batch):
                    if a <= f <= b:
                        assert (out[k] > 0).all(), (name, i, hex(tok), a, b, f)
                    else:
                        assert (out[k] == 0).all(), (name, i, hex(tok), a, b, f)


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_decode_argmax_edges(pb2lib, name):
    plan, orc, C = _setup(pb2lib, CONFIGS[name])
    nt = orc.nt_in
    _, edges = _bands(plan, orc)
    rng = random.Random(1000 + zlib.crc32(name.encode()))
    tuples = []
    for _ in range(12):
        i = rng.randrange(plan.ntrees)
        M, P, Dout, Dcore = _kinfo(orc, i)
        t = plan.trees[i]
        m = rng.choice(edges[i] + [rng.randrange(M)])
        p = rng.choice([0, P - 1, rng.randrange(P)])
        dt = _dt(p, Dcore)
        tt = rng.choice([0, Dout // dt - 1, rng.randrange(Dout // dt)]) * dt
        idm = rng.choice([0, t.ndm_out - 1, rng.randrange(t.ndm_out)])
        ito = rng.choice([0, t.nt_out - 1, rng.randrange(t.nt_out)])
        tuples.append((i, (m << 16) | (p << 8) | tt, idm, ito))

    per_run = orc.B // 3
    ce = C - 1                      # the evaluated chunk
    for j0 in range(0, len(tuples), per_run):
        run = tuples[j0:j0 + per_run]
        dec = [plan.decode_argmax(tok, i, idm, ito) for i, tok, idm, ito in run]
        for fmin, fmax, tlo, thi, _ in dec:
            assert 0 <= fmin <= fmax < 2 ** orc.rank and tlo <= thi <= nt and ce * nt + tlo - 1 >= 0

        def fill(c, x):
            t0 = c * nt
            for k, (fmin, fmax, tlo, thi, _) in enumerate(dec):
                glo, ghi = ce * nt + tlo, ce * nt + thi          # exclusive global trailing edges
                if t0 <= glo - 1 < t0 + nt:
                    x[3 * k, fmin, glo - 1 - t0] = 1.0
                if t0 <= ghi - 1 < t0 + nt:
                    x[3 * k + 1, fmax, ghi - 1 - t0] = 1.0
                x[3 * k + 2, :fmin, :] = 1.0
                x[3 * k + 2, fmax + 1:, :] = 1.0
                if glo - t0 < nt:
                    x[3 * k + 2, fmin, max(glo - t0, 0):] = 1.0
                if ghi - t0 < nt:
                    x[3 * k + 2, fmax, max(ghi - t0, 0):] = 1.0

        ws = _run(orc, C, fill)
        for k, (i, tok, idm, ito) in enumerate(run):
            out = _eval(orc, ws, i, {3 * k: tok, 3 * k + 1: tok, 3 * k + 2: tok})
            msg = (name, i, hex(tok), idm, ito, dec[k])
            assert out[3 * k, idm, ito] > 0, ("P1", msg)
            assert out[3 * k + 1, idm, ito] > 0, ("P2", msg)
            assert out[3 * k + 2, idm, ito] == 0, ("P3", msg)
