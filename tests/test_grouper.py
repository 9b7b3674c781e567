"""Host side of the toy grouper: batch token decoding (DedispersionPlan.decode_argmax_batch /
decode_argmax2_batch, src_pybind11/pirate_pybind11.cpp:396-409) and event building
(pirate_frb/rpc/FrbGrouper.py:295-420)."""

import numpy as np
import pytest

import helpers as H


def _plan(pb):
    return pb.DedispersionPlan(pb.DedispersionConfig.from_dict(H.toy_config(rank=8, nfreq=300, nt=512)))


def _valid_tokens(plan, rng, n):
    """n random (token, itree, idm, itime) with well-formed tokens."""
    import oracle as O
    orc = O.OracleDedisperser(H.toy_config(rank=8, nfreq=300, nt=512), 1, 32)
    out = []
    for _ in range(n):
        i = int(rng.integers(plan.ntrees))
        t = orc.trees[i]
        M, P, Dout, Dcore = t["M"], t["nprofiles"], t["nt_ds"] // t["nt_out"], t["Dcore"]
        p = int(rng.integers(P))
        dt = min(Dcore, 2 ** ((p - 1) // 3 if p else 0))
        tok = (int(rng.integers(M)) << 16) | (p << 8) | (int(rng.integers(Dout // dt)) * dt)
        out.append((tok, i, int(rng.integers(t["ndm_out"])), int(rng.integers(t["nt_out"]))))
    return out


def test_decode_batch_equals_scalar(pb2lib):
    plan = _plan(pb2lib)
    rng = np.random.default_rng(4)
    ev = _valid_tokens(plan, rng, 200)
    tok, it, idm, itm = (np.array(c) for c in zip(*ev))
    dec = plan.decode_argmax_batch(tok, it, idm, itm)
    phys = plan.decode_argmax2_batch(it, *dec)
    for k, (t, i, d, s) in enumerate(ev):
        sc = plan.decode_argmax(t, i, d, s)
        assert tuple(int(a[k]) for a in dec) == sc
        assert tuple(float(a[k]) for a in phys) == plan.decode_argmax2(i, *sc)
    assert (phys[0] < phys[1]).all() and (phys[2] >= 0).all() and (phys[4] > 0).all()


def test_decode_batch_rejects_empty_and_bad(pb2lib):
    plan = _plan(pb2lib)
    e = np.zeros(0, dtype=np.int64)
    with pytest.raises(RuntimeError):
        plan.decode_argmax_batch(np.zeros(0, np.uint32), e, e, e)
    with pytest.raises(RuntimeError):
        plan.decode_argmax2_batch(e, e, e, e, e, e)
    with pytest.raises(RuntimeError):      # itree out of range in the second element
        plan.decode_argmax_batch(np.zeros(2, np.uint32), np.array([0, plan.ntrees]), np.zeros(2), np.zeros(2))


def test_make_events(pb2lib):
    from pirate_b200.grouper import make_events
    plan = _plan(pb2lib)
    rng = np.random.default_rng(5)
    nb = 10
    ev = _valid_tokens(plan, rng, nb)
    tok, it, idm, itm = (np.array(c) for c in zip(*ev))
    peak = np.array([3, 12, 9.99, 10.0, 10.01, 50, -np.inf, 11, 0, 20], dtype=np.float32)
    it = it.copy()
    it[9] = -1                                   # no tree qualified for beam 9
    out = make_events(plan, 7, peak, it, idm, itm, tok, 10.0)
    assert list(out["ibeam"]) == [1, 4, 5, 7]
    for e in out:
        b = e["ibeam"]
        f = plan.decode_argmax(tok[b], it[b], idm[b], itm[b])
        assert (e["fmin"], e["fmax"], e["tlo"], e["thi"], e["p"]) == f
        flo, fhi, dm, ts, w = plan.decode_argmax2(it[b], *f)
        assert (e["freq_lo_mhz"], e["freq_hi_mhz"], e["dm"], e["width_samples"]) == (flo, fhi, dm, w)
        assert e["time_samples"] == 7 * plan.nt_in + ts and e["snr"] == peak[b] and e["token"] == tok[b]
    assert make_events(plan, 0, peak, it, idm, itm, tok, 100.0).size == 0
    with pytest.raises(ValueError):
        make_events(plan, -1, peak, it, idm, itm, tok, 10.0)
