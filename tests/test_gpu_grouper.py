"""pirate_b200.beam_peaks (one kernel) and ToyGrouper on the GPU, against a numpy restatement of
pirate's toy-grouper loop (pirate_frb/run_toy_grouper.py:79-116, cupy max/argmax per tree, then a
strictly-greater update across trees). numpy's max and argmax follow the same rules as cupy's: NaN
propagates through max, argmax returns the first maximal position."""

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def toy_peaks_numpy(maxes, args):
    """maxes[i]: (B, ndm, nt) float arrays; args[i]: the uint32 tokens. Per beam: (peak, tree, idm,
    itime, token), as pirate's per-batch loop computes them."""
    B = maxes[0].shape[0]
    peak = np.full(B, -np.inf, np.float32)
    tree = np.full(B, -1, np.int64)
    idm = np.full(B, -1, np.int64)
    itime = np.full(B, -1, np.int64)
    tok = np.zeros(B, np.uint32)
    for i, (m, a) in enumerate(zip(maxes, args)):
        _, ndm, nt = m.shape
        flat = m.reshape(B, ndm * nt)
        with np.errstate(invalid="ignore"):
            bmax = flat.max(axis=1).astype(np.float32)
            barg = flat.argmax(axis=1)
            upd = bmax > peak
        peak = np.where(upd, bmax, peak)
        tree = np.where(upd, i, tree)
        idm = np.where(upd, barg // nt, idm)
        itime = np.where(upd, barg % nt, itime)
        tok = np.where(upd, a.reshape(B, ndm * nt)[np.arange(B), barg], tok)
    return peak, tree, idm, itime, tok


def _check(got, want):
    peak, tree, idm, itime, tok = (g.cpu().numpy() for g in got)
    wp, wt, wd, wi, wk = want
    assert np.array_equal(peak, wp)
    assert np.array_equal(tree, wt) and np.array_equal(idm[wt >= 0], wd[wt >= 0])
    assert np.array_equal(itime[wt >= 0], wi[wt >= 0])
    assert np.array_equal(tok.view(np.uint32)[wt >= 0], wk[wt >= 0])
    assert (idm[wt < 0] == -1).all() and (itime[wt < 0] == -1).all()


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_beam_peaks_planted(pb2lib, dtype):
    """Ties within a tree and across trees, a NaN-poisoned tree, an all -inf beam, shapes on the
    vector path (multiples of 8) and off it."""
    import torch
    tdt = getattr(torch, dtype)
    rng = np.random.default_rng(8)
    B = 7
    shapes = [(64, 32), (33, 7), (128, 16), (5, 3)]
    maxes, args = [], []
    for ndm, nt in shapes:
        m = rng.integers(-20, 20, size=(B, ndm, nt)).astype(np.float32) / 4   # exact in all three dtypes
        maxes.append(m)
        args.append(rng.integers(0, 2 ** 32, size=(B, ndm, nt), dtype=np.uint64).astype(np.uint32))
    maxes[0][0, 3, 5] = maxes[0][0, 9, 1] = 100.0       # beam 0: tie inside tree 0
    maxes[1][1, :, :] = -30
    maxes[0][1, 2, 2] = maxes[2][1, 7, 3] = 80.0        # beam 1: tie across trees 0 and 2
    maxes[2][2, 0, 0] = 90.0
    maxes[2][2, 5, 5] = np.nan                          # beam 2: tree 2 poisoned by NaN
    for m in maxes:
        m[3] = -np.inf                                  # beam 3: nothing qualifies
    maxes[3][4, 4, 2] = 1000.0                          # beam 4: winner in the scalar-path tree
    dm = [torch.from_numpy(m).to(tdt).cuda() for m in maxes]
    da = [torch.from_numpy(a.view(np.int32)).cuda() for a in args]
    got = pb2lib.beam_peaks((dm, da))
    torch.cuda.synchronize()
    want = toy_peaks_numpy([m.to(torch.float32).cpu().numpy() for m in dm], args)
    _check(got, want)
    assert got[1][3].item() == -1 and got[0][3].item() == -np.inf


def test_toy_grouper_on_dedisperser_outputs(pb2lib):
    """ToyGrouper over several chunks of a float16 plan with 2 batches: per-beam peaks equal the
    numpy loop on the same outputs, and the events are the thresholded, decoded peaks."""
    import torch
    from pirate_b200.grouper import ToyGrouper, make_events
    cfg = H.toy_config(rank=8, nfreq=300, nt=512, dtype="float16", beams_per_gpu=4, beams_per_batch=2)
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    # both batches of a chunk are launched before they are consumed: two output slots
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=2, nbatches_out=2)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    grouper = ToyGrouper(dd, plan, consumer_id=0, snr_threshold=3.5)
    xs = H.make_inputs(cfg, 3, seed=12)
    nb = 2
    for ichunk in range(3):
        for ib in range(nb):
            with dd.get_input() as x:
                x.copy_(torch.from_numpy(xs[ichunk * nb + ib]).to(x.dtype).to(x.device))
        # consumer 1 copies the outputs to the host for the numpy restatement
        ref = [[], [], [], [], []]
        for ib in range(nb):
            with dd.get_output(1, sync=True) as out:
                w = toy_peaks_numpy([m.float().cpu().numpy() for m in out.out_max],
                                    [a.cpu().numpy().view(np.uint32) for a in out.out_argmax])
            for k in range(5):
                ref[k].append(w[k])
        ref = [np.concatenate(r) for r in ref]
        events, peak = grouper.process_chunk(ichunk)
        assert np.array_equal(peak, ref[0])
        want = make_events(plan, ichunk, *ref, 3.5)
        assert np.array_equal(events, want)


@pytest.mark.parametrize("dtype", ["float32", "float16"])
def test_candidate_stage_peaks(pb2lib, dtype):
    """The candidate stage's split per-beam reduction (many blocks per tree and beam, then one warp per
    beam) gives the numpy loop's peaks on real outputs, NaN inputs included."""
    import torch
    cfg = H.toy_config(rank=9, nfreq=300, nt=512, dtype=dtype, beams_per_gpu=6, beams_per_batch=6)
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    dd.enable_sifter(threshold=4.0)
    xs = H.make_inputs(cfg, 4, seed=44)
    xs[2][3, :, 10:20] = np.nan      # beam 3 of chunk 2: NaN in every channel
    for x in xs:
        with dd.get_input() as a:
            a.copy_(torch.from_numpy(x).to(a.dtype).to(a.device))
        with dd.get_output(0, sync=True) as out:
            want = toy_peaks_numpy([m.float().cpu().numpy() for m in out.out_max],
                                   [a.cpu().numpy().view(np.uint32) for a in out.out_argmax])
            c = out.candidates
            got = (c["peak"], c["tree"], c["idm"], c["itime"], c["token"])
            _check(got, want)
            valid = c["valid"].cpu().numpy()
            assert np.array_equal(valid == 1, want[0] >= 4.0)
