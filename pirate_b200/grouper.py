"""pirate's toy grouper on pirate_b200's outputs: per time chunk, one event per beam whose peak SNR
over all trees, DMs and times exceeds a threshold (pirate_frb/run_toy_grouper.py:15-125). Events
are decoded into trial parameters as pirate's grouper does (FrbGrouper.create_events,
pirate_frb/rpc/FrbGrouper.py:295-420). pirate's version also converts to FPGA counts and beam ids
from the network handshake's metadata; that part is left out (the network side is not part of this
library), so times are in samples since the first chunk.

The reduction runs on the GPU (pirate_b200.beam_peaks, one kernel per batch); only the per-beam
peaks (a few bytes per beam) come back to the host.
"""

import numpy as np

from . import beam_peaks

EVENT_DTYPE = np.dtype([
    ("ibeam", np.int64), ("itree", np.int64), ("idm", np.int64), ("itime", np.int64), ("snr", np.float32),
    ("token", np.uint32), ("fmin", np.int64), ("fmax", np.int64), ("tlo", np.int64), ("thi", np.int64),
    ("p", np.int64), ("freq_lo_mhz", np.float64), ("freq_hi_mhz", np.float64), ("dm", np.float64),
    ("time_samples", np.float64), ("width_samples", np.float64)])


def make_events(plan, ichunk, peak, tree, idm, itime, token, snr_threshold):
    """Events of one chunk from per-beam peaks (host arrays, one entry per beam of the whole GPU):
    beams with peak > snr_threshold, decoded with decode_argmax_batch / decode_argmax2_batch.
    time_samples = ichunk * nt_in + the decoded chunk-relative arrival time (toplevel samples,
    extrapolated to the lowest frequency of the band, so it may lie outside the chunk)."""
    if int(ichunk) < 0:
        raise ValueError("make_events: ichunk must be >= 0")
    peak = np.asarray(peak, dtype=np.float32)
    tree, idm, itime = (np.asarray(a, dtype=np.int64) for a in (tree, idm, itime))
    token = np.asarray(token).astype(np.uint32)
    sel = np.nonzero((peak > snr_threshold) & (tree >= 0))[0]
    ev = np.zeros(sel.size, dtype=EVENT_DTYPE)
    if sel.size == 0:
        return ev
    ev["ibeam"], ev["itree"], ev["idm"], ev["itime"] = sel, tree[sel], idm[sel], itime[sel]
    ev["snr"], ev["token"] = peak[sel], token[sel]
    fmin, fmax, tlo, thi, p = plan.decode_argmax_batch(token[sel], tree[sel], idm[sel], itime[sel])
    flo, fhi, dm, ts, w = plan.decode_argmax2_batch(tree[sel], fmin, fmax, tlo, thi, p)
    ev["fmin"], ev["fmax"], ev["tlo"], ev["thi"], ev["p"] = fmin, fmax, tlo, thi, p
    ev["freq_lo_mhz"], ev["freq_hi_mhz"], ev["dm"], ev["width_samples"] = flo, fhi, dm, w
    ev["time_samples"] = int(ichunk) * plan.nt_in + ts
    return ev


class ToyGrouper:
    """Consumes a GpuDedisperser's outputs chunk by chunk as pirate's toy grouper does.

    process_chunk(ichunk) acquires every batch of the chunk (consumer 'consumer_id', in seq_id order),
    reduces each batch to per-beam peaks on the GPU, releases it, and returns (events,
    coarse_snr): the decoded events above snr_threshold and every beam's peak SNR."""

    def __init__(self, dd, plan, consumer_id=0, snr_threshold=10.0, stream=None):
        import torch
        self.dd, self.plan, self.consumer_id = dd, plan, int(consumer_id)
        self.snr_threshold = float(snr_threshold)
        self.stream = stream
        self.nbatches = plan.beams_per_gpu // plan.beams_per_batch
        self.B = plan.beams_per_batch
        n = plan.beams_per_gpu
        dev = dd.device
        self._peak = torch.empty(n, dtype=torch.float32, device=dev)
        self._ints = [torch.empty(n, dtype=torch.int32, device=dev) for _ in range(4)]

    def process_chunk(self, ichunk):
        import torch
        for ib in range(self.nbatches):
            seq = int(ichunk) * self.nbatches + ib
            out = self.dd.acquire_output(self.consumer_id, seq, self.stream)
            sl = slice(ib * self.B, (ib + 1) * self.B)
            beam_peaks(out, self.stream, out=(self._peak[sl], *[a[sl] for a in self._ints]))
            self.dd.release_output(self.consumer_id, seq, self.stream)
        if self.stream is None:
            torch.cuda.synchronize(self.dd.device)
        else:
            self.stream.synchronize()
        peak = self._peak.cpu().numpy()
        tree, idm, itime, token = (a.cpu().numpy() for a in self._ints)
        events = make_events(self.plan, ichunk, peak, tree, idm, itime, token.view(np.uint32), self.snr_threshold)
        return events, peak
