"""The learned candidate sifter behind the threshold peak finder (no pirate counterpart; the plain
threshold stays the fallback and the yardstick of the sifter's recall and false-alarm rate).

- ``Sifter``: the MLP 1728 -> 256 -> 128 -> 1 (bf16 weights, FP32 accumulation) with its CUDA forward,
  backward and Adam kernels (``libpirate_b200.so``: ``pb2_sifter_*``).
- ``CandidateGenerator``: runs a GpuDedisperser with the candidate stage on synthetic events (N(0,1)
  noise, simulated FRB pulses from pirate's simpulse model, RFI) and collects each event's candidate
  patch, peak and label.
- ``recall_at_far``: recall of a score at a fixed false-alarm fraction of the negative events.
"""

import ctypes
import math

import numpy as np

from . import _check, _stream_ptr, lib

PATCH_SHAPE = (9, 32, 6)
PATCH_LEN = 9 * 32 * 6


class Sifter:
    """pb2_sifter: the MLP, its fp32 master parameters and Adam state on one GPU."""

    def __init__(self, device=0, max_batch=1024, seed=0):
        h = ctypes.c_void_p()
        _check(lib().pb2_sifter_create(int(device), int(max_batch), int(seed), ctypes.byref(h)))
        self._h = h
        self.device = "cuda:%d" % int(device)
        self.max_batch = int(max_batch)

    @staticmethod
    def nparams():
        n = ctypes.c_long()
        _check(lib().pb2_sifter_nparams(ctypes.byref(n)))
        return n.value

    @staticmethod
    def split(params):
        """Views W1 (256, 1728), b1, W2 (128, 256), b2, W3 (1, 128), b3 of a flat parameter vector."""
        shapes = [(256, PATCH_LEN), (256,), (128, 256), (128,), (1, 128), (1,)]
        out, o = [], 0
        for s in shapes:
            n = int(np.prod(s))
            out.append(params[o:o + n].reshape(s))
            o += n
        return out

    def get_params(self):
        p = np.empty(self.nparams(), np.float32)
        _check(lib().pb2_sifter_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams()
        _check(lib().pb2_sifter_set_params(self._h, p.ctypes.data))

    def _prep(self, patches):
        import torch
        x = patches.reshape(-1, PATCH_LEN)
        if x.dtype != torch.float16 or not x.is_cuda or not x.is_contiguous():
            x = x.to(device=self.device, dtype=torch.float16).contiguous()
        return x

    def forward(self, patches, stream=None):
        """Logits (float32 CUDA tensor) of patches (n, 9, 32, 6) or (n, 1728); batched by max_batch."""
        import torch
        x = self._prep(patches)
        out = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        for i in range(0, x.shape[0], self.max_batch):
            n = min(self.max_batch, x.shape[0] - i)
            _check(lib().pb2_sifter_forward(self._h, x[i:i + n].data_ptr(), n, out[i:i + n].data_ptr(),
                                            _stream_ptr(stream)))
        return out

    def gradients(self, patches, labels, stream=None):
        """(loss, gradient vector) of the mean binary cross-entropy over one batch (n <= max_batch)."""
        import torch
        x = self._prep(patches)
        y = torch.as_tensor(labels, dtype=torch.float32, device=x.device).contiguous()
        g = np.empty(self.nparams(), np.float32)
        loss = ctypes.c_double()
        _check(lib().pb2_sifter_gradients(self._h, x.data_ptr(), y.data_ptr(), x.shape[0], g.ctypes.data,
                                          ctypes.byref(loss), _stream_ptr(stream)))
        return loss.value, g

    def train_step(self, patches, labels, lr, stream=None):
        import torch
        x = self._prep(patches)
        y = torch.as_tensor(labels, dtype=torch.float32, device=x.device).contiguous()
        loss = ctypes.c_double()
        _check(lib().pb2_sifter_train_step(self._h, x.data_ptr(), y.data_ptr(), x.shape[0], float(lr),
                                           ctypes.byref(loss), _stream_ptr(stream)))
        return loss.value

    def fit(self, patches, labels, epochs=20, batch=512, lr=1e-3, seed=0, log=None):
        """Adam on shuffled mini-batches of device patches (n, 1728) fp16 and labels (n,)."""
        import torch
        x = self._prep(patches)
        y = torch.as_tensor(labels, dtype=torch.float32, device=x.device)
        n = x.shape[0]
        g = torch.Generator(device="cpu")
        g.manual_seed(seed)
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(x.device)
            tot, cnt = 0.0, 0
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * ep / max(epochs, 1)))   # cosine schedule
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                tot += self.train_step(x[idx].contiguous(), y[idx].contiguous(), rate)
                cnt += 1
            hist.append(tot / max(cnt, 1))
            if log:
                log("epoch %d: loss %.4f" % (ep, hist[-1]))
        return hist

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().pb2_sifter_destroy(self._h)
            except Exception:
                pass
            self._h = None


def recall_at_far(scores_pos, scores_neg, far):
    """Recall of the positive events at the smallest threshold whose false-alarm fraction among the
    negative events is <= far (an event without a candidate has score -inf and is never detected).
    Returns (recall, threshold, false alarms)."""
    pos = np.asarray(scores_pos, dtype=np.float64)
    neg = np.sort(np.asarray(scores_neg, dtype=np.float64))[::-1]
    k = int(math.floor(far * neg.size))
    # detections need a score strictly above the (k+1)-th highest negative score
    thr = neg[k] if k < neg.size else -np.inf
    det = np.isfinite(pos) & (pos > thr)
    fa = int(np.sum(np.isfinite(neg) & (neg > thr)))
    return (float(det.mean()) if pos.size else 0.0), float(thr), fa


class CandidateGenerator:
    """Synthetic events through the dedispersion pipeline with the candidate stage (no sifter).

    One event = one beam over two consecutive chunks. Its kind is drawn per event:
      pulse  -- a pirate simpulse pulse (DM uniform in dm_range, intrinsic width log-uniform over
                width_range samples, scattering time log-uniform over tau_range samples at 1 GHz,
                SNR log-uniform over snr_range), arriving at the bottom of the band inside the second
                chunk, taken from a bank of precomputed pulses shifted in time;
      noise  -- N(0, 1) only;
      rfi    -- N(0, 1) plus RFI in both chunks: zero-DM broadband spikes and narrowband sinusoids, either
                the precision study's mix (spikes at 1e-3 per sample at 20 sigma per channel, 1% of
                channels with 10-sigma sinusoids) or weaker versions whose dedispersed SNR overlaps
                the pulses'.
    The event's candidate is the stronger of its two chunks' per-beam peaks (6 sigma threshold); its
    label is 1 for pulses. The dedisperser's state is cleared before every event, so that no event sees
    an earlier one through the delay lines. Inputs are float16 N(0, 1) samples written into the dedisperser's input
    slot on the GPU; peak-finding weights are pirate's analytic ones for unit variance.
    """

    def __init__(self, cfg, seed=0, threshold=6.0, nbank=96, dm_range=(30.0, 100.0), width_range=(1.0, 32.0),
                 tau_range=(0.1, 16.0), snr_range=(6.0, 30.0), kinds=(0.5, 0.2, 0.3), log=None):
        import pirate_b200 as pb
        from .simpulse import SinglePulse, config_freq_edges
        self.pb = pb
        self.cfg = dict(cfg)
        self.plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
        self.dd = pb.GpuDedisperser(self.plan, cuda_device_id=0, num_consumers=1)
        self.dd.allocate()
        self.dd.fill_analytic_weights(np.ones(self.plan.nfreq))
        self.dd.enable_sifter(threshold, None)
        self.B = self.plan.beams_per_batch
        self.F = self.plan.nfreq
        self.T = self.plan.nt_in
        self.dt_ms = float(cfg["time_sample_ms"])
        self.rng = np.random.default_rng(seed)
        self.kinds = np.asarray(kinds, dtype=np.float64) / np.sum(kinds)
        self.snr_range, self.log = snr_range, log
        edges = config_freq_edges(self.cfg)
        var = np.ones(self.F)
        # Bank of unit-SNR pulses (time shifts and SNR scaling are applied at injection), built on host
        # threads (the pulse constructor releases the GIL).
        from concurrent.futures import ThreadPoolExecutor
        import os
        pars = []
        for i in range(nbank):
            dm = self.rng.uniform(*dm_range)
            wid = math.exp(self.rng.uniform(math.log(width_range[0]), math.log(width_range[1])))
            tau = math.exp(self.rng.uniform(math.log(tau_range[0]), math.log(tau_range[1])))
            pars.append(dict(dm=dm, width=wid, tau=tau))

        def make(m):
            # sm is the scattering time in ms at 1 GHz; tau is in samples at the band centre (600 MHz)
            sm = m["tau"] * self.dt_ms * (600.0 / 1000.0) ** 4.4
            return SinglePulse(dm=m["dm"], sm=sm, intrinsic_width=m["width"] * self.dt_ms * 1e-3, spectral_index=0.0,
                               undispersed_arrival_time_sec=0.0, time_sample_ms=self.dt_ms, snr=1.0,
                               freq_edges_MHz=edges, freq_variances=var)
        with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as ex:
            sps = list(ex.map(make, pars))
        self.bank = list(zip(sps, pars))
        self.seq = 0
        self.stream = None

    def _rfi(self, x, b, strong):
        """Adds RFI to beam b of the (B, F, T) float16 input slot x (in place)."""
        import torch
        F, T = self.F, self.T
        rng = self.rng
        if strong:
            nspk = rng.poisson(1e-3 * T)
            amp_spike = 20.0
            nch = max(1, int(round(0.01 * F)))
            amp_sin = 10.0
        else:
            nspk = int(rng.integers(1, 4)) if rng.random() < 0.7 else 0
            amp_spike = math.exp(rng.uniform(math.log(0.04), math.log(0.3)))
            nch = int(rng.integers(max(1, F // 1000), max(2, F // 100))) if (nspk == 0 or rng.random() < 0.3) else 0
            amp_sin = math.exp(rng.uniform(math.log(1.0), math.log(10.0)))
        if nspk:
            ts = torch.as_tensor(rng.integers(0, T, nspk), device=x.device)
            x[b][:, ts] += amp_spike
        if nch:
            ch = torch.as_tensor(rng.choice(F, nch, replace=False), device=x.device)
            per = torch.as_tensor(rng.uniform(4.0, 256.0, nch), device=x.device, dtype=torch.float32)
            ph = torch.as_tensor(rng.uniform(0, 2 * np.pi, nch), device=x.device, dtype=torch.float32)
            t = torch.arange(T, device=x.device, dtype=torch.float32)
            wave = amp_sin * torch.sin(2 * np.pi * t[None, :] / per[:, None] + ph[:, None])
            x[b][ch] = (x[b][ch].float() + wave).to(x.dtype)

    def _run_chunk(self, events, half):
        """One chunk of every beam; returns the candidate stage's host arrays."""
        import torch
        dd = self.dd
        s = self.seq
        x = dd.acquire_input(s)
        x.normal_()
        ichunk = s // (self.plan.beams_per_gpu // self.B)
        for b, ev in enumerate(events):
            if ev["kind"] == "pulse":
                sp = self.bank[ev["bank"]][0]
                # pulse coordinates: chunk start = ichunk*T - shift
                sp.inject(x[b], ichunk * self.T - ev["shift"], weight=ev["snr"])
            elif ev["kind"] == "rfi":
                self._rfi(x, b, ev["strong"])
        dd.release_input_and_launch_dd_kernels(s)
        out = dd.acquire_output(0, s, sync=True)
        c = out.candidates
        res = dict(peak=c["peak"].cpu().numpy().copy(), valid=c["valid"].cpu().numpy().copy(),
                   tree=c["tree"].cpu().numpy().copy(), patches=c["patches"].reshape(self.B, PATCH_LEN).cpu().numpy().copy())
        dd.release_output(0, s)
        self.seq += 1
        return res

    def generate(self, nevents):
        """Returns dict of arrays over nevents events: label, kind (0 pulse, 1 noise, 2 rfi), peak
        (-inf if no candidate), valid, patch (n, 1728) float16, snr/dm/width/tau of pulses (NaN otherwise)."""
        nb = self.plan.beams_per_gpu // self.B
        assert nb == 1, "one batch per chunk"
        out = dict(label=[], kind=[], peak=[], valid=[], patch=[], snr=[], dm=[], width=[], tau=[])
        while len(out["label"]) < nevents:
            events = []
            for b in range(self.B):
                k = self.rng.choice(3, p=self.kinds)
                ev = dict(kind=("pulse", "noise", "rfi")[k])
                if k == 0:
                    ib = int(self.rng.integers(len(self.bank)))
                    sp, meta = self.bank[ib]
                    snr = math.exp(self.rng.uniform(math.log(self.snr_range[0]), math.log(self.snr_range[1])))
                    # bottom-of-band arrival at a uniform position of the second chunk
                    ichunk1 = self.seq // nb + 1
                    target = ichunk1 * self.T + int(self.rng.integers(self.T // 8, self.T - self.T // 8))
                    ev.update(bank=ib, snr=snr, shift=target - int(sp.it_end), meta=meta)
                elif k == 2:
                    ev.update(strong=bool(self.rng.random() < 0.3))
                events.append(ev)
            # A fresh history for every event pair: no event sees an earlier event's pulse or RFI through
            # the delay lines (the downsampled trees' lags reach tens of chunks back).
            self.dd.zero_state()
            r0 = self._run_chunk(events, 0)
            r1 = self._run_chunk(events, 1)
            for b, ev in enumerate(events):
                p0 = r0["peak"][b] if r0["valid"][b] else -np.inf
                p1 = r1["peak"][b] if r1["valid"][b] else -np.inf
                use = r1 if p1 >= p0 else r0
                pk = max(p0, p1)
                out["label"].append(1.0 if ev["kind"] == "pulse" else 0.0)
                out["kind"].append({"pulse": 0, "noise": 1, "rfi": 2}[ev["kind"]])
                out["peak"].append(pk)
                out["valid"].append(int(np.isfinite(pk)))
                out["patch"].append(use["patches"][b])
                m = ev.get("meta", {})
                out["snr"].append(ev.get("snr", np.nan))
                out["dm"].append(m.get("dm", np.nan))
                out["width"].append(m.get("width", np.nan))
                out["tau"].append(m.get("tau", np.nan))
            if self.log and len(out["label"]) % (self.B * 64) == 0:
                self.log("%d events" % len(out["label"]))
        res = {k: np.asarray(v[:nevents]) for k, v in out.items()}
        res["patch"] = res["patch"].astype(np.float16)
        return res
