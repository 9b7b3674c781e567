"""pirate_b200: B200-native real-time FRB dedispersion (tree gridding, lagged downsampling,
two-stage tree dedispersion, lag staging and peak finding), behind pirate's
DedispersionConfig / DedispersionPlan / GpuDedisperser interface.

The compute path is libpirate_b200.so (hand-written sm_100a kernels behind the C ABI of
include/pirate_b200.h); this module is a thin ctypes mirror of pirate's pybind11 classes
(src_pybind11/pirate_pybind11.cpp:128-593, pirate_frb/GpuDedisperser.py:123-197).
There is no CPU fallback: if the library cannot be loaded, every entry point raises.
"""

import contextlib
import ctypes
import os

import numpy as np

__all__ = ["DedispersionConfig", "DedispersionPlan", "GpuDedisperser", "Outputs", "PfAvarApproximation", "beam_peaks",
           "dequantize", "lib", "LIB_PATH"]

HERE = os.path.dirname(os.path.abspath(__file__))
# The in-tree build; PB2_LIBRARY names another build of the same library (for example one made with
# different compile options) to load instead.
LIB_PATH = os.environ.get("PB2_LIBRARY") or os.path.join(HERE, "libpirate_b200.so")
MAX_TREES = 64

_lib = None


class _TreeInfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_long) for k in (
        "primary_tree_index", "early_trigger_level", "amb_rank", "dd_rank", "nt_ds",
        "ndm_out", "nt_out", "ndm_wt", "nt_wt", "nprofiles", "Dcore",
        "max_width", "dm_downsampling", "time_downsampling", "wt_dm_downsampling", "wt_time_downsampling",
        "nsubbands", "nmultiplets", "pf_rank")] + [
        ("dm_min", ctypes.c_double), ("dm_max", ctypes.c_double), ("trigger_frequency", ctypes.c_double)]


class _DdParams(ctypes.Structure):
    _fields_ = [("cuda_device_id", ctypes.c_int), ("nbatches_out", ctypes.c_long), ("nbatches_wt", ctypes.c_long),
                ("num_consumers", ctypes.c_long), ("synchronous", ctypes.c_int), ("initial_chunk", ctypes.c_long),
                ("release_timeout_ms", ctypes.c_long)]


class _Outputs(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int), ("nbeams", ctypes.c_long), ("ichunk_zero_based", ctypes.c_long),
                ("ichunk_fpga_based", ctypes.c_long), ("ibeam", ctypes.c_long), ("ntrees", ctypes.c_long),
                ("ndm_out", ctypes.c_long * MAX_TREES), ("nt_out", ctypes.c_long * MAX_TREES),
                ("out_max", ctypes.c_void_p * MAX_TREES), ("out_argmax", ctypes.c_void_p * MAX_TREES),
                ("cand_peak", ctypes.c_void_p), ("cand_tree", ctypes.c_void_p), ("cand_idm", ctypes.c_void_p),
                ("cand_itime", ctypes.c_void_p), ("cand_valid", ctypes.c_void_p), ("cand_token", ctypes.c_void_p),
                ("patches", ctypes.c_void_p), ("scores", ctypes.c_void_p)]


def lib():
    """Loads libpirate_b200.so (built in-tree by pirate_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("pirate_b200: %s is missing; build it with 'python -m pirate_b200.build'" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    vp, lp, cp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), ctypes.c_char_p
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "pb2_last_error": (cp, []),
        "pb2_version": (cp, []),
        "pb2_config_from_yaml": (ctypes.c_int, [cp, ctypes.POINTER(vp)]),
        "pb2_config_from_yaml_string": (ctypes.c_int, [cp, ctypes.POINTER(vp)]),
        "pb2_config_to_yaml": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_long, lp]),
        "pb2_config_channel_map": (ctypes.c_int, [vp, dp, ctypes.c_long]),
        "pb2_config_delay_to_frequency": (ctypes.c_int, [vp, ctypes.c_double, dp]),
        "pb2_config_frequency_to_delay": (ctypes.c_int, [vp, ctypes.c_double, dp]),
        "pb2_config_dm_per_unit_delay": (ctypes.c_int, [vp, dp]),
        "pb2_config_destroy": (None, [vp]),
        "pb2_plan_create": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
        "pb2_plan_destroy": (None, [vp]),
        "pb2_plan_to_yaml": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_long, lp]),
        "pb2_plan_ntrees": (ctypes.c_int, [vp, lp]),
        "pb2_plan_tree_info": (ctypes.c_int, [vp, ctypes.c_long, ctypes.POINTER(_TreeInfo)]),
        "pb2_plan_stage1_ranks": (ctypes.c_int, [vp, lp, lp, ctypes.c_long]),
        "pb2_plan_decode_argmax": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.c_long, ctypes.c_long, ctypes.c_long, lp]),
        "pb2_plan_decode_argmax2": (ctypes.c_int, [vp, ctypes.c_long, lp, dp]),
        "pb2_plan_steady_state_it0": (ctypes.c_int, [vp, ctypes.c_long, lp, ctypes.c_long]),
        "pb2_plan_decode_argmax_batch": (ctypes.c_int, [vp, ctypes.c_long, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "pb2_plan_decode_argmax2_batch": (ctypes.c_int, [vp, ctypes.c_long, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "pb2_beam_peaks": (ctypes.c_int, [ctypes.POINTER(_Outputs), vp, vp, vp, vp, vp, vp]),
        "pb2_plan_tree_subbands": (ctypes.c_int, [vp, ctypes.c_long, lp, lp, ctypes.c_long]),
        "pb2_plan_pf_variances": (ctypes.c_int, [vp, dp, ctypes.c_long, ctypes.POINTER(dp), lp, ctypes.c_long]),
        "pb2_dd_fill_analytic_weights": (ctypes.c_int, [vp, dp, ctypes.c_long]),
        "pb2_dd_create": (ctypes.c_int, [vp, ctypes.POINTER(_DdParams), ctypes.POINTER(vp)]),
        "pb2_dd_allocate": (ctypes.c_int, [vp]),
        "pb2_dd_device_bytes": (ctypes.c_int, [vp, lp]),
        "pb2_dd_host_bytes": (ctypes.c_int, [vp, lp]),
        "pb2_dd_acquire_input": (ctypes.c_int, [vp, ctypes.c_long, vp, ctypes.POINTER(vp), lp]),
        "pb2_dd_release_input": (ctypes.c_int, [vp, ctypes.c_long, vp]),
        "pb2_dd_acquire_input_int4": (ctypes.c_int, [vp, ctypes.c_long, vp, ctypes.POINTER(vp), ctypes.POINTER(vp), lp]),
        "pb2_dequantize": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, ctypes.c_long, ctypes.c_long, ctypes.c_long, vp]),
        "pb2_dd_acquire_output": (ctypes.c_int, [vp, ctypes.c_long, ctypes.c_long, vp, ctypes.c_int, ctypes.POINTER(_Outputs)]),
        "pb2_dd_release_output": (ctypes.c_int, [vp, ctypes.c_long, ctypes.c_long, vp]),
        "pb2_dd_fill_weights": (ctypes.c_int, [vp, ctypes.c_long, vp, ctypes.c_long]),
        "pb2_dd_stop": (ctypes.c_int, [vp]),
        "pb2_dd_kernels_per_batch": (ctypes.c_int, [vp, lp]),
        "pb2_dd_algorithmic_bytes": (ctypes.c_int, [vp, dp]),
        "pb2_dd_enable_timing": (ctypes.c_int, [vp, ctypes.c_int]),
        "pb2_dd_kernel_times": (ctypes.c_int, [vp, dp, lp]),
        "pb2_dd_destroy": (None, [vp]),
        "pb2_sifter_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_long, ctypes.c_uint64, ctypes.POINTER(vp)]),
        "pb2_sifter_destroy": (None, [vp]),
        "pb2_sifter_nparams": (ctypes.c_int, [lp]),
        "pb2_sifter_set_params": (ctypes.c_int, [vp, vp]),
        "pb2_sifter_get_params": (ctypes.c_int, [vp, vp]),
        "pb2_sifter_forward": (ctypes.c_int, [vp, vp, ctypes.c_long, vp, vp]),
        "pb2_sifter_gradients": (ctypes.c_int, [vp, vp, vp, ctypes.c_long, vp, dp, vp]),
        "pb2_sifter_train_step": (ctypes.c_int, [vp, vp, vp, ctypes.c_long, ctypes.c_float, dp, vp]),
        "pb2_dd_enable_sifter": (ctypes.c_int, [vp, ctypes.c_float, vp]),
        "pb2_dd_zero_state": (ctypes.c_int, [vp, vp]),
        "pb2_dd_time": (ctypes.c_int, [vp, ctypes.c_long, dp]),
        "pb2_batched_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_long, ctypes.c_int, ctypes.POINTER(vp)]),
        "pb2_batched_allocate": (ctypes.c_int, [vp]),
        "pb2_batched_ngroups": (ctypes.c_int, [vp, lp]),
        "pb2_batched_device_bytes": (ctypes.c_int, [vp, lp]),
        "pb2_batched_fill_weights": (ctypes.c_int, [vp, ctypes.c_long, ctypes.c_long, vp, ctypes.c_long]),
        "pb2_batched_fill_analytic_weights": (ctypes.c_int, [vp, ctypes.c_long, dp, ctypes.c_long]),
        "pb2_batched_input": (ctypes.c_int, [vp, ctypes.c_long, ctypes.POINTER(vp), lp]),
        "pb2_batched_outputs": (ctypes.c_int, [vp, ctypes.c_long, ctypes.POINTER(_Outputs)]),
        "pb2_batched_step": (ctypes.c_int, [vp, vp]),
        "pb2_batched_reset": (ctypes.c_int, [vp, vp]),
        "pb2_batched_set_schedule": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_int]),
        "pb2_batched_autotune": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_long, lp]),
        "pb2_batched_time_steps": (ctypes.c_int, [vp, ctypes.c_int, vp, dp]),
        "pb2_batched_kernels_per_step": (ctypes.c_int, [vp, lp]),
        "pb2_batched_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().pb2_last_error().decode())


def _yaml_out(fn, handle):
    n = ctypes.c_long(0)
    _check(fn(handle, None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value)
    _check(fn(handle, buf, n.value, ctypes.byref(n)))
    return buf.value.decode()


def _stream_ptr(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream   # torch.cuda.Stream


class DedispersionConfig:
    """pirate's DedispersionConfig (include/pirate/DedispersionConfig.hpp:21-194): same YAML keys."""

    def __init__(self, handle):
        self._h = handle
        import yaml
        self._d = yaml.safe_load(self.to_yaml_string())

    @staticmethod
    def from_yaml(path):
        h = ctypes.c_void_p()
        _check(lib().pb2_config_from_yaml(os.fsencode(path), ctypes.byref(h)))
        return DedispersionConfig(h)

    @staticmethod
    def from_yaml_string(text):
        h = ctypes.c_void_p()
        _check(lib().pb2_config_from_yaml_string(text.encode(), ctypes.byref(h)))
        return DedispersionConfig(h)

    @staticmethod
    def from_dict(d):
        import yaml
        return DedispersionConfig.from_yaml_string(yaml.safe_dump(d, default_flow_style=None, width=1 << 30))

    def to_yaml_string(self):
        return _yaml_out(lib().pb2_config_to_yaml, self._h)

    def to_dict(self):
        return dict(self._d)

    def __getattr__(self, k):
        d = self.__dict__.get("_d")
        if d is not None and k in d:
            return d[k]
        raise AttributeError(k)

    def get_total_nfreq(self):
        return int(sum(self._d["zone_nfreq"]))

    def make_random_freq_variances(self, noisy=False, rng=None):
        """Per-channel input variances for tests (DedispersionConfig::make_random_freq_variances,
        src_lib/DedispersionConfig.cpp:253-272): one uniform random value in (0, 1) per zone,
        repeated over the zone's channels. rng: a numpy Generator (default: a fresh one)."""
        rng = np.random.default_rng() if rng is None else rng
        zone_var = [float(rng.uniform(1e-6, 1.0)) for _ in self._d["zone_nfreq"]]
        if noisy:
            print("make_random_freq_variances: per-zone variances = %s" % (tuple(zone_var),))
        return np.concatenate([np.full(int(n), v) for n, v in zip(self._d["zone_nfreq"], zone_var)])

    def make_channel_map(self):
        n = 2 ** int(self._d["toplevel_tree_rank"]) + 1
        out = np.zeros(n, dtype=np.float64)
        _check(lib().pb2_config_channel_map(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out

    def delay_to_frequency(self, delay):
        x = ctypes.c_double()
        _check(lib().pb2_config_delay_to_frequency(self._h, float(delay), ctypes.byref(x)))
        return x.value

    def frequency_to_delay(self, freq):
        x = ctypes.c_double()
        _check(lib().pb2_config_frequency_to_delay(self._h, float(freq), ctypes.byref(x)))
        return x.value

    def dm_per_unit_delay(self):
        x = ctypes.c_double()
        _check(lib().pb2_config_dm_per_unit_delay(self._h, ctypes.byref(x)))
        return x.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pb2_config_destroy(self._h)
            self._h = None


class DedispersionTree:
    """Per-output-tree shapes (include/pirate/DedispersionTree.hpp:19-59)."""

    def __init__(self, info):
        for k, _ in _TreeInfo._fields_:
            setattr(self, k, getattr(info, k))

    def total_rank(self):
        return self.amb_rank + self.dd_rank

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in _TreeInfo._fields_}


class DedispersionPlan:
    """pirate's DedispersionPlan (include/pirate/DedispersionPlan.hpp:33-225)."""

    def __init__(self, config):
        if isinstance(config, str):
            config = DedispersionConfig.from_yaml(config)
        self.config = config
        h = ctypes.c_void_p()
        _check(lib().pb2_plan_create(config._h, ctypes.byref(h)))
        self._h = h
        n = ctypes.c_long()
        _check(lib().pb2_plan_ntrees(h, ctypes.byref(n)))
        self.ntrees = n.value
        self.trees = []
        for i in range(self.ntrees):
            info = _TreeInfo()
            _check(lib().pb2_plan_tree_info(h, i, ctypes.byref(info)))
            tree = DedispersionTree(info)
            flo = (ctypes.c_long * info.nsubbands)()
            fhi = (ctypes.c_long * info.nsubbands)()
            _check(lib().pb2_plan_tree_subbands(h, i, flo, fhi, info.nsubbands))
            tree.n_to_flo, tree.n_to_fhi = list(flo), list(fhi)
            self.trees.append(tree)
        d = config.to_dict()
        self.dtype = d["dtype"]
        self.nfreq = config.get_total_nfreq()
        self.nt_in = int(d["time_samples_per_chunk"])
        self.num_primary_trees = len(d["primary_trees"])
        self.beams_per_gpu = int(d["beams_per_gpu"])
        self.beams_per_batch = int(d["beams_per_batch"])
        self.num_active_batches = int(d["num_active_batches"])
        npri = self.num_primary_trees
        dd = (ctypes.c_long * npri)()
        amb = (ctypes.c_long * npri)()
        _check(lib().pb2_plan_stage1_ranks(h, dd, amb, npri))
        self.stage1_dd_rank = list(dd)
        self.stage1_amb_rank = list(amb)

    def to_yaml_string(self):
        return _yaml_out(lib().pb2_plan_to_yaml, self._h)

    def decode_argmax(self, token, itree, idm, itime):
        """Returns (fmin, fmax, tlo, thi, p) (src_lib/DedispersionPlan.cpp:481)."""
        out = (ctypes.c_long * 5)()
        _check(lib().pb2_plan_decode_argmax(self._h, int(token), int(itree), int(idm), int(itime), out))
        return tuple(out)

    def decode_argmax2(self, itree, fmin, fmax, tlo, thi, p):
        """Returns (freq_lo_MHz, freq_hi_MHz, dm, timestamp_samp, width_samp) (src_lib/DedispersionPlan.cpp:544)."""
        inp = (ctypes.c_long * 5)(fmin, fmax, tlo, thi, p)
        out = (ctypes.c_double * 5)()
        _check(lib().pb2_plan_decode_argmax2(self._h, int(itree), inp, out))
        return tuple(out)

    def decode_argmax_batch(self, tokens, itrees, idms, itimes):
        """Vectorized decode_argmax over nonempty 1-d arrays (one event per element). Returns
        (fmins, fmaxs, tlos, this, ps), int64 arrays (src_pybind11/pirate_pybind11.cpp:396-401)."""
        tok = np.ascontiguousarray(tokens, dtype=np.uint32)
        its, ids, itm = (np.ascontiguousarray(a, dtype=np.int64) for a in (itrees, idms, itimes))
        n = tok.size
        if tok.ndim != 1 or any(a.shape != tok.shape for a in (its, ids, itm)):
            raise RuntimeError("decode_argmax_batch: tokens, itrees, idms and itimes must be 1-d of one length")
        outs = [np.zeros(n, dtype=np.int64) for _ in range(5)]
        _check(lib().pb2_plan_decode_argmax_batch(self._h, n, tok.ctypes.data, its.ctypes.data, ids.ctypes.data,
                                                  itm.ctypes.data, *[o.ctypes.data for o in outs]))
        return tuple(outs)

    def decode_argmax2_batch(self, itrees, fmins, fmaxs, tlos, this, ps):
        """Vectorized decode_argmax2: (freqs_lo_MHz, freqs_hi_MHz, dms, timestamps_samp, widths_samp),
        float64 arrays; timestamps are chunk-relative toplevel samples
        (src_pybind11/pirate_pybind11.cpp:402-409)."""
        ins = [np.ascontiguousarray(a, dtype=np.int64) for a in (itrees, fmins, fmaxs, tlos, this, ps)]
        n = ins[0].size
        if ins[0].ndim != 1 or any(a.shape != ins[0].shape for a in ins):
            raise RuntimeError("decode_argmax2_batch: the arrays must be 1-d of one length")
        outs = [np.zeros(n, dtype=np.float64) for _ in range(5)]
        _check(lib().pb2_plan_decode_argmax2_batch(self._h, n, *[a.ctypes.data for a in ins],
                                                   *[o.ctypes.data for o in outs]))
        return tuple(outs)

    def compute_steady_state_it0(self, itree):
        n = self.trees[itree].ndm_out
        out = np.zeros(n, dtype=np.int64)
        _check(lib().pb2_plan_steady_state_it0(self._h, int(itree), out.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), n))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pb2_plan_destroy(self._h)
            self._h = None


class PfAvarApproximation:
    """pirate's PfAvarApproximation (include/pirate/PfVariance.hpp:86-120): analytic variances of the
    peak finder's trials under unit weights, for white-noise input with per-channel variances
    freq_variances (length nfreq, all > 0). tree_variance[itree] has shape (N, ndm_wt, nprofiles)."""

    def __init__(self, plan, freq_variances):
        fv = np.ascontiguousarray(freq_variances, dtype=np.float64)
        if fv.ndim != 1:
            raise RuntimeError("PfAvarApproximation: freq_variances must be one-dimensional")
        self.nfreq = plan.nfreq
        self.ntrees = plan.ntrees
        self.tree_variance = [np.zeros((t.nsubbands, t.ndm_wt, t.nprofiles), dtype=np.float64) for t in plan.trees]
        ptrs = (ctypes.POINTER(ctypes.c_double) * self.ntrees)(
            *[a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in self.tree_variance])
        lens = (ctypes.c_long * self.ntrees)(*[a.size for a in self.tree_variance])
        _check(lib().pb2_plan_pf_variances(plan._h, fv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), fv.size,
                                           ptrs, lens, self.ntrees))


_TORCH_DTYPES = {0: "float32", 1: "float16", 2: "bfloat16"}


def _device_tensor(ptr, shape, dtype, device):
    """Wraps device memory owned by the dedisperser as a torch tensor (no copy)."""
    import torch
    tdt = getattr(torch, dtype)
    n = int(np.prod(shape))
    esize = torch.tensor([], dtype=tdt).element_size()
    if n == 0:
        return torch.empty(shape, dtype=tdt, device=device)
    # Build a byte view via the CUDA array interface, then reinterpret.
    holder = type("_Holder", (), {})()
    holder.__cuda_array_interface__ = {"shape": (n * esize,), "typestr": "|u1", "data": (int(ptr), False), "version": 3}
    t = torch.as_tensor(holder, device=device)
    return t.view(tdt).view(*shape)


class Outputs:
    """GpuDedisperser::Outputs (include/pirate/Dedisperser.hpp:98-125); arrays are torch views."""

    def __init__(self, o, device):
        self._raw = o
        self.dtype = _TORCH_DTYPES[o.dtype]
        self.nbeams = o.nbeams
        self.ichunk_zero_based = o.ichunk_zero_based
        self.ichunk_fpga_based = o.ichunk_fpga_based
        self.ibeam = o.ibeam
        self.ndm_out = [o.ndm_out[i] for i in range(o.ntrees)]
        self.nt_out = [o.nt_out[i] for i in range(o.ntrees)]
        self.out_max = [_device_tensor(o.out_max[i], (o.nbeams, o.ndm_out[i], o.nt_out[i]), self.dtype, device)
                        for i in range(o.ntrees)]
        # uint32 tokens, exposed as int32 views (same bits).
        self.out_argmax = [_device_tensor(o.out_argmax[i], (o.nbeams, o.ndm_out[i], o.nt_out[i]), "int32", device)
                           for i in range(o.ntrees)]
        # Candidate stage (GpuDedisperser.enable_sifter), else None: per-beam device tensors.
        self.candidates = None
        if o.cand_peak:
            B = o.nbeams
            self.candidates = dict(
                peak=_device_tensor(o.cand_peak, (B,), "float32", device),
                tree=_device_tensor(o.cand_tree, (B,), "int32", device),
                idm=_device_tensor(o.cand_idm, (B,), "int32", device),
                itime=_device_tensor(o.cand_itime, (B,), "int32", device),
                token=_device_tensor(o.cand_token, (B,), "int32", device),
                valid=_device_tensor(o.cand_valid, (B,), "int32", device),
                patches=_device_tensor(o.patches, (B, 9, 32, 6), "float16", device),
                scores=_device_tensor(o.scores, (B,), "float32", device))


class GpuDedisperser:
    """pirate's GpuDedisperser (include/pirate/Dedisperser.hpp:45-254; python wrapper
    pirate_frb/GpuDedisperser.py:123-197)."""

    def __init__(self, plan, cuda_device_id=0, num_consumers=1, nbatches_out=0, nbatches_wt=0,
                 initial_chunk=0, synchronous=True, release_timeout_ms=0):
        self.plan = plan
        self.cuda_device_id = int(cuda_device_id)
        self.device = "cuda:%d" % self.cuda_device_id
        p = _DdParams(self.cuda_device_id, int(nbatches_out), int(nbatches_wt), int(num_consumers),
                      1 if synchronous else 0, int(initial_chunk), int(release_timeout_ms))
        h = ctypes.c_void_p()
        _check(lib().pb2_dd_create(plan._h, ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.num_consumers = int(num_consumers)
        self.nbatches = plan.beams_per_gpu // plan.beams_per_batch
        self.nbatches_out = int(nbatches_out) or plan.num_active_batches
        self.nbatches_wt = int(nbatches_wt) or self.nbatches_out
        # batch seq_id runs on compute stream seq_id % num_compute_streams (pirate: one stream per active batch)
        self.num_compute_streams = plan.num_active_batches
        self.dtype = plan.dtype
        self._next_in = 0
        self._next_out = [0] * self.num_consumers

    def allocate(self):
        _check(lib().pb2_dd_allocate(self._h))

    def device_bytes(self):
        n = ctypes.c_long()
        _check(lib().pb2_dd_device_bytes(self._h, ctypes.byref(n)))
        return n.value

    def host_bytes(self):
        """Pinned host bytes of the delay lines spilled beyond the config's max_gpu_clag."""
        n = ctypes.c_long()
        _check(lib().pb2_dd_host_bytes(self._h, ctypes.byref(n)))
        return n.value

    def kernels_per_batch(self):
        n = ctypes.c_long()
        _check(lib().pb2_dd_kernels_per_batch(self._h, ctypes.byref(n)))
        return n.value

    def algorithmic_bytes(self):
        """HBM bytes per (chunk, batch) for [grid_lds, sifter (0), stage1, stage2, pf]."""
        out = (ctypes.c_double * 5)()
        _check(lib().pb2_dd_algorithmic_bytes(self._h, out))
        return list(out)

    KERNEL_CLASSES = ("grid_lds", "sifter", "stage1", "stage2", "pf")

    def enable_timing(self, on=True):
        _check(lib().pb2_dd_enable_timing(self._h, 1 if on else 0))

    def kernel_times(self):
        """{class: (milliseconds, launches)} accumulated since enable_timing()."""
        ms = (ctypes.c_double * 5)()
        n = (ctypes.c_long * 5)()
        _check(lib().pb2_dd_kernel_times(self._h, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    def acquire_input(self, seq_id, stream=None):
        ptr = ctypes.c_void_p()
        shape = (ctypes.c_long * 3)()
        _check(lib().pb2_dd_acquire_input(self._h, int(seq_id), _stream_ptr(stream), ctypes.byref(ptr), shape))
        return _device_tensor(ptr.value, tuple(shape), {"float32": "float32", "float16": "float16",
                                                        "bfloat16": "bfloat16"}[self.dtype], self.device)

    def acquire_input_int4(self, seq_id, stream=None):
        """The next input slot in pirate's raw format: returns (data, scales_offsets), device tensors of
        shapes (B, nfreq, nt_in // 2) uint8 (two int4 samples per byte, low nibble first) and
        (B, nfreq, nt_in // 256, 2) float16 (scale, offset). Same seq_id cursor as acquire_input; the
        kernels dequantize while gridding (GpuDedisperser::time's input, src_lib/GpuDedisperser.cpp:1617-1660)."""
        data = ctypes.c_void_p()
        so = ctypes.c_void_p()
        shape = (ctypes.c_long * 3)()
        _check(lib().pb2_dd_acquire_input_int4(self._h, int(seq_id), _stream_ptr(stream), ctypes.byref(data),
                                               ctypes.byref(so), shape))
        B, F, T = tuple(shape)
        return (_device_tensor(data.value, (B, F, T // 2), "uint8", self.device),
                _device_tensor(so.value, (B, F, T // 256, 2), "float16", self.device))

    def release_input_and_launch_dd_kernels(self, seq_id, stream=None):
        _check(lib().pb2_dd_release_input(self._h, int(seq_id), _stream_ptr(stream)))

    def acquire_output(self, consumer_id, seq_id, stream=None, sync=False):
        o = _Outputs()
        _check(lib().pb2_dd_acquire_output(self._h, int(consumer_id), int(seq_id), _stream_ptr(stream),
                                           1 if sync else 0, ctypes.byref(o)))
        return Outputs(o, self.device)

    def release_output(self, consumer_id, seq_id, stream=None):
        _check(lib().pb2_dd_release_output(self._h, int(consumer_id), int(seq_id), _stream_ptr(stream)))

    def fill_all_weights(self, itree, pf_weights):
        """pf_weights: (nbatches_wt, beams_per_batch, ndm_wt, nt_wt, nprofiles, N) float32."""
        w = np.ascontiguousarray(pf_weights, dtype=np.float32)
        _check(lib().pb2_dd_fill_weights(self._h, int(itree), w.ctypes.data, w.size))

    def fill_analytic_weights(self, freq_variances):
        """Every weight slot and beam gets the analytic SNR weights 1/sqrt(variance) of
        PfAvarApproximation(plan, freq_variances) (src_lib/GpuDedisperser.cpp:1162-1238). Blocks until
        the weights are on the GPU."""
        fv = np.ascontiguousarray(freq_variances, dtype=np.float64)
        if fv.ndim != 1:
            raise RuntimeError("fill_analytic_weights: freq_variances must be one-dimensional")
        _check(lib().pb2_dd_fill_analytic_weights(self._h, fv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), fv.size))

    def stop(self):
        _check(lib().pb2_dd_stop(self._h))

    def time(self, niterations):
        """pirate's GpuDedisperser.time (src_lib/GpuDedisperser.cpp:1573-1665): int4 batches copied from
        pinned host memory, dedispersed and consumed in a loop; returns the real-time beams of every
        iteration (numpy array; element 0 is 0, the first 2 * num_active_batches are warm-up)."""
        out = np.zeros(int(niterations), np.float64)
        _check(lib().pb2_dd_time(self._h, int(niterations), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        self._next_in += int(niterations)
        self._next_out = [n + int(niterations) for n in self._next_out]
        return out

    def zero_state(self, stream=None):
        """Clears every delay line and tree state (later chunks see zeros as history); the seq_id
        cursors are unchanged."""
        _check(lib().pb2_dd_zero_state(self._h, _stream_ptr(stream)))

    def enable_sifter(self, threshold=6.0, sifter=None):
        """Adds the candidate stage to every later batch: each beam's strongest output over the trees,
        the fp16 patch (9 DM x 32 time x 6 width) of peaks >= threshold, and its score by 'sifter'
        (pirate_b200.sifter.Sifter, or None: the score is then the peak). Results appear in
        Outputs.candidates. The sifter must not be trained while attached."""
        self._sifter = sifter
        _check(lib().pb2_dd_enable_sifter(self._h, float(threshold), sifter._h if sifter is not None else None))

    @contextlib.contextmanager
    def get_input(self, stream=None):
        """Context manager: yields the next input buffer, then launches the kernels on exit
        (pirate_frb/GpuDedisperser.py:123-160)."""
        seq = self._next_in
        arr = self.acquire_input(seq, stream)
        yield arr
        self.release_input_and_launch_dd_kernels(seq, stream)
        self._next_in += 1

    @contextlib.contextmanager
    def get_input_int4(self, stream=None):
        """Context manager: yields (data, scales_offsets) of the next input slot in int4 form, then
        launches the kernels on exit."""
        seq = self._next_in
        arrs = self.acquire_input_int4(seq, stream)
        yield arrs
        self.release_input_and_launch_dd_kernels(seq, stream)
        self._next_in += 1

    @contextlib.contextmanager
    def get_output(self, consumer_id=0, stream=None, sync=False):
        """Context manager: yields the next Outputs for 'consumer_id', released on exit."""
        seq = self._next_out[consumer_id]
        out = self.acquire_output(consumer_id, seq, stream, sync)
        yield out
        self.release_output(consumer_id, seq, stream)
        self._next_out[consumer_id] += 1

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pb2_dd_destroy(self._h)
            self._h = None


class BatchedDedisperser:
    """Many beams with uneven plans (tree rank, primary trees), one group per plan, each group's beams
    one batch; step() runs one chunk of every group as one replayed CUDA graph (include/pirate_b200.h,
    pb2_batched_*). pirate's counterpart is one GpuDedisperser per plan on a pool of compute streams
    (src_lib/GpuDedisperser.cpp:990-1000)."""

    def __init__(self, plans, cuda_device_id=0):
        self.plans = list(plans)
        self.device = "cuda:%d" % int(cuda_device_id)
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h.value if hasattr(p._h, "value") else p._h for p in self.plans])
        h = ctypes.c_void_p()
        _check(lib().pb2_batched_create(arr, len(self.plans), int(cuda_device_id), ctypes.byref(h)))
        self._h = h

    def allocate(self):
        _check(lib().pb2_batched_allocate(self._h))

    @property
    def ngroups(self):
        return len(self.plans)

    def device_bytes(self):
        n = ctypes.c_long()
        _check(lib().pb2_batched_device_bytes(self._h, ctypes.byref(n)))
        return n.value

    def fill_all_weights(self, group, itree, pf_weights):
        """pf_weights: (1, beams, ndm_wt, nt_wt, nprofiles, N) float32 (one weight slot)."""
        w = np.ascontiguousarray(pf_weights, dtype=np.float32)
        _check(lib().pb2_batched_fill_weights(self._h, int(group), int(itree), w.ctypes.data, w.size))

    def fill_analytic_weights(self, group, freq_variances):
        fv = np.ascontiguousarray(freq_variances, dtype=np.float64)
        _check(lib().pb2_batched_fill_analytic_weights(self._h, int(group), fv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), fv.size))

    def input(self, group):
        """The group's input slot, a (beams, nfreq, nt_in) CUDA tensor view in the plan's dtype."""
        ptr = ctypes.c_void_p()
        shape = (ctypes.c_long * 3)()
        _check(lib().pb2_batched_input(self._h, int(group), ctypes.byref(ptr), shape))
        return _device_tensor(ptr.value, tuple(shape), self.plans[group].dtype, self.device)

    def outputs(self, group):
        o = _Outputs()
        _check(lib().pb2_batched_outputs(self._h, int(group), ctypes.byref(o)))
        return Outputs(o, self.device)

    def step(self, stream=None):
        _check(lib().pb2_batched_step(self._h, _stream_ptr(stream)))

    def reset(self, stream=None):
        _check(lib().pb2_batched_reset(self._h, _stream_ptr(stream)))

    def set_schedule(self, merge_stage2, pf_general, grid_block, concurrent=True):
        n = self.ngroups
        m = (ctypes.c_int * n)(*[int(bool(x)) for x in merge_stage2])
        p = (ctypes.c_int * n)(*[int(bool(x)) for x in pf_general])
        g = (ctypes.c_int * n)(*[int(x) for x in grid_block])
        _check(lib().pb2_batched_set_schedule(self._h, m, p, g, int(bool(concurrent))))

    def autotune(self, reps=5):
        """Times the schedule choices on the replayed graph, keeps the fastest, clears the state;
        returns the record of trials and the choice (dict)."""
        import json
        n = ctypes.c_long()
        buf = ctypes.create_string_buffer(1 << 16)
        _check(lib().pb2_batched_autotune(self._h, int(reps), buf, len(buf), ctypes.byref(n)))
        return json.loads(buf.value.decode())

    def time_steps(self, n, stream=None):
        ms = ctypes.c_double()
        _check(lib().pb2_batched_time_steps(self._h, int(n), _stream_ptr(stream), ctypes.byref(ms)))
        return ms.value

    def kernels_per_step(self):
        n = ctypes.c_long()
        _check(lib().pb2_batched_kernels_per_step(self._h, ctypes.byref(n)))
        return n.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pb2_batched_destroy(self._h)
            self._h = None


def beam_peaks(outputs, stream=None, out=None):
    """The toy grouper's per-chunk reduction of one batch of outputs (pirate_frb/run_toy_grouper.py:
    79-116), in one kernel: per beam, the largest out_max over all trees, dm and time, its tree, dm and
    time indices and the out_argmax token there (a tree whose maximum is NaN is passed over; ties go to
    the first tree, then the first (dm, time)). 'outputs' is an acquired Outputs, or a pair of lists
    (out_max, out_argmax) of device tensors shaped (nbeams, ndm_out, nt_out). 'out', if given, is
    (peak float32, tree int32, idm int32, itime int32, token int32 view of uint32), each of nbeams
    entries; otherwise new tensors are returned in that order."""
    import torch
    if isinstance(outputs, Outputs):
        raw = outputs._raw
        nbeams = outputs.nbeams
        device = outputs.out_max[0].device
    else:
        maxes, args = outputs
        codes = {torch.float32: 0, torch.float16: 1, torch.bfloat16: 2}
        if not maxes or len(maxes) != len(args) or len(maxes) > MAX_TREES:
            raise RuntimeError("beam_peaks: need 1..%d (out_max, out_argmax) pairs" % MAX_TREES)
        raw = _Outputs()
        raw.dtype = codes[maxes[0].dtype]
        raw.nbeams = maxes[0].shape[0]
        raw.ntrees = len(maxes)
        for i, (m, a) in enumerate(zip(maxes, args)):
            if m.dtype != maxes[0].dtype or not m.is_contiguous() or not a.is_contiguous() or m.dim() != 3 \
                    or tuple(a.shape) != tuple(m.shape) or a.element_size() != 4 or m.shape[0] != raw.nbeams:
                raise RuntimeError("beam_peaks: arrays must be contiguous (nbeams, ndm_out, nt_out), one dtype")
            raw.ndm_out[i], raw.nt_out[i] = m.shape[1], m.shape[2]
            raw.out_max[i], raw.out_argmax[i] = m.data_ptr(), a.data_ptr()
        nbeams = raw.nbeams
        device = maxes[0].device
    if out is None:
        out = (torch.empty(nbeams, dtype=torch.float32, device=device),
               *[torch.empty(nbeams, dtype=torch.int32, device=device) for _ in range(4)])
    for t, dt in zip(out, (torch.float32, torch.int32, torch.int32, torch.int32, torch.int32)):
        if t.dtype != dt or t.numel() != nbeams or not t.is_contiguous():
            raise RuntimeError("beam_peaks: out must be (float32, int32 x 4) tensors of nbeams entries")
    _check(lib().pb2_beam_peaks(ctypes.byref(raw), *[t.data_ptr() for t in out], _stream_ptr(stream)))
    return out


def dequantize(out, scales_offsets, data, stream=None):
    """pirate's GpuDequantizationKernel::launch (include/pirate/GpuDequantizationKernel.hpp:53-70) on
    torch device tensors: out (nbeams, nfreq, ntime) float32/float16/bfloat16, scales_offsets
    (nbeams, nfreq, ntime // 256, 2) float16, data (nbeams, nfreq, ntime // 2) uint8. out = 0 where the
    int4 value is -8, else scale * value + offset in fp32, rounded once to out's dtype."""
    import torch
    codes = {torch.float32: 0, torch.float16: 1, torch.bfloat16: 2}
    if out.dtype not in codes:
        raise RuntimeError("dequantize: out must be float32, float16 or bfloat16")
    nbeams, nfreq, ntime = out.shape
    if tuple(data.shape) != (nbeams, nfreq, ntime // 2) or data.dtype != torch.uint8:
        raise RuntimeError("dequantize: data must be uint8 of shape (nbeams, nfreq, ntime // 2)")
    if tuple(scales_offsets.shape) != (nbeams, nfreq, ntime // 256, 2) or scales_offsets.dtype != torch.float16:
        raise RuntimeError("dequantize: scales_offsets must be float16 of shape (nbeams, nfreq, ntime // 256, 2)")
    for t in (out, scales_offsets, data):
        if not (t.is_cuda and t.is_contiguous()):
            raise RuntimeError("dequantize: arrays must be contiguous CUDA tensors")
    _check(lib().pb2_dequantize(out.data_ptr(), codes[out.dtype], scales_offsets.data_ptr(), data.data_ptr(),
                                nbeams, nfreq, ntime, _stream_ptr(stream)))
