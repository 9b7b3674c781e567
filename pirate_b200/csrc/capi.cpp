// capi.cpp -- extern "C" boundary (include/pirate_b200.h) over the C++ plan and GpuDedisperser.

#include "../../include/pirate_b200.h"
#include "dedisperser.hpp"
#include "plan.hpp"
#include "avar.hpp"
#include "kernels.cuh"
#include "simpulse.hpp"
#include "sifter.hpp"
#include "batched.hpp"

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <memory>
#include <string>

using namespace pb2;

struct pb2_config { DedispersionConfig c; };
struct pb2_plan { std::shared_ptr<DedispersionPlan> p; };
struct pb2_dedisperser { std::unique_ptr<GpuDedisperser> d; };
struct pb2_sifter { std::unique_ptr<Sifter> s; };
struct pb2_batched { std::unique_ptr<BatchedDedisperser> b; };

static void fill_outputs(const GpuDedisperser::Outputs &o, pb2_outputs *out)
{
    memset(out, 0, sizeof(*out));
    out->dtype = int(o.dtype);
    out->nbeams = o.nbeams;
    out->ichunk_zero_based = o.ichunk_zero_based;
    out->ichunk_fpga_based = o.ichunk_fpga_based;
    out->ibeam = o.ibeam;
    out->ntrees = long(o.out_max.size());
    for (size_t i = 0; i < o.out_max.size(); i++) {
        out->ndm_out[i] = o.ndm_out[i];
        out->nt_out[i] = o.nt_out[i];
        out->out_max[i] = o.out_max[i];
        out->out_argmax[i] = o.out_argmax[i];
    }
    out->cand_peak = o.cand_peak;
    out->cand_tree = o.cand_tree;
    out->cand_idm = o.cand_idm;
    out->cand_itime = o.cand_itime;
    out->cand_valid = o.cand_valid;
    out->cand_token = o.cand_token;
    out->patches = o.patches;
    out->scores = o.scores;
}

#define CUDA_CHECK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) \
    throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(_e)); } while (0)

static thread_local std::string g_err;

template<typename F>
static int guard(F &&f)
{
    try {
        f();
        g_err.clear();
        return 0;
    } catch (std::exception &e) {
        g_err = e.what();
        return 1;
    } catch (...) {
        g_err = "unknown error";
        return 1;
    }
}

static void copy_out(const std::string &s, char *buf, long buflen, long *needed)
{
    if (needed) *needed = long(s.size()) + 1;
    if (buf && buflen > 0) {
        long n = std::min(long(s.size()), buflen - 1);
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
}

#define REQUIRE_PTR(p) do { if (!(p)) throw std::runtime_error(std::string(__func__) + ": null argument '" #p "'"); } while (0)

extern "C" {

const char *pb2_last_error(void) { return g_err.c_str(); }
const char *pb2_version(void) { return "pirate_b200 0.1 (sm_100a)"; }

int pb2_config_from_yaml(const char *path, pb2_config **out)
{
    return guard([&] { REQUIRE_PTR(path); REQUIRE_PTR(out); *out = new pb2_config{DedispersionConfig::from_yaml(path)}; });
}

int pb2_config_from_yaml_string(const char *text, pb2_config **out)
{
    return guard([&] { REQUIRE_PTR(text); REQUIRE_PTR(out); *out = new pb2_config{DedispersionConfig::from_yaml_string(text, "yaml")}; });
}

int pb2_config_to_yaml(const pb2_config *cfg, char *buf, long buflen, long *needed)
{
    return guard([&] { REQUIRE_PTR(cfg); copy_out(cfg->c.to_yaml_string(), buf, buflen, needed); });
}

int pb2_config_channel_map(const pb2_config *cfg, double *out, long n)
{
    return guard([&] {
        REQUIRE_PTR(cfg); REQUIRE_PTR(out);
        std::vector<double> cm = cfg->c.make_channel_map();
        if (n != (long) cm.size()) throw std::runtime_error("pb2_config_channel_map: expected n=" + std::to_string(cm.size()));
        memcpy(out, cm.data(), cm.size() * sizeof(double));
    });
}

int pb2_config_delay_to_frequency(const pb2_config *cfg, double delay, double *freq)
{
    return guard([&] { REQUIRE_PTR(cfg); REQUIRE_PTR(freq); *freq = cfg->c.delay_to_frequency(delay); });
}

int pb2_config_frequency_to_delay(const pb2_config *cfg, double freq, double *delay)
{
    return guard([&] { REQUIRE_PTR(cfg); REQUIRE_PTR(delay); *delay = cfg->c.frequency_to_delay(freq); });
}

int pb2_config_dm_per_unit_delay(const pb2_config *cfg, double *dm)
{
    return guard([&] { REQUIRE_PTR(cfg); REQUIRE_PTR(dm); *dm = cfg->c.dm_per_unit_delay(); });
}

void pb2_config_destroy(pb2_config *cfg) { delete cfg; }

int pb2_plan_create(const pb2_config *cfg, pb2_plan **out)
{
    return guard([&] { REQUIRE_PTR(cfg); REQUIRE_PTR(out); *out = new pb2_plan{std::make_shared<DedispersionPlan>(cfg->c)}; });
}

void pb2_plan_destroy(pb2_plan *plan) { delete plan; }

int pb2_plan_to_yaml(const pb2_plan *plan, char *buf, long buflen, long *needed)
{
    return guard([&] { REQUIRE_PTR(plan); copy_out(plan->p->to_yaml_string(), buf, buflen, needed); });
}

int pb2_plan_ntrees(const pb2_plan *plan, long *ntrees)
{
    return guard([&] { REQUIRE_PTR(plan); REQUIRE_PTR(ntrees); *ntrees = plan->p->ntrees; });
}

int pb2_plan_tree_subbands(const pb2_plan *plan, long itree, long *n_to_flo, long *n_to_fhi, long n)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(n_to_flo); REQUIRE_PTR(n_to_fhi);
        if (itree < 0 || itree >= plan->p->ntrees) throw std::runtime_error("pb2_plan_tree_subbands: itree out of range");
        const FrequencySubbands &fs = plan->p->trees[itree].frequency_subbands;
        if (n != fs.N) throw std::runtime_error("pb2_plan_tree_subbands: n must equal the tree's number of subbands N");
        for (long i = 0; i < n; i++) {
            n_to_flo[i] = fs.n_to_flo[i];
            n_to_fhi[i] = fs.n_to_fhi[i];
        }
    });
}

int pb2_plan_pf_variances(const pb2_plan *plan, const double *freq_variances, long nfreq, double *const *out,
                          const long *out_len, long ntrees)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(freq_variances); REQUIRE_PTR(out); REQUIRE_PTR(out_len);
        const DedispersionPlan &p = *plan->p;
        if (ntrees != p.ntrees) throw std::runtime_error("pb2_plan_pf_variances: ntrees must equal the plan's number of trees");
        for (long t = 0; t < ntrees; t++) {
            const DedispersionTree &tr = p.trees[t];
            const long want = tr.frequency_subbands.N * tr.ndm_wt * tr.nprofiles;
            if (!out[t] || out_len[t] != want)
                throw std::runtime_error("pb2_plan_pf_variances: out[" + std::to_string(t) + "] must hold N * ndm_wt * nprofiles = "
                                         + std::to_string(want) + " doubles");
        }
        std::vector<std::vector<double>> v = pf_analytic_variances(p, freq_variances, nfreq);
        for (long t = 0; t < ntrees; t++)
            std::copy(v[t].begin(), v[t].end(), out[t]);
    });
}

int pb2_plan_tree_info(const pb2_plan *plan, long itree, pb2_tree_info *o)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(o);
        if (itree < 0 || itree >= plan->p->ntrees) throw std::runtime_error("pb2_plan_tree_info: itree out of range");
        const DedispersionTree &t = plan->p->trees[itree];
        o->primary_tree_index = t.primary_tree_index;
        o->early_trigger_level = t.early_trigger_level;
        o->amb_rank = t.amb_rank;
        o->dd_rank = t.dd_rank;
        o->nt_ds = t.nt_ds;
        o->ndm_out = t.ndm_out;
        o->nt_out = t.nt_out;
        o->ndm_wt = t.ndm_wt;
        o->nt_wt = t.nt_wt;
        o->nprofiles = t.nprofiles;
        o->Dcore = t.Dcore;
        o->max_width = t.pf.max_width;
        o->dm_downsampling = t.pf.dm_downsampling;
        o->time_downsampling = t.pf.time_downsampling;
        o->wt_dm_downsampling = t.pf.wt_dm_downsampling;
        o->wt_time_downsampling = t.pf.wt_time_downsampling;
        o->nsubbands = t.frequency_subbands.N;
        o->nmultiplets = t.frequency_subbands.M;
        o->pf_rank = t.frequency_subbands.pf_rank;
        o->dm_min = t.dm_min;
        o->dm_max = t.dm_max;
        o->trigger_frequency = t.trigger_frequency;
    });
}

int pb2_plan_stage1_ranks(const pb2_plan *plan, long *dd_rank, long *amb_rank, long n)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(dd_rank); REQUIRE_PTR(amb_rank);
        if (n != plan->p->num_primary_trees) throw std::runtime_error("pb2_plan_stage1_ranks: n must equal num_primary_trees");
        for (long i = 0; i < n; i++) { dd_rank[i] = plan->p->stage1_dd_rank[i]; amb_rank[i] = plan->p->stage1_amb_rank[i]; }
    });
}

int pb2_plan_decode_argmax(const pb2_plan *plan, uint32_t token, long itree, long idm, long itime, long *o)
{
    return guard([&] { REQUIRE_PTR(plan); REQUIRE_PTR(o); plan->p->decode_argmax(token, itree, idm, itime, o[0], o[1], o[2], o[3], o[4]); });
}

int pb2_plan_decode_argmax2(const pb2_plan *plan, long itree, const long *in5, double *o)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(in5); REQUIRE_PTR(o);
        plan->p->decode_argmax2(itree, in5[0], in5[1], in5[2], in5[3], in5[4], o[0], o[1], o[2], o[3], o[4]);
    });
}

int pb2_plan_decode_argmax_batch(const pb2_plan *plan, long n, const uint32_t *tokens, const long *itrees,
                                 const long *idms, const long *itimes, long *fmins, long *fmaxs, long *tlos,
                                 long *this_, long *ps)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(tokens); REQUIRE_PTR(itrees); REQUIRE_PTR(idms); REQUIRE_PTR(itimes);
        REQUIRE_PTR(fmins); REQUIRE_PTR(fmaxs); REQUIRE_PTR(tlos); REQUIRE_PTR(this_); REQUIRE_PTR(ps);
        if (n <= 0) throw std::runtime_error("decode_argmax_batch: the arrays must be nonempty");
        for (long i = 0; i < n; i++)
            plan->p->decode_argmax(tokens[i], itrees[i], idms[i], itimes[i], fmins[i], fmaxs[i], tlos[i], this_[i], ps[i]);
    });
}

int pb2_plan_decode_argmax2_batch(const pb2_plan *plan, long n, const long *itrees, const long *fmins,
                                  const long *fmaxs, const long *tlos, const long *this_, const long *ps,
                                  double *freqs_lo, double *freqs_hi, double *dms, double *times, double *widths)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(itrees); REQUIRE_PTR(fmins); REQUIRE_PTR(fmaxs); REQUIRE_PTR(tlos);
        REQUIRE_PTR(this_); REQUIRE_PTR(ps); REQUIRE_PTR(freqs_lo); REQUIRE_PTR(freqs_hi); REQUIRE_PTR(dms);
        REQUIRE_PTR(times); REQUIRE_PTR(widths);
        if (n <= 0) throw std::runtime_error("decode_argmax2_batch: the arrays must be nonempty");
        for (long i = 0; i < n; i++)
            plan->p->decode_argmax2(itrees[i], fmins[i], fmaxs[i], tlos[i], this_[i], ps[i], freqs_lo[i], freqs_hi[i],
                                    dms[i], times[i], widths[i]);
    });
}

struct pb2_pulse
{
    std::unique_ptr<pb2::SinglePulse> p;
    long *d_idx = nullptr;      // device copies for injection: it0, cnt, off (3 * nfreq)
    float *d_data = nullptr;
    int device = -1;
    ~pb2_pulse()
    {
        if (d_idx) cudaFree(d_idx);
        if (d_data) cudaFree(d_data);
    }
};

int pb2_dispersion_delay(double dm, double freq_mhz, double *out)
{
    return guard([&] { REQUIRE_PTR(out); *out = pb2::dispersion_delay(dm, freq_mhz); });
}

int pb2_scattering_time(double sm, double freq_mhz, double *out)
{
    return guard([&] { REQUIRE_PTR(out); *out = pb2::scattering_time(sm, freq_mhz); });
}

int pb2_pulse_create(const pb2_pulse_params *pp, const double *freq_edges_mhz, const double *freq_variances, long nfreq,
                     pb2_pulse **out)
{
    return guard([&] {
        REQUIRE_PTR(pp); REQUIRE_PTR(freq_edges_mhz); REQUIRE_PTR(freq_variances); REQUIRE_PTR(out);
        if (nfreq < 1) throw std::runtime_error("SinglePulse: nfreq must be >= 1");
        pb2::SinglePulseParams p;
        p.dm = pp->dm; p.sm = pp->sm; p.intrinsic_width = pp->intrinsic_width; p.spectral_index = pp->spectral_index;
        p.undispersed_arrival_time_sec = pp->undispersed_arrival_time_sec; p.time_sample_ms = pp->time_sample_ms;
        p.snr = pp->snr; p.subband_freq_lo_mhz = pp->subband_freq_lo_mhz; p.subband_freq_hi_mhz = pp->subband_freq_hi_mhz;
        p.internal_nt = pp->internal_nt;
        p.freq_edges_mhz.assign(freq_edges_mhz, freq_edges_mhz + nfreq + 1);
        p.freq_variances.assign(freq_variances, freq_variances + nfreq);
        std::unique_ptr<pb2_pulse> h(new pb2_pulse);
        h->p.reset(new pb2::SinglePulse(p));
        *out = h.release();
    });
}

void pb2_pulse_destroy(pb2_pulse *pulse) { delete pulse; }

int pb2_pulse_range(const pb2_pulse *pulse, long *it_start, long *it_end, long *nsamples)
{
    return guard([&] {
        REQUIRE_PTR(pulse); REQUIRE_PTR(it_start); REQUIRE_PTR(it_end); REQUIRE_PTR(nsamples);
        *it_start = pulse->p->it_start;
        *it_end = pulse->p->it_end;
        *nsamples = (long) pulse->p->sparse_data.size();
    });
}

int pb2_pulse_sparse(const pb2_pulse *pulse, long *freq_it0, long *freq_nt, long *freq_sd_off, float *sparse_data)
{
    return guard([&] {
        REQUIRE_PTR(pulse); REQUIRE_PTR(freq_it0); REQUIRE_PTR(freq_nt); REQUIRE_PTR(freq_sd_off); REQUIRE_PTR(sparse_data);
        const pb2::SinglePulse &sp = *pulse->p;
        std::copy(sp.freq_it0.begin(), sp.freq_it0.end(), freq_it0);
        std::copy(sp.freq_nt.begin(), sp.freq_nt.end(), freq_nt);
        std::copy(sp.freq_sd_off.begin(), sp.freq_sd_off.end(), freq_sd_off);
        std::copy(sp.sparse_data.begin(), sp.sparse_data.end(), sparse_data);
    });
}

int pb2_pulse_add_to_timestream(const pb2_pulse *pulse, float *out, long nfreq, long out_nt, long row_stride,
                                long out_it0, float weight)
{
    return guard([&] { REQUIRE_PTR(pulse); pulse->p->add_to_timestream(out, nfreq, out_nt, row_stride, out_it0, weight); });
}

int pb2_pulse_shift_samples(pb2_pulse *pulse, long delta_it)
{
    return guard([&] { REQUIRE_PTR(pulse); pulse->p->shift_samples(delta_it); });
}

int pb2_pulse_inject(pb2_pulse *pulse, void *chunk, int dtype, long nfreq, long nt, long row_stride, long chunk_it0,
                     float weight, void *stream)
{
    return guard([&] {
        REQUIRE_PTR(pulse); REQUIRE_PTR(chunk);
        const pb2::SinglePulse &sp = *pulse->p;
        if (nfreq != sp.nfreq) throw std::runtime_error("pb2_pulse_inject: the chunk must have one row per pulse channel");
        int dev = 0;
        CUDA_CHECK(cudaGetDevice(&dev));
        if (pulse->d_idx && pulse->device != dev) {
            cudaFree(pulse->d_idx); cudaFree(pulse->d_data);
            pulse->d_idx = nullptr; pulse->d_data = nullptr;
        }
        if (!pulse->d_idx) {
            std::vector<long> idx(3 * sp.nfreq);
            std::copy(sp.freq_it0.begin(), sp.freq_it0.end(), idx.begin());
            std::copy(sp.freq_nt.begin(), sp.freq_nt.end(), idx.begin() + sp.nfreq);
            std::copy(sp.freq_sd_off.begin(), sp.freq_sd_off.end(), idx.begin() + 2 * sp.nfreq);
            CUDA_CHECK(cudaMalloc((void **) &pulse->d_idx, idx.size() * sizeof(long)));
            CUDA_CHECK(cudaMalloc((void **) &pulse->d_data, sp.sparse_data.size() * sizeof(float)));
            pulse->device = dev;
            CUDA_CHECK(cudaMemcpy(pulse->d_idx, idx.data(), idx.size() * sizeof(long), cudaMemcpyHostToDevice));
            CUDA_CHECK(cudaMemcpy(pulse->d_data, sp.sparse_data.data(), sp.sparse_data.size() * sizeof(float), cudaMemcpyHostToDevice));
        }
        pb2::launch_pulse_inject(chunk, dtype, nfreq, nt, row_stride, chunk_it0, pulse->d_idx, pulse->d_idx + sp.nfreq,
                                 pulse->d_idx + 2 * sp.nfreq, pulse->d_data, weight, (cudaStream_t) stream);
    });
}

int pb2_beam_peaks(const pb2_outputs *outs, float *peak, int32_t *tree, int32_t *idm, int32_t *itime, uint32_t *token,
                   void *stream)
{
    return guard([&] {
        REQUIRE_PTR(outs); REQUIRE_PTR(peak); REQUIRE_PTR(tree); REQUIRE_PTR(idm); REQUIRE_PTR(itime); REQUIRE_PTR(token);
        if (outs->ntrees < 1 || outs->ntrees > PB2_MAX_TREES) throw std::runtime_error("pb2_beam_peaks: bad ntrees");
        pb2::BeamPeakArgs a;
        memset(&a, 0, sizeof(a));
        a.ntrees = int(outs->ntrees);
        for (long t = 0; t < outs->ntrees; t++) {
            a.ndm[t] = outs->ndm_out[t];
            a.nt[t] = outs->nt_out[t];
            a.out_max[t] = outs->out_max[t];
            a.out_argmax[t] = outs->out_argmax[t];
        }
        a.peak = peak; a.tree = tree; a.idm = idm; a.itime = itime; a.token = token;
        pb2::launch_beam_peaks(a, outs->dtype, outs->nbeams, (cudaStream_t) stream);
    });
}

int pb2_plan_steady_state_it0(const pb2_plan *plan, long itree, long *out, long n)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(out);
        std::vector<long> v = plan->p->compute_steady_state_it0(itree);
        if (n != (long) v.size()) throw std::runtime_error("pb2_plan_steady_state_it0: n must equal ndm_out");
        memcpy(out, v.data(), v.size() * sizeof(long));
    });
}

int pb2_dd_create(const pb2_plan *plan, const pb2_dd_params *p, pb2_dedisperser **out)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(p); REQUIRE_PTR(out);
        if (plan->p->ntrees > PB2_MAX_TREES) throw std::runtime_error("pb2_dd_create: too many trees");
        GpuDedisperser::Params gp;
        gp.cuda_device_id = p->cuda_device_id;
        gp.nbatches_out = p->nbatches_out;
        gp.nbatches_wt = p->nbatches_wt;
        gp.num_consumers = p->num_consumers;
        gp.synchronous = p->synchronous != 0;
        gp.initial_chunk = p->initial_chunk;
        gp.release_timeout_ms = p->release_timeout_ms;
        *out = new pb2_dedisperser{std::unique_ptr<GpuDedisperser>(new GpuDedisperser(*plan->p, gp))};
    });
}

int pb2_dd_allocate(pb2_dedisperser *dd)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->allocate(); });
}

int pb2_dd_device_bytes(const pb2_dedisperser *dd, long *nbytes)
{
    return guard([&] { REQUIRE_PTR(dd); REQUIRE_PTR(nbytes); *nbytes = long(dd->d->device_bytes()); });
}

int pb2_dd_host_bytes(const pb2_dedisperser *dd, long *nbytes)
{
    return guard([&] { REQUIRE_PTR(dd); REQUIRE_PTR(nbytes); *nbytes = long(dd->d->host_bytes()); });
}

int pb2_dd_acquire_input(pb2_dedisperser *dd, long seq_id, void *stream, void **ptr, long *shape3)
{
    return guard([&] {
        REQUIRE_PTR(dd); REQUIRE_PTR(ptr);
        *ptr = dd->d->acquire_input(seq_id, (cudaStream_t) stream);
        if (shape3) {
            shape3[0] = dd->d->plan.beams_per_batch;
            shape3[1] = dd->d->plan.nfreq;
            shape3[2] = dd->d->plan.nt_in;
        }
    });
}

int pb2_dd_acquire_input_int4(pb2_dedisperser *dd, long seq_id, void *stream, void **data, void **scales_offsets, long *shape3)
{
    return guard([&] {
        REQUIRE_PTR(dd); REQUIRE_PTR(data); REQUIRE_PTR(scales_offsets);
        *data = dd->d->acquire_input_int4(seq_id, (cudaStream_t) stream, scales_offsets);
        if (shape3) {
            shape3[0] = dd->d->plan.beams_per_batch;
            shape3[1] = dd->d->plan.nfreq;
            shape3[2] = dd->d->plan.nt_in;
        }
    });
}

int pb2_dequantize(void *out, int out_dtype, const void *scales_offsets, const void *data, long nbeams, long nfreq,
                   long ntime, void *stream)
{
    return guard([&] {
        REQUIRE_PTR(out); REQUIRE_PTR(scales_offsets); REQUIRE_PTR(data);
        if (out_dtype < 0 || out_dtype > 2) throw std::runtime_error("pb2_dequantize: out_dtype must be 0 (float32), 1 (float16) or 2 (bfloat16)");
        if (nbeams < 0 || nfreq < 0) throw std::runtime_error("pb2_dequantize: negative shape");
        pb2::launch_dequantize(out, out_dtype, data, scales_offsets, nbeams, nfreq, ntime, (cudaStream_t) stream);
    });
}

int pb2_dd_release_input(pb2_dedisperser *dd, long seq_id, void *stream)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->release_input_and_launch_dd_kernels(seq_id, (cudaStream_t) stream); });
}

int pb2_dd_acquire_output(pb2_dedisperser *dd, long consumer_id, long seq_id, void *stream, int sync, pb2_outputs *out)
{
    return guard([&] {
        REQUIRE_PTR(dd); REQUIRE_PTR(out);
        GpuDedisperser::Outputs o = dd->d->acquire_output(consumer_id, seq_id, (cudaStream_t) stream, sync != 0);
        memset(out, 0, sizeof(*out));
        out->dtype = int(o.dtype);
        out->nbeams = o.nbeams;
        out->ichunk_zero_based = o.ichunk_zero_based;
        out->ichunk_fpga_based = o.ichunk_fpga_based;
        out->ibeam = o.ibeam;
        out->ntrees = long(o.out_max.size());
        for (size_t i = 0; i < o.out_max.size(); i++) {
            out->ndm_out[i] = o.ndm_out[i];
            out->nt_out[i] = o.nt_out[i];
            out->out_max[i] = o.out_max[i];
            out->out_argmax[i] = o.out_argmax[i];
        }
        out->cand_peak = o.cand_peak;
        out->cand_tree = o.cand_tree;
        out->cand_idm = o.cand_idm;
        out->cand_itime = o.cand_itime;
        out->cand_valid = o.cand_valid;
        out->cand_token = o.cand_token;
        out->patches = o.patches;
        out->scores = o.scores;
    });
}

int pb2_dd_release_output(pb2_dedisperser *dd, long consumer_id, long seq_id, void *stream)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->release_output(consumer_id, seq_id, (cudaStream_t) stream); });
}

int pb2_dd_fill_weights(pb2_dedisperser *dd, long itree, const float *host, long nelts)
{
    return guard([&] { REQUIRE_PTR(dd); REQUIRE_PTR(host); dd->d->fill_all_weights(itree, host, nelts); });
}

int pb2_dd_fill_analytic_weights(pb2_dedisperser *dd, const double *freq_variances, long nfreq)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->fill_analytic_weights(freq_variances, nfreq); });
}

int pb2_dd_stop(pb2_dedisperser *dd)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->stop(); });
}

int pb2_dd_time(pb2_dedisperser *dd, long niterations, double *rtb)
{
    return guard([&] { REQUIRE_PTR(dd); REQUIRE_PTR(rtb); dd->d->time(niterations, rtb); });
}

int pb2_dd_zero_state(pb2_dedisperser *dd, void *stream)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->zero_state((cudaStream_t) stream); });
}

int pb2_dd_kernels_per_batch(const pb2_dedisperser *dd, long *n)
{
    return guard([&] { REQUIRE_PTR(dd); REQUIRE_PTR(n); *n = dd->d->kernels_per_batch(); });
}

int pb2_dd_algorithmic_bytes(const pb2_dedisperser *dd, double *out5)
{
    return guard([&] {
        REQUIRE_PTR(dd); REQUIRE_PTR(out5);
        std::vector<double> v = dd->d->algorithmic_bytes();
        for (int i = 0; i < 5; i++) out5[i] = v[i];
    });
}

int pb2_dd_enable_timing(pb2_dedisperser *dd, int on)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->enable_timing(on != 0); });
}

int pb2_dd_kernel_times(pb2_dedisperser *dd, double *ms5, long *counts5)
{
    return guard([&] { REQUIRE_PTR(dd); REQUIRE_PTR(ms5); REQUIRE_PTR(counts5); dd->d->kernel_times(ms5, counts5); });
}

void pb2_dd_destroy(pb2_dedisperser *dd) { delete dd; }

int pb2_sifter_create(int cuda_device_id, long max_batch, uint64_t seed, pb2_sifter **out)
{
    return guard([&] { REQUIRE_PTR(out); *out = new pb2_sifter{std::unique_ptr<Sifter>(new Sifter(cuda_device_id, max_batch, seed))}; });
}

void pb2_sifter_destroy(pb2_sifter *s) { delete s; }

int pb2_sifter_nparams(long *n)
{
    return guard([&] { REQUIRE_PTR(n); *n = Sifter::nparams(); });
}

int pb2_sifter_set_params(pb2_sifter *s, const float *host_params)
{
    return guard([&] { REQUIRE_PTR(s); REQUIRE_PTR(host_params); s->s->set_params(host_params); });
}

int pb2_sifter_get_params(const pb2_sifter *s, float *host_params)
{
    return guard([&] { REQUIRE_PTR(s); REQUIRE_PTR(host_params); s->s->get_params(host_params); });
}

int pb2_sifter_forward(pb2_sifter *s, const void *patches, long n, float *logits, void *stream)
{
    return guard([&] {
        REQUIRE_PTR(s); REQUIRE_PTR(patches); REQUIRE_PTR(logits);
        CUDA_CHECK(cudaSetDevice(s->s->device));
        s->s->forward((const uint16_t *) patches, n, logits, (cudaStream_t) stream);
    });
}

int pb2_sifter_gradients(pb2_sifter *s, const void *patches, const float *labels, long n, float *grad, double *loss,
                         void *stream)
{
    return guard([&] {
        REQUIRE_PTR(s); REQUIRE_PTR(patches); REQUIRE_PTR(labels); REQUIRE_PTR(grad); REQUIRE_PTR(loss);
        *loss = s->s->gradients((const uint16_t *) patches, labels, n, grad, (cudaStream_t) stream);
    });
}

int pb2_sifter_train_step(pb2_sifter *s, const void *patches, const float *labels, long n, float lr, double *loss,
                          void *stream)
{
    return guard([&] {
        REQUIRE_PTR(s); REQUIRE_PTR(patches); REQUIRE_PTR(labels); REQUIRE_PTR(loss);
        *loss = s->s->train_step((const uint16_t *) patches, labels, n, lr, (cudaStream_t) stream);
    });
}

int pb2_dd_enable_sifter(pb2_dedisperser *dd, float threshold, pb2_sifter *sifter)
{
    return guard([&] { REQUIRE_PTR(dd); dd->d->enable_sifter(threshold, sifter ? sifter->s.get() : nullptr); });
}

int pb2_batched_create(const pb2_plan *const *plans, long nplans, int cuda_device_id, pb2_batched **out)
{
    return guard([&] {
        REQUIRE_PTR(plans); REQUIRE_PTR(out);
        if (nplans < 1) throw std::runtime_error("pb2_batched_create: no plans");
        std::vector<DedispersionPlan> ps;
        for (long i = 0; i < nplans; i++) {
            REQUIRE_PTR(plans[i]);
            if (plans[i]->p->ntrees > PB2_MAX_TREES) throw std::runtime_error("pb2_batched_create: too many trees");
            ps.push_back(*plans[i]->p);
        }
        *out = new pb2_batched{std::unique_ptr<BatchedDedisperser>(new BatchedDedisperser(ps, cuda_device_id))};
    });
}

int pb2_batched_allocate(pb2_batched *b) { return guard([&] { REQUIRE_PTR(b); b->b->allocate(); }); }

int pb2_batched_ngroups(const pb2_batched *b, long *n)
{
    return guard([&] { REQUIRE_PTR(b); REQUIRE_PTR(n); *n = b->b->ngroups(); });
}

int pb2_batched_device_bytes(const pb2_batched *b, long *nbytes)
{
    return guard([&] {
        REQUIRE_PTR(b); REQUIRE_PTR(nbytes);
        long t = 0;
        for (long g = 0; g < b->b->ngroups(); g++) t += long(b->b->group(g).device_bytes());
        *nbytes = t;
    });
}

int pb2_batched_fill_weights(pb2_batched *b, long group, long itree, const float *host, long nelts)
{
    return guard([&] { REQUIRE_PTR(b); REQUIRE_PTR(host); b->b->group(group).fill_all_weights(itree, host, nelts); });
}

int pb2_batched_fill_analytic_weights(pb2_batched *b, long group, const double *freq_variances, long nfreq)
{
    return guard([&] { REQUIRE_PTR(b); REQUIRE_PTR(freq_variances); b->b->group(group).fill_analytic_weights(freq_variances, nfreq); });
}

int pb2_batched_input(pb2_batched *b, long group, void **ptr, long *shape3)
{
    return guard([&] {
        REQUIRE_PTR(b); REQUIRE_PTR(ptr); REQUIRE_PTR(shape3);
        GpuDedisperser &g = b->b->group(group);
        *ptr = g.input_ptr(0);
        shape3[0] = g.plan.beams_per_batch;
        shape3[1] = g.plan.nfreq;
        shape3[2] = g.plan.nt_in;
    });
}

int pb2_batched_outputs(pb2_batched *b, long group, pb2_outputs *out)
{
    return guard([&] {
        REQUIRE_PTR(b); REQUIRE_PTR(out);
        GpuDedisperser::Outputs o = b->b->group(group).outputs_ptr(0);
        o.ichunk_zero_based = b->b->chunks_done() - 1;
        o.ichunk_fpga_based = o.ichunk_zero_based;
        fill_outputs(o, out);
    });
}

int pb2_batched_step(pb2_batched *b, void *stream) { return guard([&] { REQUIRE_PTR(b); b->b->step((cudaStream_t) stream); }); }

int pb2_batched_reset(pb2_batched *b, void *stream) { return guard([&] { REQUIRE_PTR(b); b->b->reset((cudaStream_t) stream); }); }

int pb2_batched_set_schedule(pb2_batched *b, const int *merge_stage2, const int *pf_general, const int *grid_block,
                             int concurrent)
{
    return guard([&] {
        REQUIRE_PTR(b); REQUIRE_PTR(merge_stage2); REQUIRE_PTR(pf_general); REQUIRE_PTR(grid_block);
        std::vector<GroupTuning> t(b->b->ngroups());
        for (size_t g = 0; g < t.size(); g++) {
            t[g].merge_stage2 = merge_stage2[g] != 0;
            t[g].pf_general = pf_general[g] != 0;
            t[g].grid_block = grid_block[g];
        }
        b->b->set_schedule(t, concurrent != 0);
    });
}

int pb2_batched_autotune(pb2_batched *b, int reps, char *buf, long buflen, long *needed)
{
    return guard([&] { REQUIRE_PTR(b); copy_out(b->b->autotune(reps), buf, buflen, needed); });
}

int pb2_batched_time_steps(pb2_batched *b, int nsteps, void *stream, double *ms_per_step)
{
    return guard([&] { REQUIRE_PTR(b); REQUIRE_PTR(ms_per_step); *ms_per_step = b->b->time_steps(nsteps, (cudaStream_t) stream); });
}

int pb2_batched_kernels_per_step(const pb2_batched *b, long *n)
{
    return guard([&] { REQUIRE_PTR(b); REQUIRE_PTR(n); *n = b->b->kernels_per_step(); });
}

void pb2_batched_destroy(pb2_batched *b) { delete b; }

int pb2_dedisperse_chunk_noalloc(const pb2_plan *plan, const void *in, const float *const *weights,
                                 void *const *out_max, uint32_t *const *out_argmax, void *stream)
{
    return guard([&] {
        REQUIRE_PTR(plan); REQUIRE_PTR(in); REQUIRE_PTR(weights); REQUIRE_PTR(out_max); REQUIRE_PTR(out_argmax);
        for (long i = 0; i < plan->p->ntrees; i++) {
            REQUIRE_PTR(weights[i]); REQUIRE_PTR(out_max[i]); REQUIRE_PTR(out_argmax[i]);
        }
        pb2::dedisperse_chunk_noalloc(*plan->p, in, weights, out_max, out_argmax, (cudaStream_t) stream);
    });
}

}  // extern "C"
