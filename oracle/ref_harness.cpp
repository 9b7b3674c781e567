// Test infrastructure: a C entry layer over pirate's OWN reference CPU implementation
// (ReferenceDedisperser, ReferenceTree, ReferenceLagbuf, ReferencePeakFindingKernel and the plan
// code), compiled unmodified from pirate's source tree against the minimal ksgpu / yaml-cpp
// stand-ins in oracle/ksgpu_shim. Built by 'make -C oracle ref PIRATE_SRC=...' into oracle/_ref/.
// Only the fixture generator (tests/golden/make_ref_golden.py) and tests use it, as the checker that
// pins oracle/refdd.cpp (and through it the CUDA path) to pirate's own arithmetic.
//
// The API mirrors oracle/refdd.cpp's orc_* functions:
//   ref_create(...)        DedispersionConfig built in code (src_lib/DedispersionConfig.cpp:333),
//                          DedispersionPlan(config, gpu_runnable=false) (src_lib/DedispersionPlan.cpp:29),
//                          every tree's Dcore set to min(time_downsampling, dcore_max) (the plan's
//                          tree.Dcore and stage2_pf_params[i].Dcore, src_lib/DedispersionPlan.cpp:143,335),
//                          ReferenceDedisperserBase::make(sophistication) (src_lib/ReferenceDedisperser.cpp:649)
//   ref_dedisperse(...)    fills input_array and wt_arrays, calls dedisperse(ichunk, ibatch), copies
//                          out_max / out_argmax (include/pirate/Dedisperser.hpp:455-473)
//   ref_eval_tokens(...)   ReferencePeakFindingKernel::eval_tokens (src_lib/PeakFindingKernel.cu:460)
//   ref_self_tests(...)    ReferenceTree::test_basics/test_subbands, ReferenceLagbuf::test_random
//   ref_pulse_*(...)       SinglePulse (src_lib/simpulse.cpp), with MKL's c2r DFT supplied by
//                          oracle/ksgpu_shim/mkl_dfti.h

#include "pirate/DedispersionConfig.hpp"
#include "pirate/DedispersionPlan.hpp"
#include "pirate/Dedisperser.hpp"
#include "pirate/PeakFindingKernel.hpp"
#include "pirate/ReferenceLagbuf.hpp"
#include "pirate/ReferenceTree.hpp"
#include "pirate/simpulse.hpp"

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace pirate;
using pirate::simpulse::SinglePulse;

namespace {

std::string ref_err;

struct RefHandle
{
    std::shared_ptr<DedispersionPlan> plan;
    std::shared_ptr<ReferenceDedisperserBase> dd;
    int tree_domain = 0;
};

template<typename F>
int guard(F &&f)
{
    try { f(); return 0; }
    catch (std::exception &e) { ref_err = e.what(); return -1; }
}

// Copies a C-contiguous host buffer into a (possibly strided) reference array of the same shape.
void copy_in(const ksgpu::Array<float> &dst, const float *src)
{
    ksgpu::Array<float> tmp(dst.shape_vec(), ksgpu::af_uhost);
    memcpy(tmp.data, src, tmp.size * sizeof(float));
    dst.fill(tmp);
}

template<typename T>
void copy_out(T *dst, const ksgpu::Array<T> &src)
{
    ksgpu::Array<T> tmp(src.shape_vec(), ksgpu::af_uhost);
    tmp.fill(src);
    memcpy(dst, tmp.data, tmp.size * sizeof(T));
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char *ref_last_error() { return ref_err.c_str(); }

// Primary tree i: ptrees[6*i .. 6*i+5] = (num_early_triggers, max_width, dm_downsampling,
// time_downsampling, wt_dm_downsampling, wt_time_downsampling), as orc_create.
__attribute__((visibility("default")))
void *ref_create(int nzones, const long *zone_nfreq, const double *zone_freq_edges, double time_sample_ms,
                 long toplevel_tree_rank, long time_samples_per_chunk, long nbits,
                 int nsb, const long *subband_counts, int npri, const long *ptrees,
                 long beams_per_gpu, long beams_per_batch, long dcore_max, int sophistication, int tree_domain)
{
    RefHandle *h = nullptr;
    int rc = guard([&] {
        DedispersionConfig c;
        c.zone_nfreq.assign(zone_nfreq, zone_nfreq + nzones);
        c.zone_freq_edges.assign(zone_freq_edges, zone_freq_edges + nzones + 1);
        c.time_sample_ms = time_sample_ms;
        c.toplevel_tree_rank = toplevel_tree_rank;
        c.time_samples_per_chunk = time_samples_per_chunk;
        c.dtype = ksgpu::Dtype(ksgpu::df_float, int(nbits));
        c.frequency_subband_counts.assign(subband_counts, subband_counts + nsb);
        for (int i = 0; i < npri; i++) {
            const long *p = ptrees + 6 * i;
            DedispersionConfig::PrimaryTree t;
            t.num_early_triggers = p[0];
            t.max_width = p[1];
            t.dm_downsampling = p[2];
            t.time_downsampling = p[3];
            t.wt_dm_downsampling = p[4];
            t.wt_time_downsampling = p[5];
            c.primary_trees.push_back(t);
        }
        c.beams_per_gpu = beams_per_gpu;
        c.beams_per_batch = beams_per_batch;
        c.num_active_batches = 1;
        c.validate();

        DedispersionPlan::Params pp;
        pp.gpu_runnable = false;
        auto plan = std::make_shared<DedispersionPlan>(c, pp);
        for (size_t i = 0; i < plan->trees.size(); i++) {
            long D = std::min(plan->trees[i].pf.time_downsampling, dcore_max);
            plan->trees[i].Dcore = D;
            plan->stage2_pf_params.at(i).Dcore = D;
        }

        ReferenceDedisperserBase::Params rp;
        rp.plan = plan;
        rp.sophistication = sophistication;
        rp.tree_domain_input = (tree_domain != 0);
        h = new RefHandle;
        h->plan = plan;
        h->tree_domain = tree_domain;
        h->dd = ReferenceDedisperserBase::make(rp);
    });
    if (rc != 0) { delete h; return nullptr; }
    return h;
}

__attribute__((visibility("default"))) void ref_destroy(void *h) { delete (RefHandle *) h; }

__attribute__((visibility("default"))) long ref_ntrees(void *h) { return ((RefHandle *) h)->plan->ntrees; }

// info[16] = ipri, early_trigger_level, amb_rank, dd_rank, nt_ds, ndm_out, nt_out, ndm_wt, nt_wt,
//            nprofiles, N, M, Dcore, max_width, pf_rank, time_downsampling (orc_tree_info's order)
__attribute__((visibility("default")))
int ref_tree_info(void *hv, long itree, long *info)
{
    return guard([&] {
        RefHandle *h = (RefHandle *) hv;
        const DedispersionTree &t = h->plan->trees.at(itree);
        const FrequencySubbands &fs = t.frequency_subbands;
        long v[16] = { t.primary_tree_index, t.early_trigger_level, t.amb_rank, t.dd_rank, t.nt_ds, t.ndm_out, t.nt_out,
                       t.ndm_wt, t.nt_wt, t.nprofiles, fs.N, fs.M, t.Dcore, t.pf.max_width, fs.pf_rank,
                       t.pf.time_downsampling };
        memcpy(info, v, sizeof(v));
    });
}

// in: C-contiguous (B, nfreq, nt_in) float32 (or (B, 2^rank, nt_in) with tree-domain input);
// wts[i]: (B, ndm_wt, nt_wt, nprofiles, N); out_max[i], out_argmax[i]: (B, ndm_out, nt_out).
__attribute__((visibility("default")))
int ref_dedisperse(void *hv, long ichunk, long ibatch, const float *in, const float *const *wts,
                   float *const *out_max, uint32_t *const *out_argmax)
{
    return guard([&] {
        RefHandle *h = (RefHandle *) hv;
        ReferenceDedisperserBase &dd = *h->dd;
        copy_in(dd.input_array, in);
        for (long i = 0; i < dd.ntrees; i++)
            copy_in(dd.wt_arrays.at(i), wts[i]);
        dd.dedisperse(ichunk, ibatch);
        for (long i = 0; i < dd.ntrees; i++) {
            copy_out<float>(out_max[i], dd.out_max.at(i));
            copy_out<uint>(out_argmax[i], dd.out_argmax.at(i));
        }
    });
}

// ReferencePeakFindingKernel::eval_tokens on tree itree: the weighted trial value that each token names,
// evaluated on the subband input of the last dedisperse() call.
__attribute__((visibility("default")))
int ref_eval_tokens(void *hv, long itree, const uint32_t *tokens, const float *wt, float *out)
{
    return guard([&] {
        RefHandle *h = (RefHandle *) hv;
        ReferenceDedisperserBase &dd = *h->dd;
        ReferencePeakFindingKernel &pf = *dd.pf_kernels.at(itree);
        ksgpu::Array<uint> tok(dd.out_argmax.at(itree).shape_vec(), ksgpu::af_uhost);
        memcpy(tok.data, tokens, tok.size * sizeof(uint));
        ksgpu::Array<float> w(dd.wt_arrays.at(itree).shape_vec(), ksgpu::af_uhost);
        memcpy(w.data, wt, w.size * sizeof(float));
        ksgpu::Array<float> o(dd.out_max.at(itree).shape_vec(), ksgpu::af_uhost | ksgpu::af_zero);
        pf.eval_tokens(o, tok, w);
        memcpy(out, o.data, o.size * sizeof(float));
    });
}

// Runs pirate's own CPU self-tests of the reference building blocks ('niter' random instances each).
__attribute__((visibility("default")))
int ref_self_tests(long niter)
{
    return guard([&] {
        for (long i = 0; i < niter; i++) {
            ReferenceTree::test_basics();
            ReferenceTree::test_subbands();
            ReferenceLagbuf::test_random();
        }
    });
}

// SinglePulse (include/pirate/simpulse.hpp:40-119). p[9] = dm, sm, intrinsic_width, spectral_index,
// undispersed_arrival_time_sec, time_sample_ms, snr, subband_freq_lo_MHz, subband_freq_hi_MHz.
struct RefPulse
{
    ksgpu::Array<double> edges, var;
    std::unique_ptr<SinglePulse> sp;
};

__attribute__((visibility("default")))
void *ref_pulse_create(const double *p, long internal_nt, const double *freq_edges, const double *freq_variances, long nfreq)
{
    RefPulse *h = new RefPulse;
    int rc = guard([&] {
        h->edges = ksgpu::Array<double>({nfreq + 1}, ksgpu::af_uhost);
        h->var = ksgpu::Array<double>({nfreq}, ksgpu::af_uhost);
        memcpy(h->edges.data, freq_edges, (nfreq + 1) * sizeof(double));
        memcpy(h->var.data, freq_variances, nfreq * sizeof(double));
        SinglePulse::Params sp;
        sp.dm = p[0]; sp.sm = p[1]; sp.intrinsic_width = p[2]; sp.spectral_index = p[3];
        sp.undispersed_arrival_time_sec = p[4]; sp.time_sample_ms = p[5]; sp.snr = p[6];
        sp.subband_freq_lo_MHz = p[7]; sp.subband_freq_hi_MHz = p[8];
        sp.internal_nt = internal_nt;
        sp.freq_edges_MHz = h->edges;
        sp.freq_variances = h->var;
        h->sp.reset(new SinglePulse(sp));
    });
    if (rc != 0) { delete h; return nullptr; }
    return h;
}

__attribute__((visibility("default"))) void ref_pulse_destroy(void *h) { delete (RefPulse *) h; }

// out[3] = it_start, it_end, number of stored samples.
__attribute__((visibility("default")))
int ref_pulse_range(void *hv, long *out)
{
    return guard([&] {
        const SinglePulse &sp = *((RefPulse *) hv)->sp;
        out[0] = sp.it_start; out[1] = sp.it_end; out[2] = sp.sparse_data.size;
    });
}

__attribute__((visibility("default")))
int ref_pulse_sparse(void *hv, long *freq_it0, long *freq_nt, long *freq_sd_off, float *sparse_data)
{
    return guard([&] {
        const SinglePulse &sp = *((RefPulse *) hv)->sp;
        long nfreq = sp.freq_it0.size;
        memcpy(freq_it0, sp.freq_it0.data, nfreq * sizeof(long));
        memcpy(freq_nt, sp.freq_nt.data, nfreq * sizeof(long));
        memcpy(freq_sd_off, sp.freq_sd_off.data, nfreq * sizeof(long));
        memcpy(sparse_data, sp.sparse_data.data, sp.sparse_data.size * sizeof(float));
    });
}

// SinglePulse::add_to_timestream on a C-contiguous (nfreq, nt) float32 array starting at out_it0.
__attribute__((visibility("default")))
int ref_pulse_add_to_timestream(void *hv, float *out, long nfreq, long nt, long out_it0, float weight)
{
    return guard([&] {
        const SinglePulse &sp = *((RefPulse *) hv)->sp;
        ksgpu::Array<float> a({nfreq, nt}, ksgpu::af_uhost);
        memcpy(a.data, out, nfreq * nt * sizeof(float));
        sp.add_to_timestream(a, out_it0, weight);
        memcpy(out, a.data, nfreq * nt * sizeof(float));
    });
}

}  // extern "C"
