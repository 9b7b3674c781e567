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

#include "pirate/DedispersionConfig.hpp"
#include "pirate/DedispersionPlan.hpp"
#include "pirate/Dedisperser.hpp"
#include "pirate/PeakFindingKernel.hpp"
#include "pirate/ReferenceLagbuf.hpp"
#include "pirate/ReferenceTree.hpp"

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace pirate;

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

}  // extern "C"
