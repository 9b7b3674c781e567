// kernels.cuh -- device-side data structures shared by the B200 dedispersion kernels and their host driver.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pb2 {

// Tree samples per tile in the tree kernels (one warp-wide run of samples per row).
constexpr int kTreeTile = 32;
constexpr int kTreeThreads = 512;
constexpr int kMaxTreeRows = 256;   // 2^8: stage ranks are <= 8 for tree rank <= 16

// One operation of a tree "program". A program is a list of phases; phase k is
// ops[phase_begin[k] .. phase_begin[k+1]) and all ops of a phase read the rows as they were at the
// start of the phase.
//
//  kind 0 (butterfly, in place):  row0' = (row0[t-lag]   + row1[t]) / sqrt2
//                                 row1' = (row0[t-lag-1] + row1[t]) / sqrt2
//  kind 1 (staggered butterfly):  same arithmetic, results only go to outputs out0/out1
//  kind 2 (copy):                 out0 = row0[t]
//
// Butterflies keep the last (lag+1) samples of their row0 input in a history delay line of
// capacity hist_mask+1 (a power of two) at offset hist_off of the block's history area.
// out0/out1 >= 0 name subband output rows (stage-2 programs), -1 for none.
struct TreeOp
{
    int16_t row0, row1;
    int16_t kind, pad;
    int32_t lag;
    int32_t hist_off;
    int32_t hist_mask;
    int32_t out0, out1;
};

// Arguments of the stage-1 tree kernel (one primary tree).
struct Stage1Args
{
    const TreeOp *ops;
    const int *phase_begin;
    int nphases;
    int nrows;              // 2^stage1_dd_rank
    long hist_per_block;    // floats of history per (beam, block)
    float *hist;            // (total_beams, nblocks, hist_per_block)

    // Input rows: element (b, row c, time s) at in + b*in_beam_stride + c*in_row_stride + ((s - lag(c)) & in_mask),
    // lag(c) = in_lag0 - in_lag1 * (c % nrows); s counts samples of this tree's time base.
    const void *in;
    long in_beam_stride, in_row_stride, in_mask;
    long in_s0;             // time of the chunk's first sample in the input's indexing
    int in_lag0, in_lag1;
    int in_beam0;           // beam index of batch beam 0 in the input (0 for per-batch buffers)

    // Output delay lines: row (a, n) -> ring + b*ring_beam_stride + ring_off[row], capacity ring_cap[row].
    void *ring;
    const long *ring_off;
    const int *ring_cap;
    long ring_beam_stride;

    long s0;                // stream time of the chunk's first sample (ichunk * nt)
    int nt;                 // samples per chunk at this tree's time resolution
    int beam0;              // total-beam index of batch beam 0
};

// Arguments of the stage-2 tree kernel (one output tree).
struct Stage2Args
{
    const TreeOp *ops;
    const int *phase_begin;
    int nphases;
    int nrows;              // 2^tree.dd_rank
    long hist_per_block;
    float *hist;            // (total_beams, 2^amb_rank, hist_per_block)

    // Input: stage-1 delay lines of the primary tree; row (a, d) = a * 2^amb_rank + d.
    const void *ring;
    const long *ring_off;
    const int *ring_cap;
    long ring_beam_stride;
    int amb_rank;           // stage-2 ambient rank (= stage-1 dd rank)
    int dd_rank;            // stage-2 active rank (= rows)
    int uflag;              // 1 for downsampled primary trees (upper half of the DM range)

    // Output: peak-finder delay lines, row ((b*ndm_out + dm) * M + m), capacity pf_cap (power of two).
    void *pf;
    int M;
    int ndm_out;
    int pf_shift;           // dd_rank - pf_rank: coarse dm of block d starts at bitrev(d) << pf_shift
    long pf_cap;

    long s0;
    int nt;
    int beam0;
};

// Arguments of the peak-finding kernel (one output tree).
struct PfArgs
{
    const void *pf;         // delay lines written by the stage-2 kernel
    long pf_cap;
    const float *wt;        // (B, ndm_wt, nt_wt, P, N) for this batch
    void *out_max;          // (B, ndm_out, nt_out), storage dtype
    uint32_t *out_argmax;   // (B, ndm_out, nt_out)
    const int *m_to_n;      // (M,)
    const int *final_lag;   // (2^pf_shift, M): subband alignment lag of (pf_dm, m)
    int M, N, P, L;         // multiplets, subbands, profiles, boxcar levels
    int ndm_out, nt_out, ndm_wt, nt_wt;
    int Dout, Dcore, tpad;
    int pf_shift;
    long s0;                // stream time of the chunk's first sample
    int beam0;
};

// Arguments of the tree-gridding kernel.
struct GridArgs
{
    const void *in;         // (B, F, T) storage dtype
    void *out;              // (B, N, T) storage dtype
    const int *chan_f0;     // (N,) first input channel of tree channel n
    const int *chan_cnt;    // (N,) number of input channels
    const int *chan_woff;   // (N,) offset into chan_w
    const float *chan_w;    // overlap weights, ascending input channel
    int F, N, T;
};

// Arguments of the lagged-downsampling kernel.
struct LdsArgs
{
    const void *in;         // level-0 tree (B, 2^rank, T) storage dtype
    int rank, T, nlev;      // nlev = num_primary_trees - 1
    void *ring[6];          // per level p=1..nlev: delay lines (total_beams, 2^(rank-1), cap[p])
    long cap_mask[6];
    float *state;           // (2, total_beams, nlev, 2^(rank-1)) last even-channel sample per level
    long ichunk;
    int beam0, B, total_beams;
};

void launch_grid(const GridArgs &a, int dtype, int B, cudaStream_t s);
void launch_lds(const LdsArgs &a, int dtype, cudaStream_t s);
void launch_stage1(const Stage1Args &a, int dtype, int nblocks, int B, cudaStream_t s);
void launch_stage2(const Stage2Args &a, int dtype, int nblocks, int B, cudaStream_t s);
void launch_pf(const PfArgs &a, int dtype, int B, cudaStream_t s);

}  // namespace pb2
