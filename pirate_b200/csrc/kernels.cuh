// kernels.cuh -- device-side data structures shared by the B200 dedispersion kernels and their host driver.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "regtree.cuh"

namespace pb2 {

// Split of a rank-R tree into register trees: phase b takes the upper RB = ceil(R/2) row bits (for a
// stage-2 tree this is its peak-finding rank, so subband rows come out of phase b aligned).
__host__ __device__ constexpr int split_rb(int R) { return (R + 1) / 2; }
__host__ __device__ constexpr int split_ra(int R) { return R - (R + 1) / 2; }

// Threads per block of a two-phase tree kernel of rank R: one warp per phase-a group (2^RB of
// them) followed by one warp per phase-b group (2^RA).
__host__ __device__ constexpr int tree_threads(int R)
{
    return 32 * ((1 << split_ra(R)) + (1 << split_rb(R)));
}

// Stage 1 (one primary tree): input rows -> two-phase tree -> per-row output delay lines.
struct Stage1Args
{
    int rank;               // stage-1 dd rank (rows per block = 2^rank)
    long state_per_block;   // floats
    float *state;           // (total_beams, nblocks, state_per_block)

    // Input element (b, row c, time s) at in + (in_beam0 + b)*in_beam_stride + c*in_row_stride + (s & in_mask),
    // (in_lag0 and in_lag1 must be zero: rows are read aligned).
    const void *in;
    long in_beam_stride, in_row_stride, in_mask;
    long in_s0;             // time of the chunk's first sample in the input's indexing
    int in_lag0, in_lag1;
    int in_beam0;

    // Output delay lines: row (a, n) -> ring + bt*ring_beam_stride + ring_off[row], capacity ring_cap[row].
    void *ring;
    const long *ring_off;
    const int *ring_cap;
    long ring_beam_stride;

    long s0;                // stream time of the chunk's first sample (ichunk * nt)
    int nt;                 // samples per chunk at this tree's time resolution
    int beam0;              // total-beam index of batch beam 0
    // If not null, the chunk index is read from device memory at launch (a replayed CUDA graph advances
    // it): s0 = *chunk_ctr * nt, and in_s0 = *chunk_ctr * nt for delay-line inputs (in_mask != -1).
    const long *chunk_ctr;
};

// Stage 2 (one output tree): stage-1 delay lines -> two-phase subband tree -> peak-finder delay lines.
struct Stage2Args
{
    int rank;               // stage-2 dd rank (rows per block = 2^rank)
    long state_per_block;
    float *state;           // (total_beams, 2^amb_rank, state_per_block)

    // Input: stage-1 delay lines of the primary tree; row (a, d) = a * 2^amb_rank + d.
    const void *ring;
    const long *ring_off;
    const int *ring_cap;
    long ring_beam_stride;
    int amb_rank;           // stage-2 ambient rank (= stage-1 dd rank)
    int uflag;              // 1 for downsampled primary trees (upper half of the DM range)

    // Subbands: counts per pf level (0..pf_rank) and first multiplet index of each level.
    int sb_count[5];
    int sb_mbase[5];

    // Output: peak-finder delay lines, row ((bt*ndm_out + dm) * M + m), capacity pf_cap (power of two).
    void *pf;
    int M;
    int ndm_out;
    long pf_cap;

    long s0;
    int nt;
    int beam0;
    const long *chunk_ctr;  // if not null: s0 = *chunk_ctr * nt
};

// Arguments of the peak-finding kernel (one output tree).
struct PfArgs
{
    const void *pf;         // delay lines written by the stage-2 kernel (subband-aligned)
    long pf_cap;
    const float *wt;        // (B, ndm_wt, nt_wt, P, N) for this batch
    void *out_max;          // (B, ndm_out, nt_out), storage dtype
    uint32_t *out_argmax;   // (B, ndm_out, nt_out)
    const int *m_to_n;      // (M,)
    int M, N, P, L;         // multiplets, subbands, profiles, boxcar levels
    int ndm_out, nt_out, ndm_wt, nt_wt;
    int Dout, Dcore, tpad;
    long s0;                // stream time of the chunk's first sample
    int beam0;
    const long *chunk_ctr;  // if not null: s0 = *chunk_ctr * nt_chunk
    int nt_chunk;
    int force_general;      // 1: the general kernel even where the fast one applies
};

// Arguments of the fused tree-gridding + lagged-downsampling kernel.
struct GridLdsArgs
{
    const void *in;         // input (B, F, T) storage dtype
    void *tree0;            // level-0 tree (B, 2^rank, T) storage dtype
    const int *chan_f0;     // (2^rank,) first input channel of tree channel n
    const int *chan_cnt;    // (2^rank,) number of input channels
    const int *chan_woff;   // (2^rank,) offset into chan_w
    const float *chan_w;    // overlap weights, ascending input channel
    int F, rank, T, nlev;   // nlev = num_primary_trees - 1
    void *ring[6];          // per level p=1..nlev: delay lines (total_beams, 2^(rank-1), cap[p])
    long cap_mask[6];
    float *state;           // (2, total_beams, nlev, 2^(rank-1)) last even-channel sample per level
    int lag_rank;           // output row c is written delayed by 2^lag_rank - 1 - (c mod 2^lag_rank) samples
    long ichunk;
    int beam0, B, total_beams;
    // int4 input in place of 'in' (null when the input is in the storage dtype): q_data (B, F, T/2)
    // bytes, two samples per byte (low nibble first); q_scoff (B, F, T/256, 2) fp16 (scale, offset).
    const void *q_data;
    const void *q_scoff;
    const long *chunk_ctr;  // if not null: the chunk index is *chunk_ctr instead of ichunk
    int block_target;       // threads per block to aim for (0: 128); blocks hold whole rows of windows
};

// Floats of persistent state per block of the stage kernels (host and device agree by construction).
// Per-block state, rounded up to a multiple of 4 floats so that every block's state starts on a
// 16-byte boundary (the kernels move its delay-line part with 16-byte copies).
inline long stage1_state_floats(int R) { return (tree_state_floats(split_ra(R), split_rb(R), false) + 3) & ~3L; }
inline long stage2_state_floats(int R) { return (tree_state_floats(split_ra(R), split_rb(R), true) + 3) & ~3L; }

// Per-beam peak of a batch's outputs, as pirate's toy grouper reduces them (pirate_frb/run_toy_grouper.py:
// 79-116): over every tree, the maximum of out_max[tree][b] and its first (dm, time) position; a tree
// whose maximum is NaN is passed over; across trees the first tree with the strictly largest maximum
// wins. peak/tree/idm/itime/token hold nbeams entries (peak -inf and tree -1 when no tree qualified).
constexpr int kBeamPeakMaxTrees = 64;
struct BeamPeakArgs
{
    int ntrees;
    long ndm[kBeamPeakMaxTrees], nt[kBeamPeakMaxTrees];
    const void *out_max[kBeamPeakMaxTrees];
    const uint32_t *out_argmax[kBeamPeakMaxTrees];
    float *peak;
    int *tree, *idm, *itime;
    uint32_t *token;
};
void launch_beam_peaks(const BeamPeakArgs &a, int dtype, long nbeams, cudaStream_t s);
// The same reduction spread over nsplit blocks per (tree, beam) (a few beams fill a few SMs otherwise),
// then one warp per beam combines the partial results. scratch: nbeams * ntrees * nsplit * 16 bytes.
void launch_beam_peaks_split(const BeamPeakArgs &a, int dtype, long nbeams, void *scratch, int nsplit, cudaStream_t s);

// Adds a sparse pulse (channel f: cnt[f] samples from sample index it0[f], values data[off[f] ...])
// times 'weight' to the chunk out (nfreq rows of row_stride elements, dtype 0/1/2 = f32/f16/bf16)
// holding samples [chunk_it0, chunk_it0 + nt); samples outside the chunk are skipped. The index
// arrays and data are device arrays.
void launch_pulse_inject(void *out, int dtype, long nfreq, long nt, long row_stride, long chunk_it0, const long *it0,
                         const long *cnt, const long *off, const float *data, float weight, cudaStream_t s);

// Host spill of stage-1 delay lines (the MegaRingbuf host zones of pirate, src_lib/MegaRingbuf.cpp:155-183,
// and its g2h/h2g copies, src_lib/GpuDedisperser.cpp:628-707). A spilled row's readers all need chunks
// d = ceil((lag + 1) / nt) >= 2 back; on the GPU it keeps a one-chunk write slot (stage 1 writes chunk c
// there) and a two-chunk read ring (stage 2 reads chunks c - d and c - d + 1 there); in mapped pinned host
// memory its zone (all rows of equal d) keeps S = d + 1 chunk slots per beam. Per step, after stage 1,
// the g2h kernel copies every spilled row's chunk c to host slot c mod S, and the h2g kernel copies chunk
// c - d + 1 from host slot (c - d + 1) mod S into read-ring half (c - d + 1) mod 2.
struct SpillRow
{
    long w_off;     // write slot (nt samples) in the beam's delay-line region
    long r_off;     // read ring (2 nt samples) in the beam's delay-line region
    long h_base;    // the row's zone in the host buffer: element (slot, beam, k, t) at
                    // h_base + ((slot * total_beams + beam) * n_z + k) * nt + t
    int n_z, k, S, d;
};
struct SpillArgs
{
    void *ring;                 // stage-1 delay lines (total_beams regions of ring_beam_stride samples)
    long ring_beam_stride;
    void *host;                 // mapped pinned host buffer (device-accessible pointer)
    const SpillRow *rows;       // device table of the spilled rows
    int nrows, nt, esize, total_beams, beam0, B;
    long ichunk;
    const long *chunk_ctr;      // if not null: the chunk index is *chunk_ctr
};
void launch_spill_g2h(const SpillArgs &a, cudaStream_t s);
void launch_spill_h2g(const SpillArgs &a, cudaStream_t s);

void launch_grid_lds(const GridLdsArgs &a, int dtype, cudaStream_t s);
// int4 -> out_dtype dequantization of (nbeams, nfreq, ntime) samples (ntime a multiple of 256).
void launch_dequantize(void *out, int out_dtype, const void *data, const void *scales_offsets, long nbeams, long nfreq,
                       long ntime, cudaStream_t s);
void launch_stage1(const Stage1Args &a, int dtype, int nblocks, int B, cudaStream_t s);
void launch_stage2(const Stage2Args &a, int dtype, int nblocks, int B, cudaStream_t s);

// Stage 2 of several output trees that use the same kernel (same dd rank and staggered-subband flag)
// as one grid: blocks [blk0[i], blk0[i+1]) are tree i's. One grid has one partial last wave instead of
// one per tree (the downsampled trees' grids are 3.5 waves).
constexpr int kStage2MaxTrees = 8;
struct Stage2Multi
{
    Stage2Args t[kStage2MaxTrees];
    int blk0[kStage2MaxTrees + 1];
    int n;
};
bool stage2_same_kernel(const Stage2Args &x, const Stage2Args &y);
void launch_stage2_multi(const Stage2Args *a, const int *nblocks, int n, int dtype, int B, cudaStream_t s);
void launch_pf(const PfArgs &a, int dtype, int B, cudaStream_t s);

struct DedispersionPlan;
void dedisperse_chunk_noalloc(const DedispersionPlan &plan, const void *in, const float *const *weights,
                              void *const *out_max, uint32_t *const *out_argmax, cudaStream_t stream);

}  // namespace pb2
