// regtree.cuh -- register-resident tree dedispersion (lane = time sample) used by the stage kernels.
//
// A rank-R tree (rows i, butterfly at step r pairs i and i + 2^r with lag bit_reverse(i mod 2^r, r)) is
// computed as two register trees joined by a delay line:
//
//   phase a: rank RA over the low RA row bits (one warp per group of 2^RA consecutive rows),
//   delay:   row (f, d) of the phase-a output is delayed by P(f, d) = (2^RB - 1 - f) * bit_reverse(d, RA),
//   phase b: rank RB over the high RB row bits (one warp per phase-a output index d).
//
// Shifting a row in time commutes with the butterflies' adds, so every output is the same fp32
// expression of the same inputs as in the one-shot tree (bitwise identical); the phase-b butterfly
// lags reduce to bit_reverse(j, r') < 2^RB. Outputs produced after phase-b step r' of a subband tree
// carry the delay (2^RB - fhi) * bit_reverse(d, RA), which is exactly the subband alignment lag of
// pirate's ReferenceTree (src_lib/ReferenceTree.cpp:41-50), so subband rows come out aligned.
//
// Within a register tree a lane holds one time sample of 2^K rows. A butterfly needs row0 at t-L and
// t-L-1 (L < 32): each lane offers its current value, or its value from the previous 32-sample tile
// if the reader is in the next tile, and one shuffle moves it (one shuffle per lagged operand).

#pragma once

#include <cstdint>

namespace pb2 {

__host__ __device__ constexpr int bitrev_c(int x, int n)
{
    int r = 0;
    for (int i = 0; i < n; i++) r = (r << 1) | ((x >> i) & 1);
    return r;
}

// Lag of pair q (0 <= q < 2^(K-1)) at step r of a register tree.
__host__ __device__ constexpr int rt_lag(int r, int q) { return bitrev_c(q & ((1 << r) - 1), r); }

// Compact state of a rank-K register tree: pair (r, q) keeps (lag+1) samples.
__host__ __device__ constexpr int rt_state(int K)
{
    int s = 0;
    for (int r = 0; r < K; r++)
        for (int q = 0; q < (1 << (K > 0 ? K - 1 : 0)) && K > 0; q++) s += rt_lag(r, q) + 1;
    return s;
}

__host__ __device__ constexpr int rt_off(int K, int r0, int q0)
{
    int s = 0;
    for (int r = 0; r < K; r++)
        for (int q = 0; q < (1 << (K > 0 ? K - 1 : 0)) && K > 0; q++) {
            if (r == r0 && q == q0) return s;
            s += rt_lag(r, q) + 1;
        }
    return s;
}

// Staggered subband butterflies of a rank-K phase-b tree at step r: pairs (2k+1, 2k+2) of the
// (K - r)-bit upper index, k < 2^(K-r-1) - 1, for every lower index j < 2^r.
__host__ __device__ constexpr int st_count(int K, int r) { return (K - r - 1 >= 0) ? (((1 << (K - r - 1)) - 1) << r) : 0; }

__host__ __device__ constexpr int st_state(int K)
{
    int s = 0;
    for (int r = 0; r < K; r++)
        for (int u = 0; u < st_count(K, r); u++) s += rt_lag(r, u & ((1 << r) - 1)) + 1;
    return s;
}

__host__ __device__ constexpr int st_off(int K, int r0, int u0)
{
    int s = 0;
    for (int r = 0; r < K; r++)
        for (int u = 0; u < st_count(K, r); u++) {
            if (r == r0 && u == u0) return s;
            s += rt_lag(r, u & ((1 << r) - 1)) + 1;
        }
    return s;
}

// Delay line between the phases: row (f, d) holds P(f, d) + 65 samples (phase a writes tile k while
// phase b reads tile k-1 and, for step 0, the sample before it), rounded up to a multiple of 32 so
// that a tile never wraps on write.
__host__ __device__ constexpr int ring_cap(int RA, int RB, int f, int d)
{
    return (((1 << RB) - 1 - f) * bitrev_c(d, RA) + 65 + 31) & ~31;
}

__host__ __device__ constexpr int ring_floats(int RA, int RB)
{
    int s = 0;
    for (int f = 0; f < (1 << RB); f++)
        for (int d = 0; d < (1 << RA); d++) s += ring_cap(RA, RB, f, d);
    return s;
}

// Per-block persistent state of a two-phase tree: delay line + phase-a, phase-b (and staggered) histories.
__host__ __device__ constexpr int tree_state_floats(int RA, int RB, bool subbands)
{
    return ring_floats(RA, RB) + (1 << RB) * rt_state(RA) + (1 << RA) * (rt_state(RB) + (subbands ? st_state(RB) : 0));
}

}  // namespace pb2
