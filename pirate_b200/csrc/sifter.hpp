// sifter.hpp -- the learned candidate sifter behind the threshold peak finder.
//
// A candidate is one beam's strongest peak-finder output of a chunk above a threshold (the toy
// grouper's per-beam reduction, pirate_frb/run_toy_grouper.py:79-116). Its patch is a window of the
// dedispersed data around the peak, read from the stage-2 subband rows of the peak's tree:
//   9 fine DMs (the peak's fine DM +-4) x 32 output times x 6 boxcar widths (1, 2, 4, ..., 32),
// each value a trailing boxcar sum of the rows scaled to sigma units (each row times the peak finder's
// width-1 full-band weight, 1/sqrt(variance), of its coarse DM) divided by sqrt(width), then
// compressed as 8 asinh(x / 8) (linear within +-8 sigma, logarithmic beyond), stored fp16.
// The sifter is an MLP 1728 -> 256 -> 128 -> 1 (ReLU) with bf16 weights and FP32 accumulation on the
// tensor cores (mma.sync m16n8k16 bf16), trained with its own forward/backward/Adam kernels on the
// binary cross-entropy of the logit. The threshold peak finder stays the fallback and the yardstick of the
// sifter's recall and false-alarm rate.

#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

namespace pb2 {

constexpr int kPatchDm = 9, kPatchT = 32, kPatchW = 6;
constexpr int kPatchLen = kPatchDm * kPatchT * kPatchW;   // 1728
constexpr int kPatchPeakAt = 23;                          // window time index of the peak's last sample
constexpr int kMlpIn = kPatchLen, kMlpH1 = 256, kMlpH2 = 128;
constexpr int kPatchMaxTrees = 16;

// One output tree's stage-2 subband rows, as the patch kernel reads them.
struct PatchTree
{
    const void *pf;       // rows ((beam * ndm_out + dm) * M + m), capacity pf_cap (power of two)
    long pf_cap;
    int M, ndm_out, nt_ds, Dout, Dcore, pf_rank;
    int d_to_m[16];       // full-band multiplet of fine DM offset d < 2^pf_rank (-1: none)
    // Peak-finder weights of this batch, (B, ndm_wt, nt_wt, P, N): the row scale of coarse dm 'c' and
    // output time 'it' is wt[((b * ndm_wt + c / (ndm_out / ndm_wt)) * nt_wt + it / (nt_out / nt_wt)) * P * N + nfull].
    const float *wt;
    int ndm_wt, nt_wt, nt_out, P, N, nfull;
};

struct PatchArgs
{
    int ntrees;
    PatchTree t[kPatchMaxTrees];
    // Per batch beam b (B of them): the beam's peak (beam-peak kernel outputs).
    const float *peak;
    const int *tree, *idm, *itime;
    const uint32_t *token;
    float threshold;
    long ichunk;
    const long *chunk_ctr;  // if not null: the chunk index is *chunk_ctr instead of ichunk
    int beam0, B;
    uint16_t *patches;    // (B, 1728) fp16 bits, layout ((d * 32 + j) * 6 + w)
    int *valid;           // (B,) 1 where peak >= threshold
};
void launch_patches(const PatchArgs &a, int dtype, cudaStream_t s);

// Sets scores[b] = logits[b] where valid[b], else -inf.
void launch_mask_scores(const float *logits, const int *valid, float *scores, int n, cudaStream_t s);

// The MLP (weights in pirate's/PyTorch's Linear layout: W (out, in) row-major).
class Sifter
{
public:
    Sifter(int device, long max_batch, uint64_t seed);
    ~Sifter();
    Sifter(const Sifter &) = delete;
    Sifter &operator=(const Sifter &) = delete;

    // Host fp32 parameters in the order W1 (256x1728), b1, W2 (128x256), b2, W3 (1x128), b3.
    static long nparams();
    void set_params(const float *host);
    void get_params(float *host) const;

    // logits[n] (device) of n patches (device fp16 (n, 1728)), on 'stream'.
    void forward(const uint16_t *patches, long n, float *logits, cudaStream_t stream);
    // Mean binary cross-entropy gradients of a batch (labels 0/1, device) into host 'grad' (nparams
    // floats, same order as the parameters); returns the loss. Synchronizes.
    double gradients(const uint16_t *patches, const float *labels, long n, float *grad_host, cudaStream_t stream);
    // One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on a batch; returns the batch loss. Synchronizes.
    double train_step(const uint16_t *patches, const float *labels, long n, float lr, cudaStream_t stream);

    int device = 0;
    long max_batch = 0;

private:
    void backward(const uint16_t *patches, const float *labels, long n, cudaStream_t stream);
    void refresh_bf16(cudaStream_t stream);

    float *master = nullptr;     // nparams fp32
    float *grad = nullptr;       // nparams fp32
    float *adam_m = nullptr, *adam_v = nullptr;
    uint16_t *wb = nullptr;      // bf16 copies of W1, W2, W3 (biases stay fp32)
    float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr, *g = nullptr, *loss = nullptr;
    uint16_t *h1 = nullptr, *h2 = nullptr;   // bf16 activations
    float *g2 = nullptr, *g1 = nullptr;
    long step = 0;
};

}  // namespace pb2
