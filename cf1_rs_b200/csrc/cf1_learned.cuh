// Host-side owner of the per-bin learned index (built by cf1_learned.cu).
#pragma once
#include "cf1_internal.cuh"

namespace cf1 {

constexpr int LI_NPARAM = 3 * LI_HIDDEN + 1;  // w1, b1, w2, b2

struct LearnedOpts {
  int train_steps = 300;       // < 0: no training (root stays the identity CDF y = x)
  float lr = 0.02f;
  uint32_t max_samples = 2048; // CDF samples per bin
  uint32_t leaf_size = 32;     // target keys per leaf
  uint32_t max_err = 1024;     // bins with a larger leaf error fall back to BBHash
};

struct LearnedStats {
  uint64_t learned_bins = 0, fallback_bins = 0, max_err = 0, leaves = 0, bytes = 0;
  uint64_t max_err_all = 0;     // largest leaf error over every non-empty bin
  uint64_t verify_miss_bins = 0; // bins where some key fell outside its window
  double mean_err = 0;         // mean leaf error bound over keys of learned bins
  double mean_window = 0;      // mean search window (2*err+1) over keys of learned bins
  double train_loss = 0;       // mean final training loss over bins
};

template <class KeyT>
struct LearnedBuild {
  uint32_t nbins = 0;
  LearnedStats stats;
  LearnedBuild() = default;
  LearnedBuild(const LearnedBuild &) = delete;
  LearnedBuild &operator=(const LearnedBuild &) = delete;

  // keys: distinct keys, bins in order, each sorted; dist_off device [nbins+1].
  // On return fallback_sel[b] (device) is 1 for bins that BBHash must serve.
  void build(const KeyT *keys, const uint64_t *dist_off, uint32_t nbins, int k, const LearnedOpts &o, cudaStream_t s);
  LIView view(int k) const;
  const uint32_t *fallback_sel() const { return sel_.as<const uint32_t>(); }
  const LIRoot *roots_device() const { return roots_.as<const LIRoot>(); }
  const LILeaf *leaves_device() const { return leaves_.as<const LILeaf>(); }

 private:
  DevBuf roots_, leaves_, lfirst_, llast_, ln_, leaf_off_, tile_off_, sel_, loss_, errsum_;
};

// Full-batch MSE loss and gradient of the root MLP on the device (the same
// code the training kernel runs).  params: LI_NPARAM floats.  Host pointers.
void learned_grad_host(const float *params, const float *x, const float *t, size_t n, float *grad, float *loss);
// dL/dQ of one training step (Q = knot logits[16], w2[16], b2), on the current device.
void learned_grad_q_host(const float *q, const float *x, const float *t, size_t n, float *grad_q, float *loss);

}  // namespace cf1
