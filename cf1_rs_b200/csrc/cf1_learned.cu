// Per-bin learned index over the bins' sorted distinct keys.
//
// Two stages per bin (a recursive-model index):
//   root  : an MLP 1 -> LI_HIDDEN (ReLU) -> 1 trained on the GPU to map the
//           key's scaled top bits x to its rank fraction (the bin's empirical
//           CDF); leaf = floor(root(x) * n_leaves);
//   leaves: per leaf a line through its first and last key's (key, rank);
//           err = max |prediction - rank| over the keys the root sends there.
// A query evaluates the root, the leaf's line, and searches the sorted keys
// in [pred - err, pred + err].  A verification pass queries every key; a bin with a
// key outside its window, or with err above the threshold, is served by
// BBHash instead.
//
// The hidden units are clipped ReLUs, clamp(w1 x + b1, 0, 1): a sum of
// bounded non-decreasing ramps can follow any non-decreasing CDF, concave
// ones included (canonical k-mers are denser at small values).  Training
// projects the weights of both layers onto [0, inf) after every step.  With
// non-negative weights every rounded fma and the clamp are non-decreasing,
// so root(x) -- and the leaf index -- is non-decreasing in the key: the keys
// routed to a leaf are one contiguous run of ranks, and a leaf's error bound
// only measures how far the run bends from its line.  Before training the root is the identity (y = x), which
// is the same index without the network: the comparison of the two is
// reported in the stats.
#include <cmath>
#include <cstring>

#include "cf1_device_util.cuh"
#include "cf1_learned.cuh"
#include "cf1_mphf.cuh"

namespace cf1 {

namespace {

constexpr int LT_BLOCK = 256;
constexpr int LT_NW = LT_BLOCK / 32;
constexpr uint32_t LT_TILE = 4096;
constexpr uint32_t LT_MAX_SAMPLES = 4096;
constexpr int H = LI_HIDDEN;

// Adds one sample's MSE term (weight `scale`) and its gradient to g.
// Parameter layout: w1[0,H) b1[H,2H) w2[2H,3H) b2[3H]; hidden units are
// clipped ReLUs clamp(w1 x + b1, 0, 1) (li_act).  Queries evaluate the same
// function on its piecewise-linear form (LIRoot, li_root_eval).
CF1_HD void mlp_accumulate(const float *P, float x, float t, float scale, float *g, float &loss) {
  float z[H];
  float y = P[3 * H];
#pragma unroll
  for (int j = 0; j < H; j++) {
    z[j] = f_fma(P[j], x, P[H + j]);
    y = f_fma(P[2 * H + j], li_act(z[j]), y);
  }
  float e = y - t;
  loss += e * e * scale;
  float dy = 2.f * e * scale;
  g[3 * H] += dy;
#pragma unroll
  for (int j = 0; j < H; j++) {
    g[2 * H + j] += dy * li_act(z[j]);
    float dz = (z[j] > 0.f && z[j] < 1.f) ? dy * P[2 * H + j] : 0.f;
    g[j] += dz * x;
    g[H + j] += dz;
  }
}

// Trained parameters Q (2H+1): knot logits theta[H], output weights w2[H],
// output bias b2.  The first layer is derived from the knots: widths
// d = softmax(theta), knots t_j = sum_{i<j} d_i, w1_j = 1/d_j,
// b1_j = -t_j/d_j, so unit j ramps over [t_j, t_j + d_j] and the ramps tile
// [0, 1] without gaps (a gap would be a flat stretch of the root, sending
// every key in it to one leaf).
constexpr int LI_NQ = 2 * H + 1;

// P (the MLP's w1 b1 w2 b2) from Q; d and t kept for the chain rule.
CF1_D void derive_params(const float *Q, float *P, float *d, float *t) {
  float m = Q[0];
  for (int j = 1; j < H; j++) m = fmaxf(m, Q[j]);
  float s = 0.f;
  for (int j = 0; j < H; j++) {
    d[j] = expf(Q[j] - m);
    s += d[j];
  }
  float acc = 0.f;
  for (int j = 0; j < H; j++) {
    d[j] = d[j] / s;
    t[j] = acc;
    acc += d[j];
    P[j] = 1.f / d[j];
    P[H + j] = -t[j] / d[j];
    P[2 * H + j] = Q[H + j];
  }
  P[3 * H] = Q[2 * H];
}

// dL/dQ from dL/dP (chain rule through w1 = 1/d, b1 = -t/d, the knot sums
// and the softmax).
CF1_D void grad_q(const float *G, const float *d, const float *t, float *GQ) {
  float gd[H];
  for (int j = 0; j < H; j++) gd[j] = -G[j] / (d[j] * d[j]) + G[H + j] * t[j] / (d[j] * d[j]);
  float acc = 0.f;  // t_j = sum_{i<j} d_i: d_i collects dL/dt_j of every j > i
  for (int j = H - 1; j >= 0; j--) {
    gd[j] += acc;
    acc += -G[H + j] / d[j];
  }
  float dot = 0.f;
  for (int j = 0; j < H; j++) dot += d[j] * gd[j];
  for (int j = 0; j < H; j++) GQ[j] = d[j] * (gd[j] - dot);
  for (int j = 0; j < H; j++) GQ[H + j] = G[2 * H + j];
  GQ[2 * H] = G[3 * H];
}

// Adam step size per group: logits O(1), output weights O(1/H).
CF1_D float lr_scale_q(int q) { return q < H ? 1.f : 1.f / (float)H; }

// Block reduction of the NPARAM gradient sums and the loss into red/sl.
CF1_D void reduce_grads(float *g, float loss, float (*red)[LI_NPARAM + 1]) {
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
#pragma unroll
  for (int p = 0; p < LI_NPARAM; p++) {
    float v = warp_sum(g[p]);
    if (lane == 0) red[warp][p] = v;
  }
  float l = warp_sum(loss);
  if (lane == 0) red[warp][LI_NPARAM] = l;
}

template <class KeyT>
__global__ void __launch_bounds__(LT_BLOCK) li_train_kernel(const KeyT *keys, const uint64_t *dist_off, LIRoot *roots,
                                                           int k, int steps, float lr, uint32_t max_samples,
                                                           float *loss_out) {
  __shared__ float sx[LT_MAX_SAMPLES], st[LT_MAX_SAMPLES];
  __shared__ float P[LI_NPARAM], Q[LI_NQ], GQ[LI_NQ], M1[LI_NQ], M2[LI_NQ], sd[H], stk[H];
  __shared__ float red[LT_NW][LI_NPARAM + 1];
  __shared__ float s_loss;
  const uint32_t b = blockIdx.x;
  const unsigned tid = threadIdx.x;
  const uint64_t base = dist_off[b], n = dist_off[b + 1] - base;
  LIRoot &R = roots[b];
  uint64_t hmin = 0, hmax = 0;
  float inv = 0.f;
  if (n) {
    hmin = KOps<KeyT>::high64(keys[base], k);
    hmax = KOps<KeyT>::high64(keys[base + n - 1], k);
    inv = hmax > hmin ? __fdiv_rn(1.f, u64_to_f(hmax - hmin)) : 0.f;
  }
  uint32_t S = (uint32_t)(n < max_samples ? n : max_samples);
  for (uint32_t i = tid; i < S; i += LT_BLOCK) {
    uint64_t r = (uint64_t)i * n / S;
    uint64_t h = KOps<KeyT>::high64(keys[base + r], k);
    sx[i] = f_mul(u64_to_f(h - hmin), inv);
    st[i] = (float)((double)r / (double)n);
  }
  if (tid < LI_NQ) {
    // identity root: equal knot logits (unit j ramps over [j/H, (j+1)/H]),
    // output weights 1/H, so root(x) = x -- the index without a trained network
    Q[tid] = tid < H ? 0.f : (tid < 2 * H ? 1.f / (float)H : 0.f);
    M1[tid] = 0.f;
    M2[tid] = 0.f;
  }
  if (tid == 0) s_loss = 0.f;
  __syncthreads();
  if (tid == 0) derive_params(Q, P, sd, stk);
  __syncthreads();
  const float scale = S ? 1.f / (float)S : 0.f;
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  float b1t = 1.f, b2t = 1.f;
  for (int step = 0; step < steps && S > 0; step++) {
    float g[LI_NPARAM];
#pragma unroll
    for (int p = 0; p < LI_NPARAM; p++) g[p] = 0.f;
    float loss = 0.f;
    for (uint32_t i = tid; i < S; i += LT_BLOCK) mlp_accumulate(P, sx[i], st[i], scale, g, loss);
    reduce_grads(g, loss, red);
    __syncthreads();
    if (tid == 0) {
      float G[LI_NPARAM];
      for (int p = 0; p < LI_NPARAM; p++) {
        float v = 0.f;
        for (int w = 0; w < LT_NW; w++) v += red[w][p];
        G[p] = v;
      }
      grad_q(G, sd, stk, GQ);
      float l = 0.f;
      for (int w = 0; w < LT_NW; w++) l += red[w][LI_NPARAM];
      s_loss = l;
    }
    __syncthreads();
    if (tid < LI_NQ) {
      float G = GQ[tid];
      b1t *= beta1;
      b2t *= beta2;
      M1[tid] = beta1 * M1[tid] + (1.f - beta1) * G;
      M2[tid] = beta2 * M2[tid] + (1.f - beta2) * G * G;
      float mh = M1[tid] / (1.f - b1t), vh = M2[tid] / (1.f - b2t);
      float nq = Q[tid] - lr * lr_scale_q(tid) * mh / (sqrtf(vh) + eps);
      // projection onto w2 >= 0 (w1 = 1/d > 0 already): non-decreasing root
      if (tid >= H && tid < 2 * H && nq < 0.f) nq = 0.f;
      Q[tid] = nq;
    }
    __syncthreads();
    if (tid == 0) derive_params(Q, P, sd, stk);
    __syncthreads();
  }
  // The network on its piecewise-linear form: on [t_j, t_j + d_j) ramps
  // i < j are saturated and ramps i > j are 0, so the value is
  // b2 + sum_{i<j} w2_i + (w2_j / d_j) (x - t_j).  Then the output fold: an
  // affine map with a positive slope sends the bin's smallest key to 0 and
  // its largest to just below 1, so the leaves cover the keys.
  __shared__ LIRoot s_root;
  if (tid == 0) {
    float c = P[3 * H];
    for (int j = 0; j < H; j++) {
      s_root.knot[j] = stk[j];
      s_root.base[j] = c;
      s_root.slope[j] = P[2 * H + j] / sd[j];
      c += P[2 * H + j];
    }
    s_root.hmin = hmin;
    s_root.inv_range = inv;
    float y0 = li_root_eval(s_root, li_x(s_root, hmin)), y1 = li_root_eval(s_root, li_x(s_root, hmax));
    if (n && y1 > y0) {
      float a = 0.99999905f / (y1 - y0);
      for (int j = 0; j < H; j++) {
        P[2 * H + j] *= a;
        s_root.base[j] = a * (s_root.base[j] - y0);
        s_root.slope[j] *= a;
      }
      P[3 * H] = a * P[3 * H] - a * y0;
    }
  }
  __syncthreads();
  // final loss with the trained parameters
  {
    float g[LI_NPARAM];
#pragma unroll
    for (int p = 0; p < LI_NPARAM; p++) g[p] = 0.f;
    float loss = 0.f;
    for (uint32_t i = tid; i < S; i += LT_BLOCK) mlp_accumulate(P, sx[i], st[i], scale, g, loss);
    reduce_grads(g, loss, red);
    __syncthreads();
    if (tid == 0) {
      float l = 0.f;
      for (int w = 0; w < LT_NW; w++) l += red[w][LI_NPARAM];
      loss_out[b] = l;
    }
  }
  if (tid < H) {
    R.knot[tid] = s_root.knot[tid];
    R.base[tid] = s_root.base[tid];
    R.slope[tid] = s_root.slope[tid];
  }
  if (tid == 0) {
    R.hmin = hmin;
    R.inv_range = inv;
  }
}

template <class KeyT>
CF1_D uint32_t key_leaf(const LIRoot &R, const KeyT &key, int k, uint64_t &h) {
  h = KOps<KeyT>::high64(key, k);
  return li_leaf_of(R, li_root_eval(R, li_x(R, h)));
}

// Runs of equal leaves inside a warp (the lanes hold consecutive keys, and a
// monotone root sends consecutive keys to non-decreasing leaves, so a leaf is
// one run; the reductions below stay exact for any order): the lane of the
// run's first key, from the ballot of run heads.
CF1_D uint32_t run_head_lane(uint32_t leaf, unsigned lane, unsigned &heads) {
  const uint32_t prev = __shfl_up_sync(FULL, leaf, 1);
  heads = __ballot_sync(FULL, lane == 0 || leaf != prev);
  return 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
}
CF1_D bool run_tail(uint32_t leaf, unsigned lane) {
  const uint32_t next = __shfl_down_sync(FULL, leaf, 1);
  return lane == 31 || leaf != next;
}

// Per leaf: first and last local rank and key count, one atomic of each kind
// per run of a warp.
template <class KeyT>
__global__ void __launch_bounds__(LT_BLOCK) li_assign_kernel(const KeyT *keys, const uint64_t *dist_off,
                                                            const uint32_t *tile_off, uint32_t nbins,
                                                            const LIRoot *roots, int k, uint32_t *lfirst,
                                                            uint32_t *llast, uint32_t *ln) {
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(dist_off, tile_off, nbins, t, LT_TILE);
  const LIRoot &R = roots[sp.seg];
  const uint64_t base = dist_off[sp.seg];
  const unsigned lane = lane_id();
  for (uint64_t i0 = sp.start; i0 < sp.end; i0 += LT_BLOCK) {
    uint64_t i = i0 + threadIdx.x;
    bool act = i < sp.end;
    uint64_t h;
    uint32_t leaf = act ? key_leaf(R, keys[i], k, h) : 0xFFFFFFFFu;
    uint32_t rank = (uint32_t)(i - base);
    unsigned heads;
    const uint32_t hl = run_head_lane(leaf, lane, heads);
    const bool tail = run_tail(leaf, lane);
    if (act) {
      const uint64_t g = R.leaf_off + leaf;
      if (lane == hl) atomicMin(&lfirst[g], rank);
      if (tail) {
        atomicMax(&llast[g], rank);
        atomicAdd(&ln[g], lane - hl + 1);
      }
    }
  }
}

template <class KeyT>
__global__ void li_fit_kernel(const KeyT *keys, const uint64_t *dist_off, const uint64_t *leaf_off, uint32_t nbins,
                              uint64_t total_leaves, int k, const uint32_t *lfirst, const uint32_t *llast,
                              const uint32_t *ln, LILeaf *leaves) {
  uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total_leaves) return;
  LILeaf L;
  L.n = ln[g];
  if (L.n == 0) {
    L.hfirst = 0;
    L.first_rank = 0;
    L.err = 0;
    L.slope = 0.f;
    leaves[g] = L;
    return;
  }
  uint32_t b = upper_segment(leaf_off, nbins, g);
  uint64_t base = dist_off[b];
  uint32_t f = lfirst[g], l = llast[g];
  uint64_t hf = KOps<KeyT>::high64(keys[base + f], k), hl = KOps<KeyT>::high64(keys[base + l], k);
  L.hfirst = hf;
  L.first_rank = f;
  L.err = 0;
  L.slope = (l > f && hl > hf) ? __fdiv_rn((float)(l - f), u64_to_f(hl - hf)) : 0.f;
  leaves[g] = L;
}

// Per leaf: the largest |prediction - rank| over its keys (a segmented max
// over each warp's runs, one atomic per run).
template <class KeyT>
__global__ void __launch_bounds__(LT_BLOCK) li_err_kernel(const KeyT *keys, const uint64_t *dist_off,
                                                         const uint32_t *tile_off, uint32_t nbins,
                                                         const LIRoot *roots, int k, LILeaf *leaves) {
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(dist_off, tile_off, nbins, t, LT_TILE);
  const LIRoot &R = roots[sp.seg];
  const uint64_t base = dist_off[sp.seg];
  const unsigned lane = lane_id();
  for (uint64_t i0 = sp.start; i0 < sp.end; i0 += LT_BLOCK) {
    uint64_t i = i0 + threadIdx.x;
    bool act = i < sp.end;
    uint64_t h = 0;
    uint32_t leaf = act ? key_leaf(R, keys[i], k, h) : 0xFFFFFFFFu;
    uint32_t e = 0;
    if (act) {
      int64_t p = li_predict(leaves[R.leaf_off + leaf], h);
      int64_t d = p - (int64_t)(i - base);
      d = d < 0 ? -d : d;
      e = d > 0xFFFFFFF0ll ? 0xFFFFFFF0u : (uint32_t)d;
    }
    unsigned heads;
    const uint32_t hl = run_head_lane(leaf, lane, heads);
    const bool tail = run_tail(leaf, lane);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(FULL, e, d);
      if (lane >= hl + d) e = v > e ? v : e;
    }
    if (act && tail) atomicMax(&leaves[R.leaf_off + leaf].err, e);
  }
}

// One CTA per bin: the bin's largest leaf error decides learned vs BBHash.
__global__ void __launch_bounds__(LT_BLOCK) li_decide_kernel(const uint64_t *dist_off, LIRoot *roots,
                                                            const LILeaf *leaves, uint32_t max_err, uint32_t *sel,
                                                            unsigned long long *errsum) {
  __shared__ uint32_t s_max;
  __shared__ unsigned long long s_sum;
  const uint32_t b = blockIdx.x;
  LIRoot &R = roots[b];
  if (threadIdx.x == 0) {
    s_max = 0;
    s_sum = 0;
  }
  __syncthreads();
  uint32_t m = 0;
  unsigned long long sum = 0;
  for (uint32_t j = threadIdx.x; j < R.n_leaves; j += LT_BLOCK) {
    const LILeaf &L = leaves[R.leaf_off + j];
    if (L.n) {
      m = L.err > m ? L.err : m;
      sum += (unsigned long long)L.err * L.n;
    }
  }
  atomicMax(&s_max, m);
  atomicAdd(&s_sum, sum);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t n = dist_off[b + 1] - dist_off[b];
    R.max_err = s_max;
    R.use_learned = (n > 0 && s_max <= max_err) ? 1u : 0u;
    sel[b] = (n > 0 && !R.use_learned) ? 1u : 0u;
    errsum[b] = s_sum;
  }
}

// Verification, the bijection judge: every key of a learned bin must come
// back as its own rank.  A query for keys[i] is the lower bound of the key in
// its window (li_local_slot); in a bin whose keys strictly increase that is i
// exactly when the window holds i.  So the pass checks each key's window and
// the order of each adjacent pair -- together a proof that the learned index
// maps the bin's keys one to one onto [0, n) -- in one streaming read of the
// keys, with no search.
template <class KeyT>
__global__ void __launch_bounds__(LT_BLOCK) li_verify_kernel(const KeyT *keys, const uint64_t *dist_off,
                                                           const uint32_t *tile_off, uint32_t nbins, LIView v,
                                                           uint32_t *miss) {
  const uint32_t t = blockIdx.x;
  if (t >= tile_off[nbins]) return;
  TileSpan sp = tile_span(dist_off, tile_off, nbins, t, LT_TILE);
  if (!v.roots[sp.seg].use_learned) return;
  const uint64_t base = dist_off[sp.seg], n = dist_off[sp.seg + 1] - base;
  bool bad = false;
  for (uint64_t i = sp.start + threadIdx.x; i < sp.end; i += LT_BLOCK) {
    const KeyT key = keys[i];
    const int64_t r = (int64_t)(i - base);
    int64_t lo, hi;
    const bool found = li_window(v, n, sp.seg, key, lo, hi) && lo <= r && r <= hi;
    bad |= !found || (r > 0 && !(keys[i - 1] < key));
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) miss[sp.seg] = 1;
}

__global__ void li_fixup_kernel(LIRoot *roots, const uint32_t *miss, uint32_t *sel, uint32_t nbins) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins && miss[b]) {
    roots[b].use_learned = 0;
    sel[b] = 1;
  }
}

__global__ void __launch_bounds__(LT_BLOCK) li_grad_kernel(const float *params, const float *x, const float *t,
                                                          uint32_t n, float *grad, float *loss_out) {
  __shared__ float P[LI_NPARAM];
  __shared__ float red[LT_NW][LI_NPARAM + 1];
  if (threadIdx.x < LI_NPARAM) P[threadIdx.x] = params[threadIdx.x];
  __syncthreads();
  float g[LI_NPARAM];
#pragma unroll
  for (int p = 0; p < LI_NPARAM; p++) g[p] = 0.f;
  float loss = 0.f;
  const float scale = n ? 1.f / (float)n : 0.f;
  for (uint32_t i = threadIdx.x; i < n; i += LT_BLOCK) mlp_accumulate(P, x[i], t[i], scale, g, loss);
  reduce_grads(g, loss, red);
  __syncthreads();
  if (threadIdx.x <= LI_NPARAM) {
    float s = 0.f;
    for (int w = 0; w < LT_NW; w++) s += red[w][threadIdx.x];
    if (threadIdx.x < LI_NPARAM) grad[threadIdx.x] = s;
    else *loss_out = s;
  }
}

// One training step's gradient with respect to the trained parameters Q:
// the same derive_params, mlp_accumulate, reduce_grads and grad_q calls
// li_train_kernel makes before its Adam update, over n given samples.
__global__ void __launch_bounds__(LT_BLOCK) li_grad_q_kernel(const float *q, const float *x, const float *t,
                                                            uint32_t n, float *gq_out, float *loss_out) {
  __shared__ float P[LI_NPARAM], Q[LI_NQ], GQ[LI_NQ], sd[H], stk[H];
  __shared__ float red[LT_NW][LI_NPARAM + 1];
  const unsigned tid = threadIdx.x;
  if (tid < LI_NQ) Q[tid] = q[tid];
  __syncthreads();
  if (tid == 0) derive_params(Q, P, sd, stk);
  __syncthreads();
  float g[LI_NPARAM];
#pragma unroll
  for (int p = 0; p < LI_NPARAM; p++) g[p] = 0.f;
  float loss = 0.f;
  const float scale = n ? 1.f / (float)n : 0.f;
  for (uint32_t i = tid; i < n; i += LT_BLOCK) mlp_accumulate(P, x[i], t[i], scale, g, loss);
  reduce_grads(g, loss, red);
  __syncthreads();
  if (tid == 0) {
    float G[LI_NPARAM];
    for (int p = 0; p < LI_NPARAM; p++) {
      float v = 0.f;
      for (int w = 0; w < LT_NW; w++) v += red[w][p];
      G[p] = v;
    }
    grad_q(G, sd, stk, GQ);
    float l = 0.f;
    for (int w = 0; w < LT_NW; w++) l += red[w][LI_NPARAM];
    *loss_out = l;
  }
  __syncthreads();
  if (tid < LI_NQ) gq_out[tid] = GQ[tid];
}

}  // namespace

template <class KeyT>
void LearnedBuild<KeyT>::build(const KeyT *keys, const uint64_t *dist_off, uint32_t nb, int k, const LearnedOpts &o,
                               cudaStream_t s) {
  nbins = nb;
  stats = LearnedStats();
  std::vector<uint64_t> hoff(nbins + 1);
  CF1_CUDA(cudaMemcpyAsync(hoff.data(), dist_off, (nbins + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  std::vector<LIRoot> hroots(nbins);
  std::vector<uint64_t> hleaf(nbins + 1);
  uint64_t total_leaves = 0;
  uint32_t leaf_size = o.leaf_size ? o.leaf_size : 32;
  for (uint32_t b = 0; b < nbins; b++) {
    uint64_t n = hoff[b + 1] - hoff[b];
    uint64_t nl = n ? (n + leaf_size - 1) / leaf_size : 1;
    std::memset(&hroots[b], 0, sizeof(LIRoot));
    for (int p = 0; p < H; p++) {  // identity root until training writes its own
      hroots[b].knot[p] = (float)p / (float)H;
      hroots[b].base[p] = (float)p / (float)H;
      hroots[b].slope[p] = 1.f;
    }
    hroots[b].n_leaves = (uint32_t)nl;
    hroots[b].leaf_off = total_leaves;
    hroots[b].use_learned = n > 0;
    hleaf[b] = total_leaves;
    total_leaves += nl;
  }
  hleaf[nbins] = total_leaves;
  uint64_t n_total = hoff[nbins];
  LIRoot *roots = roots_.get<LIRoot>(nbins);
  uint64_t *leaf_off = leaf_off_.get<uint64_t>(nbins + 1);
  CF1_CUDA(cudaMemcpyAsync(roots, hroots.data(), nbins * sizeof(LIRoot), cudaMemcpyHostToDevice, s));
  CF1_CUDA(cudaMemcpyAsync(leaf_off, hleaf.data(), (nbins + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  float *loss = loss_.get<float>(nbins);
  CF1_CUDA(cudaMemsetAsync(loss, 0, nbins * sizeof(float), s));
  uint32_t samples = o.max_samples > LT_MAX_SAMPLES ? LT_MAX_SAMPLES : (o.max_samples ? o.max_samples : 1);
  if (nbins) {
    li_train_kernel<KeyT><<<nbins, LT_BLOCK, 0, s>>>(keys, dist_off, roots, k, o.train_steps < 0 ? 0 : o.train_steps,
                                                     o.lr, samples, loss);
    CF1_LAUNCH_CHECK();
  }
  uint32_t *lfirst = lfirst_.get<uint32_t>(total_leaves);
  uint32_t *llast = llast_.get<uint32_t>(total_leaves);
  uint32_t *ln = ln_.get<uint32_t>(total_leaves);
  LILeaf *leaves = leaves_.get<LILeaf>(total_leaves);
  CF1_CUDA(cudaMemsetAsync(lfirst, 0xFF, total_leaves * 4, s));
  CF1_CUDA(cudaMemsetAsync(llast, 0, total_leaves * 4, s));
  CF1_CUDA(cudaMemsetAsync(ln, 0, total_leaves * 4, s));
  uint32_t *tile_off = tile_off_.get<uint32_t>(nbins + 1);
  segment_tiles(dist_off, nbins, LT_TILE, tile_off, s);
  uint32_t ub = (uint32_t)(ceil_div(n_total, LT_TILE) + nbins);
  li_assign_kernel<KeyT><<<ub, LT_BLOCK, 0, s>>>(keys, dist_off, tile_off, nbins, roots, k, lfirst, llast, ln);
  CF1_LAUNCH_CHECK();
  li_fit_kernel<KeyT><<<(unsigned)ceil_div(total_leaves, 256), 256, 0, s>>>(keys, dist_off, leaf_off, nbins, total_leaves,
                                                                            k, lfirst, llast, ln, leaves);
  CF1_LAUNCH_CHECK();
  li_err_kernel<KeyT><<<ub, LT_BLOCK, 0, s>>>(keys, dist_off, tile_off, nbins, roots, k, leaves);
  CF1_LAUNCH_CHECK();
  uint32_t *sel = sel_.get<uint32_t>(nbins);
  unsigned long long *errsum = errsum_.get<unsigned long long>(nbins);
  li_decide_kernel<<<nbins, LT_BLOCK, 0, s>>>(dist_off, roots, leaves, o.max_err, sel, errsum);
  CF1_LAUNCH_CHECK();
  uint32_t *miss = lfirst;  // reuse: one flag per bin
  CF1_CUDA(cudaMemsetAsync(miss, 0, nbins * 4, s));
  li_verify_kernel<KeyT><<<ub, LT_BLOCK, 0, s>>>(keys, dist_off, tile_off, nbins, view(k), miss);
  CF1_LAUNCH_CHECK();
  li_fixup_kernel<<<(unsigned)ceil_div(nbins, 256), 256, 0, s>>>(roots, miss, sel, nbins);
  CF1_LAUNCH_CHECK();
  // stats
  std::vector<LIRoot> r2(nbins);
  std::vector<unsigned long long> es(nbins);
  std::vector<float> hl(nbins);
  std::vector<uint32_t> hmiss(nbins);
  CF1_CUDA(cudaMemcpyAsync(hmiss.data(), miss, nbins * 4, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaMemcpyAsync(r2.data(), roots, nbins * sizeof(LIRoot), cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaMemcpyAsync(es.data(), errsum, nbins * 8, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaMemcpyAsync(hl.data(), loss, nbins * 4, cudaMemcpyDeviceToHost, s));
  CF1_CUDA(cudaStreamSynchronize(s));
  double esum = 0, wsum = 0, keys_learned = 0, lsum = 0;
  uint64_t nonempty = 0;
  for (uint32_t b = 0; b < nbins; b++) {
    uint64_t n = hoff[b + 1] - hoff[b];
    if (!n) continue;
    nonempty++;
    lsum += hl[b];
    stats.max_err_all = r2[b].max_err > stats.max_err_all ? r2[b].max_err : stats.max_err_all;
    stats.verify_miss_bins += hmiss[b] ? 1 : 0;
    if (r2[b].use_learned) {
      stats.learned_bins++;
      stats.max_err = r2[b].max_err > stats.max_err ? r2[b].max_err : stats.max_err;
      esum += (double)es[b];
      wsum += 2.0 * (double)es[b] + (double)n;
      keys_learned += (double)n;
    } else {
      stats.fallback_bins++;
    }
  }
  stats.leaves = total_leaves;
  stats.mean_err = keys_learned ? esum / keys_learned : 0;
  stats.mean_window = keys_learned ? wsum / keys_learned : 0;
  stats.train_loss = nonempty ? lsum / nonempty : 0;
  stats.bytes = nbins * sizeof(LIRoot) + total_leaves * sizeof(LILeaf);
}

template <class KeyT>
LIView LearnedBuild<KeyT>::view(int k) const {
  LIView v;
  v.roots = roots_.as<const LIRoot>();
  v.leaves = leaves_.as<const LILeaf>();
  v.k = k;
  return v;
}

template struct LearnedBuild<uint64_t>;
template struct LearnedBuild<Key2>;

void learned_grad_host(const float *params, const float *x, const float *t, size_t n, float *grad, float *loss) {
  DevBuf dp, dx, dt, dg;
  float *p = dp.get<float>(LI_NPARAM + 1);
  float *xx = dx.get<float>(n + 1);
  float *tt = dt.get<float>(n + 1);
  float *g = dg.get<float>(LI_NPARAM + 1);
  CF1_CUDA(cudaMemcpy(p, params, LI_NPARAM * 4, cudaMemcpyHostToDevice));
  if (n) {
    CF1_CUDA(cudaMemcpy(xx, x, n * 4, cudaMemcpyHostToDevice));
    CF1_CUDA(cudaMemcpy(tt, t, n * 4, cudaMemcpyHostToDevice));
  }
  li_grad_kernel<<<1, LT_BLOCK>>>(p, xx, tt, (uint32_t)n, g, g + LI_NPARAM);
  CF1_LAUNCH_CHECK();
  float out[LI_NPARAM + 1];
  CF1_CUDA(cudaMemcpy(out, g, (LI_NPARAM + 1) * 4, cudaMemcpyDeviceToHost));
  std::memcpy(grad, out, LI_NPARAM * 4);
  *loss = out[LI_NPARAM];
}

void learned_grad_q_host(const float *q, const float *x, const float *t, size_t n, float *grad_q, float *loss) {
  DevBuf dq, dx, dt, dg;
  float *qq = dq.get<float>(LI_NQ + 1);
  float *xx = dx.get<float>(n + 1);
  float *tt = dt.get<float>(n + 1);
  float *g = dg.get<float>(LI_NQ + 1);
  CF1_CUDA(cudaMemcpy(qq, q, LI_NQ * 4, cudaMemcpyHostToDevice));
  if (n) {
    CF1_CUDA(cudaMemcpy(xx, x, n * 4, cudaMemcpyHostToDevice));
    CF1_CUDA(cudaMemcpy(tt, t, n * 4, cudaMemcpyHostToDevice));
  }
  li_grad_q_kernel<<<1, LT_BLOCK>>>(qq, xx, tt, (uint32_t)n, g, g + LI_NQ);
  CF1_LAUNCH_CHECK();
  float out[LI_NQ + 1];
  CF1_CUDA(cudaMemcpy(out, g, (LI_NQ + 1) * 4, cudaMemcpyDeviceToHost));
  std::memcpy(grad_q, out, LI_NQ * 4);
  *loss = out[LI_NQ];
}

}  // namespace cf1
