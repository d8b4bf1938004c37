// mlp.cu — training of the surrogate's MLP ensemble with hand-written
// forward/backward kernels.
//
// Models: one per (centre species z, member m), nin → H → H → 1 with SiLU,
// FP32 master parameters [W1 H×nin | b1 H | W2 H×H | b2 H | w3 H | b3].
// Loss: mean squared error of the standardised site energy over the samples
// of the model's species.  The reference trains its feature head on the CPU
// through Lux/Zygote (ACE/feature_energy.jl, ext/PotentialFrameWorkLuxCoreExt.jl);
// there is no GPU counterpart.
//
//   k_mlp_grad   one block per (tile of 32 samples, model): weights and the
//                tile in shared memory, forward pass, backward pass, the
//                tile's parameter gradient written as one partial row
//   k_mlp_adam   sums the partial rows of every tile in tile order
//                (deterministic) and applies Adam with bias correction
#include <algorithm>
#include <cmath>
#include <vector>

#include "pfw_internal.h"

namespace pfw {

constexpr int MLP_TILE = 32;
constexpr int MLP_THREADS = 256;
constexpr int MLP_MAXW = 64;  // training supports nin, H <= 64

struct MlpDims {
  int nin, H, np;             // inputs, hidden width, parameters per model
  int oW1, ob1, oW2, ob2, ow3, ob3;
  __host__ __device__ void make(int nin_, int H_) {
    nin = nin_;
    H = H_;
    oW1 = 0;
    ob1 = H * nin;
    oW2 = ob1 + H;
    ob2 = oW2 + H * H;
    ow3 = ob2 + H;
    ob3 = ow3 + H;
    np = ob3 + 1;
  }
};

static size_t mlp_smem_floats(const MlpDims& d) {
  const int ni = d.nin + 1, h = d.H + 1;
  return (size_t)d.H * ni + (size_t)d.H * h + 3 * d.H + 1 + MLP_TILE * ni + 6 * MLP_TILE * h + 3 * MLP_TILE;
}

__device__ __forceinline__ void silu_d(float z, float& h, float& ds) {
  const float sg = 1.f / (1.f + expf(-z));
  h = z * sg;
  ds = sg * (1.f + z * (1.f - sg));
}

// order[model * stride + k], k < count[model]: the samples of this step.
__global__ void __launch_bounds__(MLP_THREADS)
    k_mlp_grad(MlpDims dm, const float* __restrict__ params, const float* __restrict__ X, const float* __restrict__ y,
               const int* __restrict__ order, int stride, const int* __restrict__ count, float* __restrict__ partial,
               double* __restrict__ loss_part) {
  extern __shared__ float sm[];
  const int tile = blockIdx.x, model = blockIdx.y, ntiles = gridDim.x;
  const int nin = dm.nin, H = dm.H, ni = nin + 1, h = H + 1;
  float* W1 = sm;
  float* W2 = W1 + H * ni;
  float* b1 = W2 + H * h;
  float* b2 = b1 + H;
  float* w3 = b2 + H;
  float* b3 = w3 + H;
  float* Xs = b3 + 1;
  float* H1 = Xs + MLP_TILE * ni;
  float* S1 = H1 + MLP_TILE * h;
  float* H2 = S1 + MLP_TILE * h;
  float* S2 = H2 + MLP_TILE * h;
  float* D2 = S2 + MLP_TILE * h;
  float* D1 = D2 + MLP_TILE * h;
  float* yp = D1 + MLP_TILE * h;
  float* dy = yp + MLP_TILE;
  float* er = dy + MLP_TILE;
  const float* P = params + (size_t)model * dm.np;
  const int tid = threadIdx.x;
  for (int k = tid; k < H * nin; k += MLP_THREADS) W1[(k / nin) * ni + k % nin] = P[dm.oW1 + k];
  for (int k = tid; k < H * H; k += MLP_THREADS) W2[(k / H) * h + k % H] = P[dm.oW2 + k];
  for (int k = tid; k < H; k += MLP_THREADS) {
    b1[k] = P[dm.ob1 + k];
    b2[k] = P[dm.ob2 + k];
    w3[k] = P[dm.ow3 + k];
  }
  if (tid == 0) b3[0] = P[dm.ob3];
  const int cnt = count[model];
  const int s0 = tile * MLP_TILE;
  const int* ord = order + (size_t)model * stride;
  for (int k = tid; k < MLP_TILE * nin; k += MLP_THREADS) {
    const int s = k / nin, i = k - s * nin;
    Xs[s * ni + i] = (s0 + s < cnt) ? X[(size_t)ord[s0 + s] * nin + i] : 0.f;
  }
  __syncthreads();
  // forward
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    float z = b1[o];
    for (int i = 0; i < nin; ++i) z = fmaf(W1[o * ni + i], Xs[s * ni + i], z);
    silu_d(z, H1[s * h + o], S1[s * h + o]);
  }
  __syncthreads();
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    float z = b2[o];
    for (int i = 0; i < H; ++i) z = fmaf(W2[o * h + i], H1[s * h + i], z);
    silu_d(z, H2[s * h + o], S2[s * h + o]);
  }
  __syncthreads();
  if (tid < MLP_TILE) {
    const int s = tid;
    float v = b3[0];
    for (int o = 0; o < H; ++o) v = fmaf(w3[o], H2[s * h + o], v);
    yp[s] = v;
    const bool live = s0 + s < cnt;
    const float e = live ? v - y[ord[s0 + s]] : 0.f;
    dy[s] = live ? 2.f * e / (float)cnt : 0.f;
    er[s] = e * e;
  }
  __syncthreads();
  // backward
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    D2[s * h + o] = dy[s] * w3[o] * S2[s * h + o];
  }
  __syncthreads();
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, i = k - s * H;
    float acc = 0.f;
    for (int o = 0; o < H; ++o) acc = fmaf(D2[s * h + o], W2[o * h + i], acc);
    D1[s * h + i] = acc * S1[s * h + i];
  }
  __syncthreads();
  float* out = partial + ((size_t)model * ntiles + tile) * dm.np;
  for (int k = tid; k < H * nin; k += MLP_THREADS) {
    const int o = k / nin, i = k - o * nin;
    float acc = 0.f;
    for (int s = 0; s < MLP_TILE; ++s) acc = fmaf(D1[s * h + o], Xs[s * ni + i], acc);
    out[dm.oW1 + k] = acc;
  }
  for (int k = tid; k < H * H; k += MLP_THREADS) {
    const int o = k / H, i = k - o * H;
    float acc = 0.f;
    for (int s = 0; s < MLP_TILE; ++s) acc = fmaf(D2[s * h + o], H1[s * h + i], acc);
    out[dm.oW2 + k] = acc;
  }
  for (int o = tid; o < H; o += MLP_THREADS) {
    float g1 = 0.f, g2 = 0.f, g3 = 0.f;
    for (int s = 0; s < MLP_TILE; ++s) {
      g1 += D1[s * h + o];
      g2 += D2[s * h + o];
      g3 = fmaf(dy[s], H2[s * h + o], g3);
    }
    out[dm.ob1 + o] = g1;
    out[dm.ob2 + o] = g2;
    out[dm.ow3 + o] = g3;
  }
  if (tid == 0) {
    float g = 0.f;
    double l = 0.0;
    for (int s = 0; s < MLP_TILE; ++s) {
      g += dy[s];
      l += er[s];
    }
    out[dm.ob3] = g;
    loss_part[(size_t)model * ntiles + tile] = l;
  }
}

// Sum of the tile partials (tile order) → gradient; Adam step when lr > 0,
// else the gradient is written to grad_out.
__global__ void k_mlp_adam(MlpDims dm, int ntiles, const float* __restrict__ partial,
                           const double* __restrict__ loss_part, float* __restrict__ params, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float bc1, float bc2, float* __restrict__ grad_out,
                           double* __restrict__ loss_acc) {
  const int model = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < dm.np) {
    float g = 0.f;
    for (int t = 0; t < ntiles; ++t) g += partial[((size_t)model * ntiles + t) * dm.np + j];
    const size_t k = (size_t)model * dm.np + j;
    if (grad_out) {
      grad_out[k] = g;
    } else {
      const float a = 0.9f * m1[k] + 0.1f * g;
      const float b = 0.999f * m2[k] + 0.001f * g * g;
      m1[k] = a;
      m2[k] = b;
      params[k] -= lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double l = 0.0;
    for (int t = 0; t < ntiles; ++t) l += loss_part[(size_t)model * ntiles + t];
    loss_acc[model] += l;
  }
}

// ---------------------------------------------------------------------------
// Energy + force training.  For a site with standardised features x, the
// model output y(x) is the standardised site energy, and the site's
// contribution to the forces is -(dE/dx)·(dx/dr).  With the force error ΔF
// pulled back into feature space as a tangent v = D_ΔF x (the change of the
// site's features along ΔF, standardised), the force loss Σ|ΔF|² has the
// parameter gradient Σ_sites c·∂/∂θ (v·∇_x y) (c carries -2 and the loss
// and unit scales).  v·∇_x y is a forward-mode (tangent) pass through the
// network:  t1 = W1 v, u1 = s1'⊙t1, t2 = W2 u1, u2 = s2'⊙t2, ẏ = w3·u2,
// and its reverse runs through the tangent and through the SiLU slopes
// (s'' = σ(1-σ)(2 + z(1-2σ))).  k_mlp_ef_grad adds it to the energy loss
// gradient of the same tile, one partial row per (tile, model) as k_mlp_grad.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void silu_dd(float z, float& h, float& ds, float& dds) {
  const float sg = 1.f / (1.f + expf(-z));
  h = z * sg;
  ds = sg * (1.f + z * (1.f - sg));
  dds = sg * (1.f - sg) * (2.f + z * (1.f - 2.f * sg));
}

static size_t mlp_ef_smem_floats(const MlpDims& d) {
  const int ni = d.nin + 1, h = d.H + 1;
  return (size_t)d.H * ni + (size_t)d.H * h + 3 * d.H + 1 + 2 * MLP_TILE * ni + 13 * MLP_TILE * h + 3 * MLP_TILE;
}

// V: [members][n][nin] standardised tangents (or null: energy loss only);
// c: [n] force weight per sample; wE: energy loss weight.
__global__ void __launch_bounds__(MLP_THREADS)
    k_mlp_ef_grad(MlpDims dm, int members, int n, const float* __restrict__ params, const float* __restrict__ X,
                  const float* __restrict__ y, const float* __restrict__ V, const float* __restrict__ c, float wE,
                  const int* __restrict__ order, int stride, const int* __restrict__ count,
                  float* __restrict__ partial, double* __restrict__ loss_part) {
  extern __shared__ float sm[];
  const int tile = blockIdx.x, model = blockIdx.y, ntiles = gridDim.x;
  const int member = model % members;
  const int nin = dm.nin, H = dm.H, ni = nin + 1, h = H + 1;
  float* W1 = sm;
  float* W2 = W1 + H * ni;
  float* b1 = W2 + H * h;
  float* b2 = b1 + H;
  float* w3 = b2 + H;
  float* b3 = w3 + H;
  float* Xs = b3 + 1;
  float* Vs = Xs + MLP_TILE * ni;
  float* H1 = Vs + MLP_TILE * ni;
  float* S1 = H1 + MLP_TILE * h;
  float* Q1 = S1 + MLP_TILE * h;
  float* T1 = Q1 + MLP_TILE * h;
  float* H2 = T1 + MLP_TILE * h;
  float* S2 = H2 + MLP_TILE * h;
  float* Q2 = S2 + MLP_TILE * h;
  float* T2 = Q2 + MLP_TILE * h;
  float* G2 = T2 + MLP_TILE * h;
  float* B2 = G2 + MLP_TILE * h;  // ∂/∂t2 of the force term
  float* G1 = B2 + MLP_TILE * h;
  float* B1 = G1 + MLP_TILE * h;  // ∂/∂t1 of the force term
  float* BU = B1 + MLP_TILE * h;  // ∂/∂u1 of the force term
  float* dy = BU + MLP_TILE * h;
  float* cw = dy + MLP_TILE;
  float* er = cw + MLP_TILE;
  const float* P = params + (size_t)model * dm.np;
  const int tid = threadIdx.x;
  for (int k = tid; k < H * nin; k += MLP_THREADS) W1[(k / nin) * ni + k % nin] = P[dm.oW1 + k];
  for (int k = tid; k < H * H; k += MLP_THREADS) W2[(k / H) * h + k % H] = P[dm.oW2 + k];
  for (int k = tid; k < H; k += MLP_THREADS) {
    b1[k] = P[dm.ob1 + k];
    b2[k] = P[dm.ob2 + k];
    w3[k] = P[dm.ow3 + k];
  }
  if (tid == 0) b3[0] = P[dm.ob3];
  const int cnt = count[model];
  const int s0 = tile * MLP_TILE;
  const int* ord = order + (size_t)model * stride;
  const float* Vm = V ? V + (size_t)member * n * nin : nullptr;
  for (int k = tid; k < MLP_TILE * nin; k += MLP_THREADS) {
    const int s = k / nin, i = k - s * nin;
    const bool live = s0 + s < cnt;
    Xs[s * ni + i] = live ? X[(size_t)ord[s0 + s] * nin + i] : 0.f;
    Vs[s * ni + i] = (live && Vm) ? Vm[(size_t)ord[s0 + s] * nin + i] : 0.f;
  }
  if (tid < MLP_TILE) cw[tid] = (s0 + tid < cnt && c) ? c[ord[s0 + tid]] : 0.f;
  __syncthreads();
  // forward and tangent, layer 1
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    float z = b1[o], t = 0.f;
    for (int i = 0; i < nin; ++i) {
      z = fmaf(W1[o * ni + i], Xs[s * ni + i], z);
      t = fmaf(W1[o * ni + i], Vs[s * ni + i], t);
    }
    silu_dd(z, H1[s * h + o], S1[s * h + o], Q1[s * h + o]);
    T1[s * h + o] = t;
  }
  __syncthreads();
  // layer 2 (tangent input u1 = s1'·t1)
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    float z = b2[o], t = 0.f;
    for (int i = 0; i < H; ++i) {
      z = fmaf(W2[o * h + i], H1[s * h + i], z);
      t = fmaf(W2[o * h + i], S1[s * h + i] * T1[s * h + i], t);
    }
    silu_dd(z, H2[s * h + o], S2[s * h + o], Q2[s * h + o]);
    T2[s * h + o] = t;
  }
  __syncthreads();
  if (tid < MLP_TILE) {
    const int s = tid;
    float v = b3[0];
    for (int o = 0; o < H; ++o) v = fmaf(w3[o], H2[s * h + o], v);
    const bool live = s0 + s < cnt;
    const float e = live ? v - y[ord[s0 + s]] : 0.f;
    dy[s] = live ? 2.f * wE * e / (float)cnt : 0.f;
    er[s] = e * e;
  }
  __syncthreads();
  // reverse: G2 = ∂/∂z2 (energy through h2, force through s2'), B2 = ∂/∂t2
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    const float a = w3[o];
    G2[s * h + o] = dy[s] * a * S2[s * h + o] + cw[s] * a * T2[s * h + o] * Q2[s * h + o];
    B2[s * h + o] = cw[s] * a * S2[s * h + o];
  }
  __syncthreads();
  // G1 = ∂/∂z1 = (W2ᵀ G2)⊙s1' + (W2ᵀ B2)⊙t1⊙s1'';  B1 = ∂/∂t1 = (W2ᵀ B2)⊙s1'
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, i = k - s * H;
    float bh = 0.f, bu = 0.f;
    for (int o = 0; o < H; ++o) {
      bh = fmaf(G2[s * h + o], W2[o * h + i], bh);
      bu = fmaf(B2[s * h + o], W2[o * h + i], bu);
    }
    G1[s * h + i] = bh * S1[s * h + i] + bu * T1[s * h + i] * Q1[s * h + i];
    B1[s * h + i] = bu * S1[s * h + i];
    BU[s * h + i] = bu;
  }
  __syncthreads();
  float* out = partial + ((size_t)model * ntiles + tile) * dm.np;
  for (int k = tid; k < H * nin; k += MLP_THREADS) {
    const int o = k / nin, i = k - o * nin;
    float acc = 0.f;
    for (int s = 0; s < MLP_TILE; ++s)
      acc = fmaf(G1[s * h + o], Xs[s * ni + i], fmaf(B1[s * h + o], Vs[s * ni + i], acc));
    out[dm.oW1 + k] = acc;
  }
  for (int k = tid; k < H * H; k += MLP_THREADS) {
    const int o = k / H, i = k - o * H;
    float acc = 0.f;
    for (int s = 0; s < MLP_TILE; ++s)
      acc = fmaf(G2[s * h + o], H1[s * h + i], fmaf(B2[s * h + o], S1[s * h + i] * T1[s * h + i], acc));
    out[dm.oW2 + k] = acc;
  }
  for (int o = tid; o < H; o += MLP_THREADS) {
    float g1 = 0.f, g2 = 0.f, g3 = 0.f;
    for (int s = 0; s < MLP_TILE; ++s) {
      g1 += G1[s * h + o];
      g2 += G2[s * h + o];
      g3 = fmaf(dy[s], H2[s * h + o], fmaf(cw[s], S2[s * h + o] * T2[s * h + o], g3));
    }
    out[dm.ob1 + o] = g1;
    out[dm.ob2 + o] = g2;
    out[dm.ow3 + o] = g3;
  }
  if (tid == 0) {
    float g = 0.f;
    double l = 0.0;
    for (int s = 0; s < MLP_TILE; ++s) {
      g += dy[s];
      l += er[s];
    }
    out[dm.ob3] = g;
    loss_part[(size_t)model * ntiles + tile] = l;
  }
}

// ∂y/∂x of every member at every sample: G [members][n][nin].
__global__ void __launch_bounds__(MLP_THREADS)
    k_mlp_input_grad(MlpDims dm, int members, int n, const float* __restrict__ params, const float* __restrict__ X,
                     const int* __restrict__ order, int stride, const int* __restrict__ count, float* __restrict__ G) {
  extern __shared__ float sm[];
  const int tile = blockIdx.x, model = blockIdx.y;
  const int member = model % members;
  const int nin = dm.nin, H = dm.H, ni = nin + 1, h = H + 1;
  float* W1 = sm;
  float* W2 = W1 + H * ni;
  float* b1 = W2 + H * h;
  float* b2 = b1 + H;
  float* w3 = b2 + H;
  float* Xs = w3 + H;
  float* H1 = Xs + MLP_TILE * ni;
  float* S1 = H1 + MLP_TILE * h;
  float* S2 = S1 + MLP_TILE * h;
  float* D2 = S2 + MLP_TILE * h;
  float* D1 = D2 + MLP_TILE * h;
  const float* P = params + (size_t)model * dm.np;
  const int tid = threadIdx.x;
  for (int k = tid; k < H * nin; k += MLP_THREADS) W1[(k / nin) * ni + k % nin] = P[dm.oW1 + k];
  for (int k = tid; k < H * H; k += MLP_THREADS) W2[(k / H) * h + k % H] = P[dm.oW2 + k];
  for (int k = tid; k < H; k += MLP_THREADS) {
    b1[k] = P[dm.ob1 + k];
    b2[k] = P[dm.ob2 + k];
    w3[k] = P[dm.ow3 + k];
  }
  const int cnt = count[model];
  const int s0 = tile * MLP_TILE;
  const int* ord = order + (size_t)model * stride;
  for (int k = tid; k < MLP_TILE * nin; k += MLP_THREADS) {
    const int s = k / nin, i = k - s * nin;
    Xs[s * ni + i] = (s0 + s < cnt) ? X[(size_t)ord[s0 + s] * nin + i] : 0.f;
  }
  __syncthreads();
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    float z = b1[o];
    for (int i = 0; i < nin; ++i) z = fmaf(W1[o * ni + i], Xs[s * ni + i], z);
    silu_d(z, H1[s * h + o], S1[s * h + o]);
  }
  __syncthreads();
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, o = k - s * H;
    float z = b2[o];
    for (int i = 0; i < H; ++i) z = fmaf(W2[o * h + i], H1[s * h + i], z);
    float hh;
    silu_d(z, hh, S2[s * h + o]);
    D2[s * h + o] = w3[o] * S2[s * h + o];
  }
  __syncthreads();
  for (int k = tid; k < MLP_TILE * H; k += MLP_THREADS) {
    const int s = k / H, i = k - s * H;
    float acc = 0.f;
    for (int o = 0; o < H; ++o) acc = fmaf(D2[s * h + o], W2[o * h + i], acc);
    D1[s * h + i] = acc * S1[s * h + i];
  }
  __syncthreads();
  for (int k = tid; k < MLP_TILE * nin; k += MLP_THREADS) {
    const int s = k / nin, i = k - s * nin;
    if (s0 + s >= cnt) continue;
    float acc = 0.f;
    for (int o = 0; o < H; ++o) acc = fmaf(D1[s * h + o], W1[o * ni + i], acc);
    G[((size_t)member * n + ord[s0 + s]) * nin + i] = acc;
  }
}

namespace {

struct MlpBuffers {
  DevBuf X, y, params, m1, m2, order, count, partial, loss_part, loss_acc, grad;
  ~MlpBuffers() {
    DevBuf* b[] = {&X, &y, &params, &m1, &m2, &order, &count, &partial, &loss_part, &loss_acc, &grad};
    for (auto* x : b) x->release();
  }
};

void check_shape(const pfw_mlp_shape* s) {
  if (!s) throw Error(PFW_EINVAL, "MLP shape required");
  if (s->nz < 1 || s->members < 1 || s->members > 4) throw Error(PFW_EINVAL, "1..4 members per species");
  if (s->nin < 1 || s->nin > MLP_MAXW || s->hidden < 1 || s->hidden > MLP_MAXW)
    throw Error(PFW_EINVAL, "training supports nin and hidden up to 64");
}

// species-grouped sample lists
std::vector<std::vector<int>> by_species(int64_t n, const int32_t* species, int nz) {
  std::vector<std::vector<int>> lists(nz);
  for (int64_t i = 0; i < n; ++i) {
    if (species[i] < 0 || species[i] >= nz) throw Error(PFW_EINVAL, "species channel outside the MLP shape");
    lists[species[i]].push_back((int)i);
  }
  return lists;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void launch_grad(pfw_ws* ws, const MlpDims& dm, int nmodels, int ntiles, MlpBuffers& b, int stride) {
  const size_t smem = sizeof(float) * mlp_smem_floats(dm);
  PFW_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mlp_grad<<<dim3(ntiles, nmodels), MLP_THREADS, smem, ws->stream>>>(
      dm, b.params.as<float>(), b.X.as<float>(), b.y.as<float>(), b.order.as<int>(), stride, b.count.as<int>(),
      b.partial.as<float>(), b.loss_part.as<double>());
  ws->launches += 1;
}

}  // namespace

void mlp_param_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params, int64_t n, const float* X,
                    const float* y, const int32_t* species, double* loss, float* grad) {
  check_shape(shape);
  if (n < 1 || !params || !X || !y || !species || !grad) throw Error(PFW_EINVAL, "samples and outputs required");
  MlpDims dm;
  dm.make(shape->nin, shape->hidden);
  const int nmodels = shape->nz * shape->members;
  cudaStream_t st = ws->stream;
  auto lists = by_species(n, species, shape->nz);
  size_t stride = 1;
  for (auto& l : lists) stride = std::max(stride, l.size());
  std::vector<int> order((size_t)nmodels * stride, 0), count(nmodels);
  for (int z = 0; z < shape->nz; ++z)
    for (int m = 0; m < shape->members; ++m) {
      const int md = z * shape->members + m;
      count[md] = (int)lists[z].size();
      std::copy(lists[z].begin(), lists[z].end(), order.begin() + (size_t)md * stride);
    }
  const int ntiles = (int)((stride + MLP_TILE - 1) / MLP_TILE);
  MlpBuffers b;
  PFW_CUDA(cudaMemcpyAsync(b.X.ensure(sizeof(float) * n * dm.nin), X, sizeof(float) * n * dm.nin,
                           cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(b.y.ensure(sizeof(float) * n), y, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(b.params.ensure(sizeof(float) * nmodels * dm.np), params,
                           sizeof(float) * nmodels * dm.np, cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(b.order.ensure(sizeof(int) * order.size()), order.data(), sizeof(int) * order.size(),
                           cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(b.count.ensure(sizeof(int) * nmodels), count.data(), sizeof(int) * nmodels,
                           cudaMemcpyHostToDevice, st));
  b.partial.ensure(sizeof(float) * (size_t)nmodels * ntiles * dm.np);
  b.loss_part.ensure(sizeof(double) * (size_t)nmodels * ntiles);
  double* lacc = static_cast<double*>(b.loss_acc.ensure(sizeof(double) * nmodels));
  PFW_CUDA(cudaMemsetAsync(lacc, 0, sizeof(double) * nmodels, st));
  float* g = static_cast<float*>(b.grad.ensure(sizeof(float) * nmodels * dm.np));
  launch_grad(ws, dm, nmodels, ntiles, b, (int)stride);
  k_mlp_adam<<<dim3((dm.np + 255) / 256, nmodels), 256, 0, st>>>(dm, ntiles, b.partial.as<float>(),
                                                                 b.loss_part.as<double>(), nullptr, nullptr, nullptr,
                                                                 0.f, 1.f, 1.f, g, lacc);
  ws->launches += 1;
  std::vector<double> hl(nmodels);
  PFW_CUDA(cudaMemcpyAsync(grad, g, sizeof(float) * nmodels * dm.np, cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaMemcpyAsync(hl.data(), lacc, sizeof(double) * nmodels, cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
  if (loss)
    for (int md = 0; md < nmodels; ++md) loss[md] = count[md] ? hl[md] / count[md] : 0.0;
}

void mlp_train(pfw_ws* ws, const pfw_mlp_shape* shape, float* params, int64_t n, const float* X, const float* y,
               const int32_t* species, const pfw_mlp_train_options* opt, float* epoch_loss) {
  check_shape(shape);
  if (n < 1 || !params || !X || !y || !species || !opt) throw Error(PFW_EINVAL, "samples and options required");
  if (opt->epochs < 1 || opt->batch < MLP_TILE || opt->batch % MLP_TILE || !(opt->lr > 0.f) || opt->lr_final < 0.f)
    throw Error(PFW_EINVAL, "epochs >= 1, batch a positive multiple of 32, lr > 0");
  MlpDims dm;
  dm.make(shape->nin, shape->hidden);
  const int nmodels = shape->nz * shape->members, batch = opt->batch, ntiles = batch / MLP_TILE;
  cudaStream_t st = ws->stream;
  auto lists = by_species(n, species, shape->nz);
  size_t nmax = 1;
  for (auto& l : lists) nmax = std::max(nmax, l.size());
  const int steps = (int)((nmax + batch - 1) / batch);
  MlpBuffers b;
  PFW_CUDA(cudaMemcpyAsync(b.X.ensure(sizeof(float) * n * dm.nin), X, sizeof(float) * n * dm.nin,
                           cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(b.y.ensure(sizeof(float) * n), y, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  float* P = static_cast<float*>(b.params.ensure(sizeof(float) * nmodels * dm.np));
  PFW_CUDA(cudaMemcpyAsync(P, params, sizeof(float) * nmodels * dm.np, cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemsetAsync(b.m1.ensure(sizeof(float) * nmodels * dm.np), 0, sizeof(float) * nmodels * dm.np, st));
  PFW_CUDA(cudaMemsetAsync(b.m2.ensure(sizeof(float) * nmodels * dm.np), 0, sizeof(float) * nmodels * dm.np, st));
  b.partial.ensure(sizeof(float) * (size_t)nmodels * ntiles * dm.np);
  b.loss_part.ensure(sizeof(double) * (size_t)nmodels * ntiles);
  double* lacc = static_cast<double*>(b.loss_acc.ensure(sizeof(double) * nmodels));
  const size_t stride = (size_t)steps * batch;
  int* dorder = static_cast<int*>(b.order.ensure(sizeof(int) * nmodels * stride));
  int* dcount = static_cast<int*>(b.count.ensure(sizeof(int) * nmodels));
  std::vector<int> order((size_t)nmodels * stride), count(nmodels);
  std::vector<double> hl(nmodels);
  uint64_t rng = opt->seed;
  long t = 0;
  const long total = (long)opt->epochs * steps;
  for (int ep = 0; ep < opt->epochs; ++ep) {
    // a fresh order of every model's samples (wrapping to fill the steps)
    for (int z = 0; z < shape->nz; ++z)
      for (int m = 0; m < shape->members; ++m) {
        const int md = z * shape->members + m;
        std::vector<int> perm = lists[z];
        for (size_t i = perm.size(); i > 1; --i) std::swap(perm[i - 1], perm[splitmix(rng) % i]);
        int* o = order.data() + (size_t)md * stride;
        for (size_t k = 0; k < stride; ++k) o[k] = perm.empty() ? 0 : perm[k % perm.size()];
      }
    PFW_CUDA(cudaMemcpyAsync(dorder, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, st));
    PFW_CUDA(cudaMemsetAsync(lacc, 0, sizeof(double) * nmodels, st));
    for (int k = 0; k < steps; ++k, ++t) {
      for (int z = 0; z < shape->nz; ++z)
        for (int m = 0; m < shape->members; ++m) count[z * shape->members + m] = lists[z].empty() ? 0 : batch;
      if (k == 0) PFW_CUDA(cudaMemcpyAsync(dcount, count.data(), sizeof(int) * nmodels, cudaMemcpyHostToDevice, st));
      // this step's window of the order: shift the base pointer
      const size_t smem = sizeof(float) * mlp_smem_floats(dm);
      PFW_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_mlp_grad<<<dim3(ntiles, nmodels), MLP_THREADS, smem, st>>>(dm, P, b.X.as<float>(), b.y.as<float>(),
                                                                    dorder + (size_t)k * batch, (int)stride, dcount,
                                                                    b.partial.as<float>(), b.loss_part.as<double>());
      const double frac = total > 1 ? (double)t / (double)(total - 1) : 1.0;
      const float lr = (float)(opt->lr_final + 0.5 * (opt->lr - opt->lr_final) * (1.0 + std::cos(3.14159265358979323846 * frac)));
      const float bc1 = 1.f - std::pow(0.9f, (float)(t + 1)), bc2 = 1.f - std::pow(0.999f, (float)(t + 1));
      k_mlp_adam<<<dim3((dm.np + 255) / 256, nmodels), 256, 0, st>>>(dm, ntiles, b.partial.as<float>(),
                                                                     b.loss_part.as<double>(), P, b.m1.as<float>(),
                                                                     b.m2.as<float>(), lr, bc1, bc2, nullptr, lacc);
      ws->launches += 2;
    }
    PFW_CUDA(cudaGetLastError());
    if (epoch_loss) {
      PFW_CUDA(cudaMemcpyAsync(hl.data(), lacc, sizeof(double) * nmodels, cudaMemcpyDeviceToHost, st));
      PFW_CUDA(cudaStreamSynchronize(st));
      double s = 0.0;
      int live = 0;
      for (int md = 0; md < nmodels; ++md)
        if (count[md]) {
          s += hl[md] / ((double)steps * batch);
          ++live;
        }
      epoch_loss[ep] = (float)(live ? s / live : 0.0);
    }
  }
  PFW_CUDA(cudaMemcpyAsync(params, P, sizeof(float) * nmodels * dm.np, cudaMemcpyDeviceToHost, st));
  PFW_CUDA(cudaStreamSynchronize(st));
}

// ---- energy + force training steps on device buffers ----
namespace {
struct EfOrder {
  std::vector<int> order, count;
  int stride = 1, ntiles = 1;
};
EfOrder ef_order(int64_t n, const int32_t* species, const pfw_mlp_shape* shape) {
  EfOrder o;
  auto lists = by_species(n, species, shape->nz);
  size_t stride = 1;
  for (auto& l : lists) stride = std::max(stride, l.size());
  const int nmodels = shape->nz * shape->members;
  o.order.assign((size_t)nmodels * stride, 0);
  o.count.assign(nmodels, 0);
  for (int z = 0; z < shape->nz; ++z)
    for (int m = 0; m < shape->members; ++m) {
      const int md = z * shape->members + m;
      o.count[md] = (int)lists[z].size();
      std::copy(lists[z].begin(), lists[z].end(), o.order.begin() + (size_t)md * stride);
    }
  o.stride = (int)stride;
  o.ntiles = (int)((stride + MLP_TILE - 1) / MLP_TILE);
  return o;
}
}  // namespace

// Device scratch of the training steps, kept by the workspace between calls
// (a training loop calls them hundreds of times).
struct MlpScratch {
  MlpBuffers b;
};

void mlp_scratch_free(pfw_ws* ws) {
  delete ws->mlp_scratch;
  ws->mlp_scratch = nullptr;
}

static MlpBuffers& ef_buffers(pfw_ws* ws) {
  if (!ws->mlp_scratch) ws->mlp_scratch = new MlpScratch();
  return ws->mlp_scratch->b;
}

void mlp_ef_step(pfw_ws* ws, const pfw_mlp_shape* shape, float* params_dev, float* m1_dev, float* m2_dev, int64_t n,
                 const float* X_dev, const float* y_dev, const int32_t* species, const float* V_dev,
                 const float* c_dev, float wE, float lr, int64_t step, float* grad_dev, double* loss) {
  check_shape(shape);
  if (n < 1 || !params_dev || !X_dev || !y_dev || !species) throw Error(PFW_EINVAL, "samples and parameters required");
  if (!grad_dev && (!m1_dev || !m2_dev || !(lr > 0.f) || step < 1))
    throw Error(PFW_EINVAL, "an Adam step needs its moments, lr > 0 and step >= 1 (or a gradient output)");
  MlpDims dm;
  dm.make(shape->nin, shape->hidden);
  const int nmodels = shape->nz * shape->members;
  cudaStream_t st = ws->stream;
  EfOrder o = ef_order(n, species, shape);
  MlpBuffers& b = ef_buffers(ws);
  int* dorder = static_cast<int*>(b.order.ensure(sizeof(int) * o.order.size()));
  int* dcount = static_cast<int*>(b.count.ensure(sizeof(int) * nmodels));
  PFW_CUDA(cudaMemcpyAsync(dorder, o.order.data(), sizeof(int) * o.order.size(), cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(dcount, o.count.data(), sizeof(int) * nmodels, cudaMemcpyHostToDevice, st));
  float* part = static_cast<float*>(b.partial.ensure(sizeof(float) * (size_t)nmodels * o.ntiles * dm.np));
  double* lp = static_cast<double*>(b.loss_part.ensure(sizeof(double) * (size_t)nmodels * o.ntiles));
  double* lacc = static_cast<double*>(b.loss_acc.ensure(sizeof(double) * nmodels));
  PFW_CUDA(cudaMemsetAsync(lacc, 0, sizeof(double) * nmodels, st));
  const size_t smem = sizeof(float) * mlp_ef_smem_floats(dm);
  PFW_CUDA(cudaFuncSetAttribute(k_mlp_ef_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mlp_ef_grad<<<dim3(o.ntiles, nmodels), MLP_THREADS, smem, st>>>(dm, shape->members, (int)n, params_dev, X_dev,
                                                                     y_dev, V_dev, c_dev, wE, dorder, o.stride,
                                                                     dcount, part, lp);
  const float bc1 = 1.f - std::pow(0.9f, (float)step), bc2 = 1.f - std::pow(0.999f, (float)step);
  k_mlp_adam<<<dim3((dm.np + 255) / 256, nmodels), 256, 0, st>>>(dm, o.ntiles, part, lp, params_dev, m1_dev, m2_dev,
                                                                 lr, bc1, bc2, grad_dev, lacc);
  ws->launches += 2;
  PFW_CUDA(cudaGetLastError());
  if (loss) {
    std::vector<double> hl(nmodels);
    PFW_CUDA(cudaMemcpyAsync(hl.data(), lacc, sizeof(double) * nmodels, cudaMemcpyDeviceToHost, st));
    PFW_CUDA(cudaStreamSynchronize(st));
    for (int md = 0; md < nmodels; ++md) loss[md] = o.count[md] ? hl[md] / o.count[md] : 0.0;
  }
}

void mlp_input_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params_dev, int64_t n, const float* X_dev,
                    const int32_t* species, float* G_dev) {
  check_shape(shape);
  if (n < 1 || !params_dev || !X_dev || !species || !G_dev) throw Error(PFW_EINVAL, "samples and outputs required");
  MlpDims dm;
  dm.make(shape->nin, shape->hidden);
  const int nmodels = shape->nz * shape->members;
  cudaStream_t st = ws->stream;
  EfOrder o = ef_order(n, species, shape);
  MlpBuffers& b = ef_buffers(ws);
  int* dorder = static_cast<int*>(b.order.ensure(sizeof(int) * o.order.size()));
  int* dcount = static_cast<int*>(b.count.ensure(sizeof(int) * nmodels));
  PFW_CUDA(cudaMemcpyAsync(dorder, o.order.data(), sizeof(int) * o.order.size(), cudaMemcpyHostToDevice, st));
  PFW_CUDA(cudaMemcpyAsync(dcount, o.count.data(), sizeof(int) * nmodels, cudaMemcpyHostToDevice, st));
  const int ni = dm.nin + 1, h = dm.H + 1;
  const size_t smem = sizeof(float) * ((size_t)dm.H * ni + (size_t)dm.H * h + 3 * dm.H + MLP_TILE * ni + 5 * MLP_TILE * h);
  PFW_CUDA(cudaFuncSetAttribute(k_mlp_input_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mlp_input_grad<<<dim3(o.ntiles, nmodels), MLP_THREADS, smem, st>>>(dm, shape->members, (int)n, params_dev, X_dev,
                                                                        dorder, o.stride, dcount, G_dev);
  ws->launches += 1;
  PFW_CUDA(cudaGetLastError());
}

}  // namespace pfw
