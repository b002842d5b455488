// Learned initial guess: MLP parameters, features, tensor-core inference
// entry point and the training kernels (forward, backward, Adam).
//
// Training is FP32 SIMT with the forward pass seeing BF16-rounded inputs,
// weights and activations exactly where the tensor-core inference rounds
// them, so the network is trained for the arithmetic it is evaluated in
// (gradients pass straight through the rounding).  One block processes 64
// samples with all activations in shared memory; per-block gradient partial
// sums are reduced in a fixed order, so a step is deterministic.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>

#include "axb_internal.hxx"
#include "axb_mlp.cuh"

using namespace axb;

namespace {

constexpr int TB = 64;        // samples per training block
constexpr int TT = 128;       // threads per training block
constexpr int LD = MLP_H + 1; // padded row of a [TB][64] activation buffer

struct Offsets {
  int64_t w1, b1, w2, b2, w3, b3, w4, b4, P;
  AXB_HD explicit Offsets(int nf) {
    w1 = 0;
    b1 = w1 + int64_t(nf) * MLP_H;
    w2 = b1 + MLP_H;
    b2 = w2 + MLP_H * MLP_H;
    w3 = b2 + MLP_H;
    b3 = w3 + MLP_H * MLP_H;
    w4 = b3 + MLP_H;
    b4 = w4 + MLP_H * 2;
    P = b4 + 2;
  }
};

} // namespace

struct axb_mlp {
  int nf;
  int act; // hidden activation (MLP_ACT_SILU / MLP_ACT_RELU)
  int device;
  int64_t P;
  float *params; // FP32 master parameters
  float *adam_m, *adam_v, *grad;
  __nv_bfloat16 *wt; // inference weights, n-major
  float *bias;       // 64 + 64 + 64 + 8
  float *partial;    // per-block gradient partial sums
  int64_t partial_blocks;
  float *loss_partial;
  long long step;
  double bracket;

  MlpDev dev() const {
    MlpDev m;
    m.nf = nf;
    m.act = act;
    m.w1 = wt;
    m.w2 = wt + MLP_H * MLP_K1;
    m.w3 = m.w2 + MLP_H * MLP_H;
    m.w4 = m.w3 + MLP_H * MLP_H;
    m.b1 = bias;
    m.b2 = bias + MLP_H;
    m.b3 = bias + 2 * MLP_H;
    m.b4 = bias + 3 * MLP_H;
    m.bracket = bracket;
    return m;
  }
};

namespace axb {
int launch_mlp_forward_tc(const MlpDev &m, const float *feat, long long n, float *out,
                          DevStatus *status, cudaStream_t s);
int launch_mlp_guess_tc(const axb_cells &c, const MlpDev &m, float2 *guess, DevStatus *status,
                        cudaStream_t s);
int launch_mlp_guess_box_tc(const MlpBoxIn &in, const MlpDev &m, float2 *guess,
                            DevStatus *status, cudaStream_t s);
MlpDev mlp_device_view(const axb_mlp *m) { return m->dev(); }
int mlp_nf(const axb_mlp *m) { return m->nf; }
} // namespace axb

namespace {

constexpr int WT_ELEMS = MLP_H * MLP_K1 + 2 * MLP_H * MLP_H + MLP_N4 * MLP_H;

// FP32 master parameters -> BF16 n-major inference weights + padded biases.
__global__ void k_mlp_pack(const float *__restrict__ p, int nf, __nv_bfloat16 *wt,
                           float *bias) {
  const Offsets o(nf);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < MLP_H * MLP_K1) { // w1T[n][k]
    const int n = i / MLP_K1, k = i % MLP_K1;
    wt[i] = __float2bfloat16_rn(k < nf ? p[o.w1 + k * MLP_H + n] : 0.0f);
  } else if (i < MLP_H * MLP_K1 + 2 * MLP_H * MLP_H) {
    const int j = i - MLP_H * MLP_K1;
    const int layer = j / (MLP_H * MLP_H), e = j % (MLP_H * MLP_H);
    const int n = e / MLP_H, k = e % MLP_H;
    const int64_t base = layer == 0 ? o.w2 : o.w3;
    wt[i] = __float2bfloat16_rn(p[base + k * MLP_H + n]);
  } else if (i < WT_ELEMS) { // w4T[n][k], n < 8
    const int j = i - MLP_H * MLP_K1 - 2 * MLP_H * MLP_H;
    const int n = j / MLP_H, k = j % MLP_H;
    wt[i] = __float2bfloat16_rn(n < 2 ? p[o.w4 + k * 2 + n] : 0.0f);
  }
  if (i < 3 * MLP_H + MLP_N4) {
    float v;
    if (i < MLP_H)
      v = p[o.b1 + i];
    else if (i < 2 * MLP_H)
      v = p[o.b2 + i - MLP_H];
    else if (i < 3 * MLP_H)
      v = p[o.b3 + i - 2 * MLP_H];
    else
      v = (i - 3 * MLP_H) < 2 ? p[o.b4 + i - 3 * MLP_H] : 0.0f;
    bias[i] = v;
  }
}

int pack(axb_mlp *m, cudaStream_t s) {
  const int n = WT_ELEMS;
  k_mlp_pack<<<(n + 255) / 256, 256, 0, s>>>(m->params, m->nf, m->wt, m->bias);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

AXB_D float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
AXB_D float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }
AXB_D float dsilu(float z) {
  const float sg = sigm(z);
  return sg * (1.0f + z * (1.0f - sg));
}
// the hidden activation and its derivative (ReLU' = 1 for z > 0, else 0)
AXB_D float act_f(float z, int act) { return act == MLP_ACT_RELU ? fmaxf(z, 0.0f) : z * sigm(z); }
AXB_D float dact(float z, int act) {
  return act == MLP_ACT_RELU ? (z > 0.0f ? 1.0f : 0.0f) : dsilu(z);
}

// ---------------------------------------------------------------------------
// features of independent cells
// ---------------------------------------------------------------------------
__global__ void k_mlp_features(const axb_cells c, int nf, float *out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.n)
    return;
  const sym3 glo{c.g[0][i], c.g[1][i], c.g[2][i], c.g[3][i], c.g[4][i], c.g[5][i]};
  const double mom[3] = {c.mom[0][i], c.mom[1][i], c.mom[2][i]};
  const double dB[3] = {c.dB[0][i], c.dB[1][i], c.dB[2][i]};
  const CellInvariants inv = cell_invariants(c.dens[i], mom, c.tau[i], c.DYe[i], dB, glo);
  float f[MLP_K1];
  mlp_features(inv, nf, f);
  for (int k = 0; k < nf; ++k)
    out[i * nf + k] = f[k];
}

// ---------------------------------------------------------------------------
// training
// ---------------------------------------------------------------------------
struct TrainSmem {
  float W1[MLP_K1 * MLP_H], W2[MLP_H * MLP_H], W3[MLP_H * MLP_H], W4[MLP_H * 2];
  float b1[MLP_H], b2[MLP_H], b3[MLP_H], b4[2];
  float X[TB * MLP_K1];
  float Z1[TB * LD], Z2[TB * LD], Z3[TB * LD];
  float B0[TB * LD], B1[TB * LD], B2[TB * LD];
  float dY[TB * 2];
  float red[TT];
};

// out[s][n] = b[n] + sum_k in[s][k] W[k][n] for 64 samples x 64 outputs:
// thread t owns output n = t % 64 for samples [32 (t / 64), +32)
__device__ void dense64(const float *in, int ldin, int K, const float *W, const float *b,
                        float *out) {
  const int n = threadIdx.x & 63, s0 = (threadIdx.x >> 6) * 32;
  float acc[32];
#pragma unroll
  for (int s = 0; s < 32; ++s)
    acc[s] = b[n];
  for (int k = 0; k < K; ++k) {
    const float w = W[k * MLP_H + n];
#pragma unroll
    for (int s = 0; s < 32; ++s)
      acc[s] += in[(s0 + s) * ldin + k] * w;
  }
#pragma unroll
  for (int s = 0; s < 32; ++s)
    out[(s0 + s) * LD + n] = acc[s];
}

// H = bf16(act(Z)) for the 64 x 64 buffer
__device__ void act64(const float *Z, float *H, int act) {
  for (int e = threadIdx.x; e < TB * MLP_H; e += TT) {
    const int s = e / MLP_H, k = e % MLP_H;
    const float z = Z[s * LD + k];
    H[s * LD + k] = bf16r(act_f(z, act));
  }
}

// dZprev[s][k] = (sum_n dZ[s][n] W[k][n]) * act'(Zprev[s][k])
__device__ void back64(const float *dZ, const float *W, const float *Zprev, float *dZprev,
                       int act) {
  const int k = threadIdx.x & 63, s0 = (threadIdx.x >> 6) * 32;
  float acc[32];
#pragma unroll
  for (int s = 0; s < 32; ++s)
    acc[s] = 0.0f;
  for (int n = 0; n < MLP_H; ++n) {
    const float w = W[k * MLP_H + n];
#pragma unroll
    for (int s = 0; s < 32; ++s)
      acc[s] += dZ[(s0 + s) * LD + n] * w;
  }
#pragma unroll
  for (int s = 0; s < 32; ++s)
    dZprev[(s0 + s) * LD + k] = acc[s] * dact(Zprev[(s0 + s) * LD + k], act);
}

// gW[k][n] = sum_s H[s][k] dZ[s][n] (K x 64), gb[n] = sum_s dZ[s][n]
__device__ void grad64(const float *H, int ldh, int K, const float *dZ, float *gW, float *gb) {
  for (int e = threadIdx.x; e < K * MLP_H; e += TT) {
    const int k = e / MLP_H, n = e % MLP_H;
    float acc = 0.0f;
    for (int s = 0; s < TB; ++s)
      acc += H[s * ldh + k] * dZ[s * LD + n];
    gW[e] = acc;
  }
  if (threadIdx.x < MLP_H) {
    float acc = 0.0f;
    for (int s = 0; s < TB; ++s)
      acc += dZ[s * LD + threadIdx.x];
    gb[threadIdx.x] = acc;
  }
}

__global__ void __launch_bounds__(TT) k_mlp_train(const float *__restrict__ p, int nf, int act,
                                                  const float *__restrict__ feat,
                                                  const float *__restrict__ tgt,
                                                  long long n, float *partial,
                                                  float *loss_partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
  const Offsets o(nf);
  const int P = int(o.P);
  const long long base = (long long)blockIdx.x * TB;
  const float inv_n = 1.0f / float(n);
  // BF16-rounded weights (what the tensor cores multiply), FP32 biases
  for (int e = threadIdx.x; e < MLP_K1 * MLP_H; e += TT) {
    const int k = e / MLP_H;
    S.W1[e] = k < nf ? bf16r(p[o.w1 + e]) : 0.0f;
  }
  for (int e = threadIdx.x; e < MLP_H * MLP_H; e += TT) {
    S.W2[e] = bf16r(p[o.w2 + e]);
    S.W3[e] = bf16r(p[o.w3 + e]);
  }
  for (int e = threadIdx.x; e < MLP_H * 2; e += TT)
    S.W4[e] = bf16r(p[o.w4 + e]);
  if (threadIdx.x < MLP_H) {
    S.b1[threadIdx.x] = p[o.b1 + threadIdx.x];
    S.b2[threadIdx.x] = p[o.b2 + threadIdx.x];
    S.b3[threadIdx.x] = p[o.b3 + threadIdx.x];
  }
  if (threadIdx.x < 2)
    S.b4[threadIdx.x] = p[o.b4 + threadIdx.x];
  for (int e = threadIdx.x; e < TB * MLP_K1; e += TT) {
    const int s = e / MLP_K1, k = e % MLP_K1;
    const long long i = base + s;
    S.X[e] = (i < n && k < nf) ? bf16r(feat[i * nf + k]) : 0.0f;
  }
  __syncthreads();
  // forward
  dense64(S.X, MLP_K1, MLP_K1, S.W1, S.b1, S.Z1);
  __syncthreads();
  act64(S.Z1, S.B0, act);
  __syncthreads();
  dense64(S.B0, LD, MLP_H, S.W2, S.b2, S.Z2);
  __syncthreads();
  act64(S.Z2, S.B0, act);
  __syncthreads();
  dense64(S.B0, LD, MLP_H, S.W3, S.b3, S.Z3);
  __syncthreads();
  act64(S.Z3, S.B0, act); // H3
  __syncthreads();
  float l = 0.0f;
  {
    const int s = threadIdx.x >> 1, q = threadIdx.x & 1;
    float y = S.b4[q];
    for (int k = 0; k < MLP_H; ++k)
      y += S.B0[s * LD + k] * S.W4[k * 2 + q];
    const long long i = base + s;
    float d = 0.0f;
    if (i < n) {
      const float r = y - tgt[2 * i + q];
      l = r * r * inv_n;
      d = 2.0f * r * inv_n;
    }
    S.dY[s * 2 + q] = d;
  }
  S.red[threadIdx.x] = l;
  __syncthreads();
  float *gp = partial + (long long)blockIdx.x * P;
  // layer 4
  {
    const int k = threadIdx.x >> 1, q = threadIdx.x & 1;
    float acc = 0.0f;
    for (int s = 0; s < TB; ++s)
      acc += S.B0[s * LD + k] * S.dY[s * 2 + q];
    gp[o.w4 + k * 2 + q] = acc;
    if (threadIdx.x < 2) {
      float b = 0.0f;
      for (int s = 0; s < TB; ++s)
        b += S.dY[s * 2 + threadIdx.x];
      gp[o.b4 + threadIdx.x] = b;
    }
  }
  // dZ3 = (dY W4^T) * act'(Z3)
  for (int e = threadIdx.x; e < TB * MLP_H; e += TT) {
    const int s = e / MLP_H, k = e % MLP_H;
    const float dh = S.dY[s * 2] * S.W4[k * 2] + S.dY[s * 2 + 1] * S.W4[k * 2 + 1];
    S.B1[s * LD + k] = dh * dact(S.Z3[s * LD + k], act);
  }
  __syncthreads();
  act64(S.Z2, S.B0, act); // H2
  __syncthreads();
  grad64(S.B0, LD, MLP_H, S.B1, gp + o.w3, gp + o.b3);
  back64(S.B1, S.W3, S.Z2, S.B2, act); // dZ2
  __syncthreads();
  act64(S.Z1, S.B0, act); // H1
  __syncthreads();
  grad64(S.B0, LD, MLP_H, S.B2, gp + o.w2, gp + o.b2);
  back64(S.B2, S.W2, S.Z1, S.B1, act); // dZ1
  __syncthreads();
  grad64(S.X, MLP_K1, nf, S.B1, gp + o.w1, gp + o.b1);
  // loss partial (fixed-order tree)
  for (int w = TT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      S.red[threadIdx.x] += S.red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    loss_partial[blockIdx.x] = S.red[0];
}

__global__ void k_mlp_reduce(const float *partial, long long nblocks, int P, float *grad,
                             const float *loss_partial, float *loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) {
    float acc = 0.0f;
    for (long long b = 0; b < nblocks; ++b)
      acc += partial[b * P + p];
    grad[p] = acc;
  }
  if (p == 0 && loss) {
    float acc = 0.0f;
    for (long long b = 0; b < nblocks; ++b)
      acc += loss_partial[b];
    *loss = acc;
  }
}

__global__ void k_mlp_adam(float *p, const float *g, float *m, float *v, int P, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P)
    return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
AXB_API int64_t axb_mlp_param_count(int nf) {
  if (nf < 1 || nf > AXB_MLP_MAXF)
    return -1;
  return Offsets(nf).P;
}

AXB_API int axb_mlp_create(int nf, const float *params, uint64_t seed, double bracket,
                           axb_mlp **out) {
  return axb_mlp_create_act(nf, AXB_MLP_SILU, params, seed, bracket, out);
}

AXB_API int axb_mlp_create_act(int nf, int activation, const float *params, uint64_t seed,
                               double bracket, axb_mlp **out) {
  if (!out || nf < 1 || nf > MLP_K1 || !(bracket > 0 && bracket < 1) ||
      !(activation == AXB_MLP_SILU || activation == AXB_MLP_RELU))
    return AXB_ERR_ARG;
  *out = nullptr;
  const Offsets o(nf);
  float *host = static_cast<float *>(std::malloc(o.P * sizeof(float)));
  if (!host)
    return AXB_ERR_ARG;
  if (params) {
    std::memcpy(host, params, o.P * sizeof(float));
  } else {
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases
    uint64_t st = seed;
    std::memset(host, 0, o.P * sizeof(float));
    auto fill = [&](int64_t off, int fan_in, int64_t count) {
      const double a = 1.0 / std::sqrt(double(fan_in));
      for (int64_t q = 0; q < count; ++q) {
        const double u = (splitmix64(st) >> 11) * (1.0 / 9007199254740992.0);
        host[off + q] = float((2.0 * u - 1.0) * a);
      }
    };
    fill(o.w1, nf, int64_t(nf) * MLP_H);
    fill(o.w2, MLP_H, MLP_H * MLP_H);
    fill(o.w3, MLP_H, MLP_H * MLP_H);
    fill(o.w4, MLP_H, MLP_H * 2);
  }
  axb_mlp *m = new (std::nothrow) axb_mlp();
  if (!m) {
    std::free(host);
    return AXB_ERR_ARG;
  }
  m->nf = nf;
  m->act = activation == AXB_MLP_RELU ? MLP_ACT_RELU : MLP_ACT_SILU;
  m->P = o.P;
  m->bracket = bracket;
  cudaGetDevice(&m->device);
  bool ok = cudaMalloc(&m->params, o.P * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->adam_m, o.P * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->adam_v, o.P * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->grad, o.P * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&m->wt, WT_ELEMS * sizeof(__nv_bfloat16)) == cudaSuccess &&
            cudaMalloc(&m->bias, (3 * MLP_H + MLP_N4) * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMemcpy(m->params, host, o.P * sizeof(float), cudaMemcpyHostToDevice) ==
                 cudaSuccess;
  ok = ok && cudaMemset(m->adam_m, 0, o.P * sizeof(float)) == cudaSuccess &&
       cudaMemset(m->adam_v, 0, o.P * sizeof(float)) == cudaSuccess;
  std::free(host);
  ok = ok && pack(m, 0) == AXB_OK && cudaDeviceSynchronize() == cudaSuccess;
  if (!ok) {
    axb_mlp_destroy(m);
    return AXB_ERR_CUDA;
  }
  *out = m;
  return AXB_OK;
}

AXB_API int axb_mlp_destroy(axb_mlp *m) {
  if (!m)
    return AXB_ERR_ARG;
  cudaFree(m->params);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  cudaFree(m->grad);
  cudaFree(m->wt);
  cudaFree(m->bias);
  cudaFree(m->partial);
  cudaFree(m->loss_partial);
  delete m;
  return AXB_OK;
}

AXB_API int axb_mlp_get_params(const axb_mlp *m, float *params) {
  if (!m || !params)
    return AXB_ERR_ARG;
  AXB_CUDA_TRY(cudaMemcpy(params, m->params, m->P * sizeof(float), cudaMemcpyDeviceToHost));
  return AXB_OK;
}

AXB_API int axb_mlp_features(axb_ctx *c, const axb_cells *cells, int nf, float *features,
                             void *stream) {
  if (!c || !cells || !features || nf < 8 || nf > 9 || cells->n < 0)
    return AXB_ERR_ARG;
  if (!cells->dens || !cells->tau || !cells->DYe)
    return AXB_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (!cells->mom[q] || !cells->dB[q])
      return AXB_ERR_ARG;
  for (int q = 0; q < 6; ++q)
    if (!cells->g[q])
      return AXB_ERR_ARG;
  if (cells->n == 0)
    return AXB_OK;
  const long long blocks = (cells->n + 127) / 128;
  k_mlp_features<<<(unsigned)blocks, 128, 0, (cudaStream_t)stream>>>(*cells, nf, features);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

AXB_API int axb_mlp_forward(axb_ctx *c, const axb_mlp *m, const float *features, int64_t n,
                            float *out, void *stream) {
  if (!c || !m || !features || !out || n < 0)
    return AXB_ERR_ARG;
  if (n == 0)
    return AXB_OK;
  return launch_mlp_forward_tc(m->dev(), features, n, out, c->status, (cudaStream_t)stream);
}


namespace axb {
// the learned guess on the tensor cores (axb_mlp_tc.cu)
int launch_mlp_guess(const axb_cells &c, const axb_mlp *m, float2 *guess, DevStatus *status,
                     cudaStream_t s) {
  return launch_mlp_guess_tc(c, m->dev(), guess, status, s);
}
int launch_mlp_guess_box(const MlpBoxIn &in, const axb_mlp *m, float2 *guess,
                         DevStatus *status, cudaStream_t s) {
  return launch_mlp_guess_box_tc(in, m->dev(), guess, status, s);
}
} // namespace axb

AXB_API int axb_mlp_train_step(axb_ctx *c, axb_mlp *m, const float *features,
                               const float *targets, int64_t n, float lr, float beta1,
                               float beta2, float adam_eps, float *loss, float *grad,
                               void *stream) {
  if (!c || !m || !features || !targets || n < 1)
    return AXB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const long long nblocks = (n + TB - 1) / TB;
  if (nblocks > m->partial_blocks) {
    // the partial-sum buffers grow with the largest batch seen
    AXB_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(m->partial);
    cudaFree(m->loss_partial);
    m->partial = nullptr;
    m->loss_partial = nullptr;
    m->partial_blocks = 0;
    AXB_CUDA_TRY(cudaMalloc(&m->partial, nblocks * m->P * sizeof(float)));
    AXB_CUDA_TRY(cudaMalloc(&m->loss_partial, nblocks * sizeof(float)));
    m->partial_blocks = nblocks;
  }
  const size_t smem = sizeof(TrainSmem);
  AXB_CUDA_TRY(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  k_mlp_train<<<(unsigned)nblocks, TT, smem, s>>>(m->params, m->nf, m->act, features, targets, n,
                                                  m->partial, m->loss_partial);
  float *g = grad ? grad : m->grad;
  k_mlp_reduce<<<(unsigned)((m->P + 255) / 256), 256, 0, s>>>(m->partial, nblocks,
                                                               (int)m->P, g, m->loss_partial,
                                                               loss);
  if (!grad) {
    ++m->step;
    const float c1 = 1.0f - std::pow(beta1, float(m->step));
    const float c2 = 1.0f - std::pow(beta2, float(m->step));
    k_mlp_adam<<<(unsigned)((m->P + 255) / 256), 256, 0, s>>>(
        m->params, m->grad, m->adam_m, m->adam_v, (int)m->P, lr, beta1, beta2, adam_eps, c1,
        c2);
    int rc = pack(m, s);
    if (rc)
      return rc;
  }
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
