// Learned initial guess for the primitive recovery: input features and the
// warp-level MLP forward pass on the tensor cores.
//
// Network: nf -> 64 -> 64 -> 64 -> 2, SiLU or ReLU on the hidden layers, BF16
// weights and activations, FP32 accumulation and biases.  A CTA stages the
// ~20 KB of weights in shared memory once (rows padded so that the B
// fragments load without bank conflicts) and each warp evaluates 32 cells
// (one per lane) as two 16-row tiles of mma.sync m16n8k16.  Hidden
// accumulator fragments become the next layer's A fragments in registers
// (the m16n8 accumulator layout of two adjacent n-tiles is the m16k16
// operand layout); only the input features pass through 1 KB of shared
// memory per warp to reach the fragment layout.
#pragma once

#include <cuda_bf16.h>

#include "axb_common.cuh"

namespace axb {

constexpr int MLP_H = AXB_MLP_HIDDEN; // 64
constexpr int MLP_K1 = 16;            // padded input width
constexpr int MLP_N4 = 8;             // padded output width

// Inference parameters on the device.  Weights are stored transposed,
// n-major (wT[n][k]), so that the two consecutive k of a B fragment are one
// 32-bit word.
enum { MLP_ACT_SILU = 0, MLP_ACT_RELU = 1 };

struct MlpDev {
  int nf;
  int act; // MLP_ACT_SILU or MLP_ACT_RELU
  const __nv_bfloat16 *w1; // [64][16]
  const __nv_bfloat16 *w2; // [64][64]
  const __nv_bfloat16 *w3; // [64][64]
  const __nv_bfloat16 *w4; // [8][64] (outputs 2..7 zero)
  const float *b1, *b2, *b3, *b4; // 64, 64, 64, 8
  double bracket;
};

// ---------------------------------------------------------------------------
// features (double arithmetic, FP32 result); must match axb_mlp_features
// ---------------------------------------------------------------------------
struct CellInvariants {
  double D, q, r, s, t, ye;
};

AXB_HD void mlp_features(const CellInvariants &c, int nf, float *f) {
  const double q = fmax(c.q, -0.999);
  const double lq = log1p(q);
  const double lr = log1p(fmax(c.r, 0.0));
  const double den = 1.0 + q + c.s;
  f[0] = float(log(fmax(c.D, 1e-300)) / 10.0);
  f[1] = float(lq);
  f[2] = float(0.5 * lr);
  f[3] = float(log1p(fmax(c.s, 0.0)));
  f[4] = float(fmin(c.t * c.t / (c.r * c.s + 1e-300), 1.0));
  f[5] = float(c.r / (den * den));
  f[6] = float(c.s / den);
  f[7] = float(lq - 0.5 * lr);
  if (nf > 8)
    f[8] = float(c.ye);
}

// Invariants from densitized conserved variables and gamma_ij
// (q, r, s, t as in c2p_1DPalenzuela.hxx:150-153,267-270).
AXB_HD CellInvariants cell_invariants(double dens, const double mom[3], double tau,
                                      double DYe, const double dB[3], const sym3 &glo) {
  const double detg = det3(glo);
  const double sq_detg = sqrt(detg);
  const double isq = 1.0 / sq_detg;
  const sym3 gup = inv3(glo, detg);
  const double D = dens * isq;
  double S[3], B[3];
  for (int i = 0; i < 3; ++i) {
    S[i] = mom[i] * isq;
    B[i] = dB[i] * isq;
  }
  double Su[3], Bl[3];
  lower3(gup, S, Su);
  lower3(glo, B, Bl);
  const double Ssq = dot3(S, Su), Bsq = dot3(B, Bl), BS = dot3(B, S);
  CellInvariants c;
  c.D = D;
  c.q = tau * isq / D;
  c.r = Ssq / (D * D);
  c.s = Bsq / D;
  c.t = BS / (D * sqrt(D));
  c.ye = DYe / dens;
  return c;
}

// ---------------------------------------------------------------------------
// tensor-core forward pass of one warp (32 cells, lane = cell)
// ---------------------------------------------------------------------------
AXB_D uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

AXB_D void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
               "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SiLU as z (1 + tanh(z/2)) / 2 with the hardware tanh approximation: one
// special-function instruction per activation instead of an exponential and
// a reciprocal (the special-function unit is what bounds this network).  Its
// relative error (~2^-11) is below the BF16 rounding that follows.
AXB_D float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
AXB_D float silu(float z) {
  const float hz = 0.5f * z;
  return fmaf(hz, tanh_approx(hz), hz);
}
// The hidden activation: SiLU, or ReLU (one FP32 max, no special-function
// instruction).  `act` is uniform over the warp.
AXB_D float mlp_act(float z, int act) { return act == MLP_ACT_RELU ? fmaxf(z, 0.0f) : silu(z); }

// Weights in shared memory, n-major with padded rows (K + 8 bf16): the
// eight rows a B-fragment load touches then fall in distinct banks.
constexpr int MLP_LD1 = MLP_K1 + 8; // 24
constexpr int MLP_LDH = MLP_H + 8;  // 72
struct MlpSmem {
  __nv_bfloat16 w1[MLP_H * MLP_LD1];
  __nv_bfloat16 w2[MLP_H * MLP_LDH];
  __nv_bfloat16 w3[MLP_H * MLP_LDH];
  __nv_bfloat16 w4[MLP_N4 * MLP_LDH];
  float b1[MLP_H], b2[MLP_H], b3[MLP_H], b4[MLP_N4];
  int act;
};

// Cooperative copy of the device weights into shared memory (all threads
// of the block; a __syncthreads must follow).
AXB_D void mlp_stage_weights(const MlpDev &m, MlpSmem &w) {
  for (int e = threadIdx.x; e < MLP_H * MLP_K1; e += blockDim.x)
    w.w1[(e / MLP_K1) * MLP_LD1 + e % MLP_K1] = m.w1[e];
  for (int e = threadIdx.x; e < MLP_H * MLP_H; e += blockDim.x) {
    w.w2[(e / MLP_H) * MLP_LDH + e % MLP_H] = m.w2[e];
    w.w3[(e / MLP_H) * MLP_LDH + e % MLP_H] = m.w3[e];
  }
  for (int e = threadIdx.x; e < MLP_N4 * MLP_H; e += blockDim.x)
    w.w4[(e / MLP_H) * MLP_LDH + e % MLP_H] = m.w4[e];
  for (int e = threadIdx.x; e < MLP_H; e += blockDim.x) {
    w.b1[e] = m.b1[e];
    w.b2[e] = m.b2[e];
    w.b3[e] = m.b3[e];
  }
  if (threadIdx.x < MLP_N4)
    w.b4[threadIdx.x] = m.b4[threadIdx.x];
  if (threadIdx.x == 0)
    w.act = m.act;
}

// B fragment words for n-tile nt, k-block kb of a weight stored wT[n][ld].
AXB_D void load_b(const __nv_bfloat16 *wT, int ld, int nt, int kb, int lane, uint32_t &b0,
                  uint32_t &b1) {
  const int n = nt * 8 + (lane >> 2);
  const int k = kb * 16 + (lane & 3) * 2;
  const uint32_t *p = reinterpret_cast<const uint32_t *>(wT + n * ld + k);
  b0 = p[0];
  b1 = p[4]; // k + 8
}

// Hidden layer: A (4 k-blocks of 16) x W [64 x 64] -> 8 n-tiles, bias, SiLU,
// repacked as the next layer's A (4 k-blocks).
AXB_D void mlp_hidden64(const __nv_bfloat16 *wT, const float *bias, int act, int lane,
                        const uint32_t (&ain)[4][4], uint32_t (&aout)[4][4]) {
  const int t2 = (lane & 3) * 2;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    float c[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb + h;
      const float bl = bias[nt * 8 + t2], bh = bias[nt * 8 + t2 + 1];
      c[h][0] = bl;
      c[h][1] = bh;
      c[h][2] = bl;
      c[h][3] = bh;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        uint32_t b0, b1;
        load_b(wT, MLP_LDH, nt, kk, lane, b0, b1);
        mma_bf16_16816(c[h], ain[kk], b0, b1);
      }
    }
    aout[kb][0] = pack_bf16x2(mlp_act(c[0][0], act), mlp_act(c[0][1], act));
    aout[kb][1] = pack_bf16x2(mlp_act(c[0][2], act), mlp_act(c[0][3], act));
    aout[kb][2] = pack_bf16x2(mlp_act(c[1][0], act), mlp_act(c[1][1], act));
    aout[kb][3] = pack_bf16x2(mlp_act(c[1][2], act), mlp_act(c[1][3], act));
  }
}

// One 16-row tile (rows 16 mt .. 16 mt + 15 of the warp's cells): returns
// the layer-4 accumulator fragment (outputs in columns 0 and 1).
AXB_D void mlp_tile(const MlpSmem &w, const uint32_t *stage, int mt, int lane,
                    float (&c)[4]) {
  const int g = lane >> 2, t = lane & 3, t2 = t * 2;
  const int r0 = mt * 16 + g, r1 = r0 + 8;
  const uint32_t a1[4] = {stage[r0 * 8 + t], stage[r1 * 8 + t], stage[r0 * 8 + t + 4],
                          stage[r1 * 8 + t + 4]};
  // layer 1: [16 x 16] x [16 x 64]
  uint32_t h1[4][4];
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    float cc[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb + h;
      const float bl = w.b1[nt * 8 + t2], bh = w.b1[nt * 8 + t2 + 1];
      cc[h][0] = bl;
      cc[h][1] = bh;
      cc[h][2] = bl;
      cc[h][3] = bh;
      uint32_t b0, b1;
      load_b(w.w1, MLP_LD1, nt, 0, lane, b0, b1);
      mma_bf16_16816(cc[h], a1, b0, b1);
    }
    h1[kb][0] = pack_bf16x2(mlp_act(cc[0][0], w.act), mlp_act(cc[0][1], w.act));
    h1[kb][1] = pack_bf16x2(mlp_act(cc[0][2], w.act), mlp_act(cc[0][3], w.act));
    h1[kb][2] = pack_bf16x2(mlp_act(cc[1][0], w.act), mlp_act(cc[1][1], w.act));
    h1[kb][3] = pack_bf16x2(mlp_act(cc[1][2], w.act), mlp_act(cc[1][3], w.act));
  }
  uint32_t h2[4][4], h3[4][4];
  mlp_hidden64(w.w2, w.b2, w.act, lane, h1, h2);
  mlp_hidden64(w.w3, w.b3, w.act, lane, h2, h3);
  // layer 4: [16 x 64] x [64 x 8]
  const float bl = w.b4[t2], bh = w.b4[t2 + 1];
  c[0] = bl;
  c[1] = bh;
  c[2] = bl;
  c[3] = bh;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t b0, b1;
    load_b(w.w4, MLP_LDH, 0, kk, lane, b0, b1);
    mma_bf16_16816(c, h3[kk], b0, b1);
  }
}

// Hidden layer for both 16-row tiles at once: the two accumulator chains
// are independent, which doubles the MMAs in flight per warp and reuses
// each B fragment for both tiles.
AXB_D void mlp_hidden64x2(const __nv_bfloat16 *wT, const float *bias, int act, int lane,
                          const uint32_t (&ain0)[4][4], const uint32_t (&ain1)[4][4],
                          uint32_t (&aout0)[4][4], uint32_t (&aout1)[4][4]) {
  const int t2 = (lane & 3) * 2;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    float c0[2][4], c1[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb + h;
      const float bl = bias[nt * 8 + t2], bh = bias[nt * 8 + t2 + 1];
      c0[h][0] = c1[h][0] = bl;
      c0[h][1] = c1[h][1] = bh;
      c0[h][2] = c1[h][2] = bl;
      c0[h][3] = c1[h][3] = bh;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        uint32_t b0, b1;
        load_b(wT, MLP_LDH, nt, kk, lane, b0, b1);
        mma_bf16_16816(c0[h], ain0[kk], b0, b1);
        mma_bf16_16816(c1[h], ain1[kk], b0, b1);
      }
    }
    aout0[kb][0] = pack_bf16x2(mlp_act(c0[0][0], act), mlp_act(c0[0][1], act));
    aout0[kb][1] = pack_bf16x2(mlp_act(c0[0][2], act), mlp_act(c0[0][3], act));
    aout0[kb][2] = pack_bf16x2(mlp_act(c0[1][0], act), mlp_act(c0[1][1], act));
    aout0[kb][3] = pack_bf16x2(mlp_act(c0[1][2], act), mlp_act(c0[1][3], act));
    aout1[kb][0] = pack_bf16x2(mlp_act(c1[0][0], act), mlp_act(c1[0][1], act));
    aout1[kb][1] = pack_bf16x2(mlp_act(c1[0][2], act), mlp_act(c1[0][3], act));
    aout1[kb][2] = pack_bf16x2(mlp_act(c1[1][0], act), mlp_act(c1[1][1], act));
    aout1[kb][3] = pack_bf16x2(mlp_act(c1[1][2], act), mlp_act(c1[1][3], act));
  }
}

// Layer 1 of one tile (K = 16 features).
AXB_D void mlp_layer1(const MlpSmem &w, const uint32_t (&a1)[4], int lane,
                      uint32_t (&h1)[4][4]) {
  const int t2 = (lane & 3) * 2;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    float cc[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb + h;
      const float bl = w.b1[nt * 8 + t2], bh = w.b1[nt * 8 + t2 + 1];
      cc[h][0] = bl;
      cc[h][1] = bh;
      cc[h][2] = bl;
      cc[h][3] = bh;
      uint32_t b0, b1;
      load_b(w.w1, MLP_LD1, nt, 0, lane, b0, b1);
      mma_bf16_16816(cc[h], a1, b0, b1);
    }
    h1[kb][0] = pack_bf16x2(mlp_act(cc[0][0], w.act), mlp_act(cc[0][1], w.act));
    h1[kb][1] = pack_bf16x2(mlp_act(cc[0][2], w.act), mlp_act(cc[0][3], w.act));
    h1[kb][2] = pack_bf16x2(mlp_act(cc[1][0], w.act), mlp_act(cc[1][1], w.act));
    h1[kb][3] = pack_bf16x2(mlp_act(cc[1][2], w.act), mlp_act(cc[1][3], w.act));
  }
}

// Both tiles of the warp through the whole network; o0 / o1 are the layer-4
// accumulator fragments of rows 0-15 and 16-31.
AXB_D void mlp_tile2(const MlpSmem &w, const uint32_t *stage, int lane, float (&o0)[4],
                     float (&o1)[4]) {
  const int g = lane >> 2, t = lane & 3, t2 = t * 2;
  uint32_t x0[4] = {stage[g * 8 + t], stage[(g + 8) * 8 + t], stage[g * 8 + t + 4],
                    stage[(g + 8) * 8 + t + 4]};
  uint32_t x1[4] = {stage[(g + 16) * 8 + t], stage[(g + 24) * 8 + t],
                    stage[(g + 16) * 8 + t + 4], stage[(g + 24) * 8 + t + 4]};
  uint32_t p0[4][4], p1[4][4], q0[4][4], q1[4][4];
  mlp_layer1(w, x0, lane, p0);
  mlp_layer1(w, x1, lane, p1);
  mlp_hidden64x2(w.w2, w.b2, w.act, lane, p0, p1, q0, q1);
  mlp_hidden64x2(w.w3, w.b3, w.act, lane, q0, q1, p0, p1);
  const float bl = w.b4[t2], bh = w.b4[t2 + 1];
  o0[0] = o1[0] = bl;
  o0[1] = o1[1] = bh;
  o0[2] = o1[2] = bl;
  o0[3] = o1[3] = bh;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t b0, b1;
    load_b(w.w4, MLP_LDH, 0, kk, lane, b0, b1);
    mma_bf16_16816(o0, p0[kk], b0, b1);
    mma_bf16_16816(o1, p1[kk], b0, b1);
  }
}

// Forward pass for the 32 cells of a warp.  `f` holds this lane's features
// (MLP_K1 floats, zero beyond nf); `stage` is 32 x 8 words of shared memory
// owned by this warp.  Returns this lane's two outputs.  Must be called by
// all 32 lanes of the warp.
AXB_D void mlp_forward_warp(const MlpSmem &w, const float (&f)[MLP_K1], uint32_t *stage,
                            float &y0, float &y1) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < 8; ++q)
    stage[lane * 8 + q] = pack_bf16x2(f[2 * q], f[2 * q + 1]);
  __syncwarp();
  float o0[4], o1[4];
  mlp_tile2(w, stage, lane, o0, o1);
  __syncwarp();
  // outputs 0, 1 of row r sit in lane 4 (r mod 8), registers 0/1 (r < 8) or
  // 2/3 (r >= 8) of the row's tile
  const int mt = lane >> 4, r = lane & 15, src = (r & 7) * 4;
  const float v00 = __shfl_sync(0xffffffffu, o0[0], src);
  const float v01 = __shfl_sync(0xffffffffu, o0[1], src);
  const float v02 = __shfl_sync(0xffffffffu, o0[2], src);
  const float v03 = __shfl_sync(0xffffffffu, o0[3], src);
  const float v10 = __shfl_sync(0xffffffffu, o1[0], src);
  const float v11 = __shfl_sync(0xffffffffu, o1[1], src);
  const float v12 = __shfl_sync(0xffffffffu, o1[2], src);
  const float v13 = __shfl_sync(0xffffffffu, o1[3], src);
  if (mt == 0) {
    y0 = r < 8 ? v00 : v02;
    y1 = r < 8 ? v01 : v03;
  } else {
    y0 = r < 8 ? v10 : v12;
    y1 = r < 8 ? v11 : v13;
  }
}

// The learned guess of cell i of `c` (all 32 lanes of the warp call this;
// lanes with valid == false take part with zero features): features from
// the conserved variables and metric, the network, and the decoded guess
// x = h W (y0 places x in the Palenzuela scheme's initial bracket
// [max(1e-10, 1 + q - s), 2 + 2 q - s], c2p_1DPalenzuela.hxx:395-398) and
// W = max(exp(y1), 1).
template <class Cells>
AXB_D void mlp_cell_guess(const Cells &c, long long i, bool valid, int nf, const MlpSmem &w,
                          uint32_t *stage, double &x, double &W) {
  float f[MLP_K1];
#pragma unroll
  for (int k = 0; k < MLP_K1; ++k)
    f[k] = 0.0f;
  CellInvariants inv{1.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (valid) {
    const sym3 glo{c.g[0][i], c.g[1][i], c.g[2][i], c.g[3][i], c.g[4][i], c.g[5][i]};
    const double mom[3] = {c.mom[0][i], c.mom[1][i], c.mom[2][i]};
    const double dB[3] = {c.dB[0][i], c.dB[1][i], c.dB[2][i]};
    inv = cell_invariants(c.dens[i], mom, c.tau[i], c.DYe[i], dB, glo);
    mlp_features(inv, nf, f);
  }
  float y0, y1;
  mlp_forward_warp(w, f, stage, y0, y1);
  const double lo = fmax(1e-10, 1.0 + inv.q - inv.s), hi = 2.0 + 2.0 * inv.q - inv.s;
  x = lo + double(y0) * (hi - lo);
  W = fmax(exp(double(y1)), 1.0);
}

} // namespace axb
