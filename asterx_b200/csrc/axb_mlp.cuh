// Learned initial guess for the primitive recovery: input features and the
// warp-level MLP forward pass on the tensor cores.
//
// Network: nf -> 64 -> 64 -> 64 -> 2, SiLU on the hidden layers, BF16
// weights and activations, FP32 accumulation and biases.  One warp evaluates
// 32 cells (one per lane) as two 16-row tiles of mma.sync m16n8k16: the
// recovery is FP64-bound and the network costs ~18 kflop per cell, so the
// warp-synchronous MMA keeps the evaluation inside the recovery kernel (no
// staging through memory, no block barrier) at a few percent of its time.
// Hidden C fragments become the next layer's A fragments in registers (the
// m16n8 accumulator layout of two adjacent n-tiles is the m16k16 operand
// layout); only the input features pass through 1 KB of shared memory per
// warp to reach the fragment layout.
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
struct MlpDev {
  int nf;
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

AXB_D float silu(float z) { return z / (1.0f + __expf(-z)); }

// B fragment words for n-tile nt, k-block kb of a weight stored wT[n][K].
AXB_D void load_b(const __nv_bfloat16 *wT, int K, int nt, int kb, int lane, uint32_t &b0,
                  uint32_t &b1) {
  const int n = nt * 8 + (lane >> 2);
  const int k = kb * 16 + (lane & 3) * 2;
  const uint32_t *p = reinterpret_cast<const uint32_t *>(wT + (size_t)n * K + k);
  b0 = __ldg(p);
  b1 = __ldg(p + 4); // k + 8
}

// Hidden layer: A (4 k-blocks of 16) x W [64 x 64] -> 8 n-tiles, bias, SiLU,
// repacked as the next layer's A (4 k-blocks).
AXB_D void mlp_hidden64(const __nv_bfloat16 *wT, const float *bias, int lane,
                        const uint32_t (&ain)[4][4], uint32_t (&aout)[4][4]) {
  const int t2 = (lane & 3) * 2;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    float c[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb + h;
      const float bl = __ldg(bias + nt * 8 + t2), bh = __ldg(bias + nt * 8 + t2 + 1);
      c[h][0] = bl;
      c[h][1] = bh;
      c[h][2] = bl;
      c[h][3] = bh;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        uint32_t b0, b1;
        load_b(wT, 64, nt, kk, lane, b0, b1);
        mma_bf16_16816(c[h], ain[kk], b0, b1);
      }
    }
    aout[kb][0] = pack_bf16x2(silu(c[0][0]), silu(c[0][1]));
    aout[kb][1] = pack_bf16x2(silu(c[0][2]), silu(c[0][3]));
    aout[kb][2] = pack_bf16x2(silu(c[1][0]), silu(c[1][1]));
    aout[kb][3] = pack_bf16x2(silu(c[1][2]), silu(c[1][3]));
  }
}

// One 16-row tile (rows 16 mt .. 16 mt + 15 of the warp's cells): returns
// the layer-4 accumulator fragment (outputs in columns 0 and 1).
AXB_D void mlp_tile(const MlpDev &m, const uint32_t *stage, int mt, int lane,
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
      const float bl = __ldg(m.b1 + nt * 8 + t2), bh = __ldg(m.b1 + nt * 8 + t2 + 1);
      cc[h][0] = bl;
      cc[h][1] = bh;
      cc[h][2] = bl;
      cc[h][3] = bh;
      uint32_t b0, b1;
      load_b(m.w1, MLP_K1, nt, 0, lane, b0, b1);
      mma_bf16_16816(cc[h], a1, b0, b1);
    }
    h1[kb][0] = pack_bf16x2(silu(cc[0][0]), silu(cc[0][1]));
    h1[kb][1] = pack_bf16x2(silu(cc[0][2]), silu(cc[0][3]));
    h1[kb][2] = pack_bf16x2(silu(cc[1][0]), silu(cc[1][1]));
    h1[kb][3] = pack_bf16x2(silu(cc[1][2]), silu(cc[1][3]));
  }
  uint32_t h2[4][4], h3[4][4];
  mlp_hidden64(m.w2, m.b2, lane, h1, h2);
  mlp_hidden64(m.w3, m.b3, lane, h2, h3);
  // layer 4: [16 x 64] x [64 x 8]
  const float bl = __ldg(m.b4 + t2), bh = __ldg(m.b4 + t2 + 1);
  c[0] = bl;
  c[1] = bh;
  c[2] = bl;
  c[3] = bh;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t b0, b1;
    load_b(m.w4, 64, 0, kk, lane, b0, b1);
    mma_bf16_16816(c, h3[kk], b0, b1);
  }
}

// Forward pass for the 32 cells of a warp.  `f` holds this lane's features
// (MLP_K1 floats, zero beyond nf); `stage` is 32 x 8 words of shared memory
// owned by this warp.  Returns this lane's two outputs.  Must be called by
// all 32 lanes of the warp.
AXB_D void mlp_forward_warp(const MlpDev &m, const float (&f)[MLP_K1], uint32_t *stage,
                            float &y0, float &y1) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int w = 0; w < 8; ++w)
    stage[lane * 8 + w] = pack_bf16x2(f[2 * w], f[2 * w + 1]);
  __syncwarp();
  float o0[4], o1[4];
  mlp_tile(m, stage, 0, lane, o0);
  mlp_tile(m, stage, 1, lane, o1);
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

} // namespace axb
