// Learned initial guess for the primitive recovery: network parameters on
// the device, the input features and the activations.  The forward pass runs
// on the tcgen05 tensor cores (axb_mlp_tc.cu).
//
// Network: nf -> 64 -> 64 -> 64 -> 2, SiLU or ReLU on the hidden layers, BF16
// weights and activations, FP32 accumulation and biases.
#pragma once

#include <cuda_bf16.h>

#include "axb_common.cuh"

namespace axb {

constexpr int MLP_H = AXB_MLP_HIDDEN; // 64
constexpr int MLP_K1 = 16;            // padded input width
constexpr int MLP_N4 = 8;             // padded output width

// Inference parameters on the device.  Weights are stored transposed,
// n-major (wT[n][k]): each output's row of K weights is contiguous, the
// K-major B operand of the tensor-core products.
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

// The interior cells of a box as the learned guess reads them: cell ci =
// ((k - ng) n_y + j - ng) n_x + i - ng, the cell-centred B the average of the
// two dB_stag faces and the cell-centred metric the average of the eight
// vertices (as the box recovery forms them, computeBfromA.cxx:67-85,
// aster_interp.hxx:23-36).
struct MlpBoxIn {
  BoxDev b;
  const double *dens, *mom[3], *tau, *DYe, *dBstag[3], *g[6];
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
  // one reciprocal of D for q, r and s
  const double iD = 1.0 / D;
  CellInvariants c;
  c.D = D;
  c.q = tau * isq * iD;
  c.r = Ssq * (iD * iD);
  c.s = Bsq * iD;
  c.t = BS * iD / sqrt(D);
  c.ye = DYe / dens;
  return c;
}

// ---------------------------------------------------------------------------
// BF16 packing and the hidden activations
// ---------------------------------------------------------------------------
AXB_D uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
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

} // namespace axb
