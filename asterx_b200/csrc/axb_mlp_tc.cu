// Learned-guess network on the 5th-generation tensor cores (tcgen05).
//
// One CTA of 128 threads evaluates tiles of 128 cells: thread t owns row t
// (cell t of the tile).  Per layer, one elected thread issues the
// 128 x N x K product as K/16 `tcgen05.mma.cta_group::1.kind::f16`
// instructions (BF16 operands in shared memory, FP32 accumulator in tensor
// memory), commits it to an mbarrier, and every thread then reads its row of
// the accumulator back with `tcgen05.ld.32x32b` (warp w owns TMEM lanes
// 32w..32w+31), applies the activation, rounds to BF16 and stores the row as
// the next layer's A operand.  The hidden layers' biases ride in the
// products: feature columns 14 and 15 of every row hold 1, and one more K = 16
// step per layer multiplies the tile's features by a block whose columns 14
// and 15 hold the bias split into a BF16 high and low part (zero elsewhere).
//
// Operands use the canonical K-major layout without swizzle: 8 x 8 core
// matrices of 8 rows x 16 bytes; element (r, k) of an R x K operand sits at
// byte (r/8) * 16K + (k/8) * 128 + (r%8) * 16 + (k%8) * 2, so the leading
// byte offset (next core matrix along K) is 128 and the stride byte offset
// (next 8 rows) is 16K.  One K = 16 step covers two core matrices along K.
//
// Numerics: BF16 weights and activations, FP32 accumulation, biases to about
// 16 bits (high + low BF16 part), so the outputs agree with the FP32 network
// of the training kernels (axb_mlp.cu) to the BF16 rounding of the operands.
// Every wait on the mbarrier is bounded: on a timeout the CTA sets
// AXB_EW_MMA_TIMEOUT, releases its tensor memory and returns.
#include <cuda_bf16.h>

#include "axb_internal.hxx"
#include "axb_mlp.cuh"

namespace axb {
namespace {

constexpr int TC_M = 128;    // cells per tile = rows of every product
constexpr int TC_COLS = 64;  // tensor-memory columns: one 128 x 64 FP32 accumulator
constexpr int TC_N4 = 16;    // output layer padded to the smallest N for M = 128
constexpr long long TC_WAIT_LIMIT = 1LL << 22; // mbarrier polls before giving up
constexpr int TC_BIAS_COL = 14; // feature columns 14, 15 hold 1: the biases' columns

// byte offset of element (r, k) of an R x K operand (canonical K-major)
AXB_HD constexpr unsigned kmaj(int r, int k, int K) {
  return unsigned((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

struct __align__(128) TcSmem {
  __nv_bfloat16 w1[MLP_H * MLP_K1]; // B of layer 1: N = 64 x K = 16
  __nv_bfloat16 w2[MLP_H * MLP_H];  // N = 64 x K = 64
  __nv_bfloat16 w3[MLP_H * MLP_H];
  __nv_bfloat16 w4[TC_N4 * MLP_H];  // N = 16 x K = 64, rows 2..15 zero
  __nv_bfloat16 w2b[MLP_H * MLP_K1]; // layer 2's bias block: N = 64 x K = 16
  __nv_bfloat16 w3b[MLP_H * MLP_K1]; // layer 3's
  __nv_bfloat16 a1[TC_M * MLP_K1];  // features of the tile (kept for the bias steps)
  __nv_bfloat16 ah[TC_M * MLP_H];   // hidden activations of the tile
  float b4[2];
  unsigned long long bar;
  unsigned int tmem;
  int act;
};

AXB_D unsigned smem_u32(const void *p) { return unsigned(__cvta_generic_to_shared(p)); }

// shared-memory matrix descriptor (no swizzle, K-major, Blackwell version 1)
AXB_D unsigned long long smem_desc(const void *p, unsigned sbo) {
  unsigned long long d = (smem_u32(p) >> 4) & 0x3FFFu;
  d |= (unsigned long long)((128u >> 4) & 0x3FFFu) << 16; // leading byte offset
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;  // stride byte offset
  d |= 1ull << 46;                                        // descriptor version
  return d;
}

// instruction descriptor: D FP32, A and B BF16, both K-major, M = 128, N
AXB_HD constexpr unsigned idesc_bf16(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(N >> 3) << 17) |
         (unsigned(TC_M >> 4) << 24);
}

AXB_D void umma(unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned idesc,
                unsigned accumulate) {
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
               :
               : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

AXB_D void umma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(bar)
               : "memory");
}

AXB_D void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
AXB_D void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
AXB_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// bounded wait for phase `parity` of the mbarrier; false on timeout
AXB_D bool mbar_wait(unsigned bar, unsigned parity) {
  for (long long it = 0; it < TC_WAIT_LIMIT; ++it) {
    unsigned done;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    if (done)
      return true;
  }
  return false;
}

// 16 consecutive FP32 accumulator columns of this thread's row; the load and
// its completion wait in one statement, so no use of the values can be
// scheduled before the wait
AXB_D void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
               "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
               "tcgen05.wait::ld.sync.aligned;"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q)
    v[q] = __uint_as_float(r[q]);
}

// 32 consecutive columns: one load, one wait
AXB_D void tmem_ld32(unsigned taddr, float (&v)[32]) {
  unsigned r[32];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
               "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
               "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, "
               "%31}, [%32];\n\t"
               "tcgen05.wait::ld.sync.aligned;"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                 "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                 "=r"(r[30]), "=r"(r[31])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q)
    v[q] = __uint_as_float(r[q]);
}

// Stage the network's weights in the canonical operand layout (all threads;
// a barrier must follow).
AXB_D void tc_stage(const MlpDev &m, TcSmem &S) {
  const int t = threadIdx.x, nt = blockDim.x;
  char *w1 = reinterpret_cast<char *>(S.w1), *w2 = reinterpret_cast<char *>(S.w2),
       *w3 = reinterpret_cast<char *>(S.w3), *w4 = reinterpret_cast<char *>(S.w4);
  // layer 1's bias rides in the product: feature columns 14 and 15 hold 1
  // and the weights there the bias split into a BF16 high and low part
  // (the features use at most 9 of the 16 columns)
  for (int e = t; e < MLP_H * MLP_K1; e += nt) {
    const int n = e / MLP_K1, k = e % MLP_K1;
    __nv_bfloat16 v = m.w1[e];
    if (k >= TC_BIAS_COL) {
      const __nv_bfloat16 hi = __float2bfloat16(m.b1[n]);
      v = k == TC_BIAS_COL ? hi : __float2bfloat16(m.b1[n] - __bfloat162float(hi));
    }
    *reinterpret_cast<__nv_bfloat16 *>(w1 + kmaj(n, k, MLP_K1)) = v;
  }
  for (int e = t; e < MLP_H * MLP_H; e += nt) {
    *reinterpret_cast<__nv_bfloat16 *>(w2 + kmaj(e / MLP_H, e % MLP_H, MLP_H)) = m.w2[e];
    *reinterpret_cast<__nv_bfloat16 *>(w3 + kmaj(e / MLP_H, e % MLP_H, MLP_H)) = m.w3[e];
  }
  for (int e = t; e < TC_N4 * MLP_H; e += nt) {
    const int n = e / MLP_H, k = e % MLP_H;
    *reinterpret_cast<__nv_bfloat16 *>(w4 + kmaj(n, k, MLP_H)) =
        n < 2 ? m.w4[n * MLP_H + k] : __float2bfloat16(0.0f);
  }
  // the bias blocks of layers 2 and 3 (against the features' unit columns)
  char *w2b = reinterpret_cast<char *>(S.w2b), *w3b = reinterpret_cast<char *>(S.w3b);
  for (int e = t; e < MLP_H * MLP_K1; e += nt) {
    const int n = e / MLP_K1, k = e % MLP_K1;
    __nv_bfloat16 v2 = __float2bfloat16(0.0f), v3 = v2;
    if (k >= TC_BIAS_COL) {
      const __nv_bfloat16 h2 = __float2bfloat16(m.b2[n]), h3 = __float2bfloat16(m.b3[n]);
      v2 = k == TC_BIAS_COL ? h2 : __float2bfloat16(m.b2[n] - __bfloat162float(h2));
      v3 = k == TC_BIAS_COL ? h3 : __float2bfloat16(m.b3[n] - __bfloat162float(h3));
    }
    *reinterpret_cast<__nv_bfloat16 *>(w2b + kmaj(n, k, MLP_K1)) = v2;
    *reinterpret_cast<__nv_bfloat16 *>(w3b + kmaj(n, k, MLP_K1)) = v3;
  }
  if (t < 2)
    S.b4[t] = m.b4[t];
  if (t == 0)
    S.act = m.act;
}

// One layer's product into tensor memory: thread 0 issues K/16 MMAs (and,
// with `Bb`, one more K = 16 step of the features against the bias block)
// and the commit; every thread waits for the result.  Returns false on a
// timeout.
AXB_D bool tc_layer(const TcSmem &S, const void *A, const void *B, int K, int N, unsigned tmem,
                    unsigned &parity, const void *Bb = nullptr) {
  const unsigned bar = smem_u32(&S.bar);
  if (threadIdx.x == 0) {
    fence_after_sync();
    const unsigned sbo = unsigned(K * 16);
    const unsigned id = idesc_bf16(N);
    for (int kk = 0; kk < K / 16; ++kk)
      umma(tmem, smem_desc(static_cast<const char *>(A) + kk * 256, sbo),
           smem_desc(static_cast<const char *>(B) + kk * 256, sbo), id, kk > 0);
    if (Bb)
      umma(tmem, smem_desc(S.a1, MLP_K1 * 16), smem_desc(Bb, MLP_K1 * 16), id, 1u);
    umma_commit(bar);
  }
  // one thread waits on the mbarrier, the others at the block barrier (so
  // they issue nothing meanwhile)
  const bool ok = threadIdx.x == 0 ? mbar_wait(bar, parity) : true;
  parity ^= 1u;
  const bool all_ok = !__syncthreads_or(!ok);
  fence_after_sync();
  return all_ok;
}

// a and b rounded to BF16 and clamped at 0 in one conversion (a in the low
// half); rounding and the clamp commute
AXB_D unsigned relu_bf16x2(float a, float b) {
  unsigned d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
  return d;
}

// This thread's row of a 64-column accumulator (bias included), activated,
// rounded to BF16 and stored as row `r` of the hidden operand.
AXB_D void tc_hidden_out(TcSmem &S, unsigned trow, int r) {
  char *ah = reinterpret_cast<char *>(S.ah);
  const bool relu = S.act == MLP_ACT_RELU;
#pragma unroll
  for (int c32 = 0; c32 < MLP_H / 32; ++c32) {
    float v[32];
    tmem_ld32(trow + unsigned(c32 * 32), v);
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      uint4 pk;
      unsigned *p = reinterpret_cast<unsigned *>(&pk);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float a = v[h * 8 + 2 * q], b = v[h * 8 + 2 * q + 1];
        p[q] = relu ? relu_bf16x2(a, b) : pack_bf16x2(silu(a), silu(b));
      }
      *reinterpret_cast<uint4 *>(ah + kmaj(r, c32 * 32 + h * 8, MLP_H)) = pk;
    }
  }
}

// The network on the tile whose features are in S.a1: outputs of row
// threadIdx.x.  Every thread of the CTA calls; false on a timeout.
AXB_D bool tc_forward(TcSmem &S, unsigned tmem, unsigned &parity, float &y0, float &y1) {
  const int r = threadIdx.x;
  const unsigned trow = tmem + (unsigned((threadIdx.x >> 5) * 32) << 16);
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  if (!tc_layer(S, S.a1, S.w1, MLP_K1, MLP_H, tmem, parity))
    return false;
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    tc_hidden_out(S, trow, r);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    const void *B = l == 0 ? static_cast<const void *>(S.w2)
                           : l == 1 ? static_cast<const void *>(S.w3) : S.w4;
    const void *Bb = l == 0 ? static_cast<const void *>(S.w2b)
                            : l == 1 ? static_cast<const void *>(S.w3b) : nullptr;
    if (!tc_layer(S, S.ah, B, MLP_H, l < 2 ? MLP_H : TC_N4, tmem, parity, Bb))
      return false;
  }
  float v[16];
  tmem_ld16(trow, v);
  y0 = v[0] + S.b4[0];
  y1 = v[1] + S.b4[1];
  fence_before_sync();
  return true;
}

// Set-up shared by the kernels: weights, mbarrier, tensor memory.
AXB_D unsigned tc_setup(const MlpDev &m, TcSmem &S) {
  tc_stage(m, S);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(TC_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  return S.tmem;
}

AXB_D void tc_teardown(unsigned tmem, bool failed, DevStatus *status) {
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TC_COLS)
                 : "memory");
  }
  if (failed && threadIdx.x == 0 && status)
    atomicOr(&status->error_word, AXB_EW_MMA_TIMEOUT);
}

// features of this thread's row (zero beyond nf) into the A operand
AXB_D void tc_put_features(TcSmem &S, float (&f)[MLP_K1]) {
  char *a1 = reinterpret_cast<char *>(S.a1);
  f[TC_BIAS_COL] = 1.0f;
  f[TC_BIAS_COL + 1] = 1.0f;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint4 pk;
    unsigned *p = reinterpret_cast<unsigned *>(&pk);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      p[q] = pack_bf16x2(f[h * 8 + 2 * q], f[h * 8 + 2 * q + 1]);
    *reinterpret_cast<uint4 *>(a1 + kmaj(threadIdx.x, h * 8, MLP_K1)) = pk;
  }
}

__global__ void __launch_bounds__(TC_M) k_mlp_forward_tc(const MlpDev m, const float *feat,
                                                          long long n, float *out,
                                                          DevStatus *status) {
  __shared__ TcSmem S;
  const unsigned tmem = tc_setup(m, S);
  unsigned parity = 0;
  bool failed = false;
  const long long ntiles = (n + TC_M - 1) / TC_M;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long i = tile * TC_M + threadIdx.x;
    float f[MLP_K1];
#pragma unroll
    for (int k = 0; k < MLP_K1; ++k)
      f[k] = (i < n && k < m.nf) ? feat[i * m.nf + k] : 0.0f;
    tc_put_features(S, f);
    float y0, y1;
    if (!tc_forward(S, tmem, parity, y0, y1)) {
      failed = true;
      break;
    }
    if (i < n) {
      out[2 * i] = y0;
      out[2 * i + 1] = y1;
    }
  }
  tc_teardown(tmem, failed, status);
}

// The invariants and features of cell_invariants / mlp_features computed in
// FP32: the features are rounded to BF16 for the first layer and the guess
// only narrows the root finder's bracket (which the FP64 iteration checks),
// so FP32 is ample, and the FP64 divisions, roots and logarithms dominated
// the kernel.  q and s (for the decoded guess) come out as well.
struct InvF {
  float q, s;
};
AXB_D InvF features_fast(double dens_d, const double (&mom_d)[3], double tau_d, double DYe_d,
                         const double (&dB_d)[3], const sym3 &gd, int nf, float *f) {
  const float gxx = float(gd.xx), gxy = float(gd.xy), gxz = float(gd.xz),
              gyy = float(gd.yy), gyz = float(gd.yz), gzz = float(gd.zz);
  const float c00 = gyy * gzz - gyz * gyz, c01 = gxz * gyz - gxy * gzz,
              c02 = gxy * gyz - gxz * gyy;
  const float det = gxx * c00 + gxy * c01 + gxz * c02;
  const float idet = __frcp_rn(det);
  const float isq = rsqrtf(det);
  // the inverse metric (cofactors / det)
  const float uxx = c00 * idet, uxy = c01 * idet, uxz = c02 * idet,
              uyy = (gxx * gzz - gxz * gxz) * idet, uyz = (gxy * gxz - gxx * gyz) * idet,
              uzz = (gxx * gyy - gxy * gxy) * idet;
  const float D = float(dens_d) * isq;
  const float S[3] = {float(mom_d[0]) * isq, float(mom_d[1]) * isq, float(mom_d[2]) * isq};
  const float B[3] = {float(dB_d[0]) * isq, float(dB_d[1]) * isq, float(dB_d[2]) * isq};
  const float Ssq = S[0] * (uxx * S[0] + uxy * S[1] + uxz * S[2]) +
                    S[1] * (uxy * S[0] + uyy * S[1] + uyz * S[2]) +
                    S[2] * (uxz * S[0] + uyz * S[1] + uzz * S[2]);
  const float Bsq = B[0] * (gxx * B[0] + gxy * B[1] + gxz * B[2]) +
                    B[1] * (gxy * B[0] + gyy * B[1] + gyz * B[2]) +
                    B[2] * (gxz * B[0] + gyz * B[1] + gzz * B[2]);
  const float BS = B[0] * S[0] + B[1] * S[1] + B[2] * S[2];
  const float iD = __frcp_rn(D);
  const float qr = float(tau_d) * isq * iD, r = Ssq * iD * iD, sv = Bsq * iD,
              t = BS * iD * rsqrtf(D);
  const float q = fmaxf(qr, -0.999f);
  const float lq = log1pf(q);
  const float lr = log1pf(fmaxf(r, 0.0f));
  const float den = 1.0f + q + sv;
  const float iden = __frcp_rn(den);
  f[0] = __logf(fmaxf(D, 1e-37f)) * 0.1f;
  f[1] = lq;
  f[2] = 0.5f * lr;
  f[3] = log1pf(fmaxf(sv, 0.0f));
  f[4] = fminf(t * t / (r * sv + 1e-37f), 1.0f);
  f[5] = r * iden * iden;
  f[6] = sv * iden;
  f[7] = lq - 0.5f * lr;
  if (nf > 8)
    f[8] = float(DYe_d / dens_d);
  return InvF{qr, sv};
}

// The learned guess of independent cells, ahead of the recovery: x = h W
// placed by y0 in the Palenzuela scheme's initial bracket
// [max(1e-10, 1 + q - s), 2 + 2 q - s] (c2p_1DPalenzuela.hxx:395-398) and
// W = max(exp(y1), 1).
// the inputs of one cell, loaded a tile ahead
struct CellIn {
  double dens, tau, DYe, mom[3], dB[3];
  sym3 g;
};

// independent cells: the arrays of axb_cells
struct CellsSrc {
  axb_cells c;
  long long n;
  AXB_D void load(long long i, int nf, CellIn &x) const {
    x.dens = c.dens[i];
    x.tau = c.tau[i];
    x.DYe = nf > 8 ? c.DYe[i] : 0.0;
    for (int q = 0; q < 3; ++q) {
      x.mom[q] = c.mom[q][i];
      x.dB[q] = c.dB[q][i];
    }
    x.g = sym3{c.g[0][i], c.g[1][i], c.g[2][i], c.g[3][i], c.g[4][i], c.g[5][i]};
  }
};

// the interior cells of a box (MlpBoxIn)
struct BoxSrc {
  MlpBoxIn in;
  long long n;
  AXB_D void load(long long ci, int nf, CellIn &x) const {
    const BoxDev &b = in.b;
    const long long nxy = (long long)b.n[0] * b.n[1];
    const int k = int(ci / nxy);
    const long long r = ci - k * nxy;
    const int j = int(r / b.n[0]);
    const int i = int(r - (long long)j * b.n[0]);
    const long long I = b.at(i + b.ng, j + b.ng, k + b.ng);
    x.dens = in.dens[I];
    x.tau = in.tau[I];
    x.DYe = nf > 8 ? in.DYe[I] : 0.0;
    for (int q = 0; q < 3; ++q)
      x.mom[q] = in.mom[q][I];
    x.dB[0] = 0.5 * (in.dBstag[0][I] + in.dBstag[0][I + 1]);
    x.dB[1] = 0.5 * (in.dBstag[1][I] + in.dBstag[1][I + b.sy]);
    x.dB[2] = 0.5 * (in.dBstag[2][I] + in.dBstag[2][I + b.sz]);
    double gv[6];
    for (int q = 0; q < 6; ++q) {
      const double *f = in.g[q];
      gv[q] = (f[I] + f[I + 1] + f[I + b.sy] + f[I + 1 + b.sy] + f[I + b.sz] +
               f[I + 1 + b.sz] + f[I + b.sy + b.sz] + f[I + 1 + b.sy + b.sz]) *
              0.125;
    }
    x.g = sym3{gv[0], gv[1], gv[2], gv[3], gv[4], gv[5]};
  }
};

template <class Src>
__global__ void __launch_bounds__(TC_M) k_mlp_guess_tc(const Src src, const MlpDev m,
                                                        float2 *guess, DevStatus *status) {
  __shared__ TcSmem S;
  const unsigned tmem = tc_setup(m, S);
  unsigned parity = 0;
  bool failed = false;
  const long long ntiles = (src.n + TC_M - 1) / TC_M;
  // the next tile's inputs are loaded before this tile's layers run, so
  // their latency hides behind the tensor-core chain
  CellIn cur{};
  {
    const long long i0 = (long long)blockIdx.x * TC_M + threadIdx.x;
    if (blockIdx.x < ntiles && i0 < src.n)
      src.load(i0, m.nf, cur);
  }
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long i = tile * TC_M + threadIdx.x;
    const bool valid = i < src.n;
    float f[MLP_K1];
#pragma unroll
    for (int k = 0; k < MLP_K1; ++k)
      f[k] = 0.0f;
    InvF inv{0.0f, 0.0f};
    if (valid)
      inv = features_fast(cur.dens, cur.mom, cur.tau, cur.DYe, cur.dB, cur.g, m.nf, f);
    const long long inext = (tile + gridDim.x) * TC_M + threadIdx.x;
    if (tile + gridDim.x < ntiles && inext < src.n)
      src.load(inext, m.nf, cur);
    tc_put_features(S, f);
    float y0, y1;
    if (!tc_forward(S, tmem, parity, y0, y1)) {
      failed = true;
      break;
    }
    if (valid) {
      const double q = inv.q, sv = inv.s;
      const double lo = fmax(1e-10, 1.0 + q - sv), hi = 2.0 + 2.0 * q - sv;
      guess[i] = make_float2(float(lo + double(y0) * (hi - lo)), fmaxf(__expf(y1), 1.0f));
    }
  }
  tc_teardown(tmem, failed, status);
}

int tc_blocks(long long n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // 5 CTAs per SM fit the shared memory (42 KB each) and tensor memory
  // (5 x 64 of 512 columns); persistent beyond that
  const long long tiles = (n + TC_M - 1) / TC_M;
  return int(tiles < 5LL * sms ? tiles : 5LL * sms);
}

} // namespace

int launch_mlp_forward_tc(const MlpDev &m, const float *feat, long long n, float *out,
                          DevStatus *status, cudaStream_t s) {
  const int blocks = tc_blocks(n);
  if (blocks < 1)
    return AXB_OK;
  k_mlp_forward_tc<<<blocks, TC_M, 0, s>>>(m, feat, n, out, status);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

int launch_mlp_guess_tc(const axb_cells &c, const MlpDev &m, float2 *guess, DevStatus *status,
                        cudaStream_t s) {
  const int blocks = tc_blocks(c.n);
  if (blocks < 1)
    return AXB_OK;
  k_mlp_guess_tc<<<blocks, TC_M, 0, s>>>(CellsSrc{c, c.n}, m, guess, status);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

int launch_mlp_guess_box_tc(const MlpBoxIn &in, const MlpDev &m, float2 *guess,
                            DevStatus *status, cudaStream_t s) {
  const long long n = (long long)in.b.n[0] * in.b.n[1] * in.b.n[2];
  const int blocks = tc_blocks(n);
  if (blocks < 1)
    return AXB_OK;
  k_mlp_guess_tc<<<blocks, TC_M, 0, s>>>(BoxSrc{in, n}, m, guess, status);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

} // namespace axb
