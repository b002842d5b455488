// Learned-guess network on the 5th-generation tensor cores (tcgen05).
//
// One CTA of 128 threads evaluates tiles of 128 cells: thread t owns row t
// (cell t of the tile).  Per layer, one elected thread issues the
// 128 x N x K product as K/16 `tcgen05.mma.cta_group::1.kind::f16`
// instructions (BF16 operands in shared memory, FP32 accumulator in tensor
// memory), commits it to an mbarrier, and every thread then reads its row of
// the accumulator back with `tcgen05.ld.32x32b` (warp w owns TMEM lanes
// 32w..32w+31), adds the bias, applies the activation, rounds to BF16 and
// stores the row as the next layer's A operand.
//
// Operands use the canonical K-major layout without swizzle: 8 x 8 core
// matrices of 8 rows x 16 bytes; element (r, k) of an R x K operand sits at
// byte (r/8) * 16K + (k/8) * 128 + (r%8) * 16 + (k%8) * 2, so the leading
// byte offset (next core matrix along K) is 128 and the stride byte offset
// (next 8 rows) is 16K.  One K = 16 step covers two core matrices along K.
//
// The network and its numerics are those of the warp-level path in
// axb_mlp.cuh (BF16 weights and activations, FP32 accumulation); the bias is
// added after the products instead of seeding the accumulator, and the
// products are summed in the tensor core's order, so outputs agree with it
// to FP32 rounding.  Every wait on the mbarrier is bounded: on a timeout the
// CTA sets AXB_EW_MMA_TIMEOUT, releases its tensor memory and returns.
#include <cuda_bf16.h>

#include "axb_internal.hxx"
#include "axb_mlp.cuh"

namespace axb {
namespace {

constexpr int TC_M = 128;    // cells per tile = rows of every product
constexpr int TC_COLS = 64;  // tensor-memory columns: one 128 x 64 FP32 accumulator
constexpr int TC_N4 = 16;    // output layer padded to the smallest N for M = 128
constexpr long long TC_WAIT_LIMIT = 1LL << 22; // mbarrier polls before giving up

// byte offset of element (r, k) of an R x K operand (canonical K-major)
AXB_HD constexpr unsigned kmaj(int r, int k, int K) {
  return unsigned((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

struct __align__(128) TcSmem {
  __nv_bfloat16 w1[MLP_H * MLP_K1]; // B of layer 1: N = 64 x K = 16
  __nv_bfloat16 w2[MLP_H * MLP_H];  // N = 64 x K = 64
  __nv_bfloat16 w3[MLP_H * MLP_H];
  __nv_bfloat16 w4[TC_N4 * MLP_H];  // N = 16 x K = 64, rows 2..15 zero
  __nv_bfloat16 a1[TC_M * MLP_K1];  // features of the tile
  __nv_bfloat16 ah[TC_M * MLP_H];   // hidden activations of the tile
  float b1[MLP_H], b2[MLP_H], b3[MLP_H], b4[2];
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

// Stage the network's weights in the canonical operand layout (all threads;
// a barrier must follow).
AXB_D void tc_stage(const MlpDev &m, TcSmem &S) {
  const int t = threadIdx.x, nt = blockDim.x;
  char *w1 = reinterpret_cast<char *>(S.w1), *w2 = reinterpret_cast<char *>(S.w2),
       *w3 = reinterpret_cast<char *>(S.w3), *w4 = reinterpret_cast<char *>(S.w4);
  for (int e = t; e < MLP_H * MLP_K1; e += nt)
    *reinterpret_cast<__nv_bfloat16 *>(w1 + kmaj(e / MLP_K1, e % MLP_K1, MLP_K1)) = m.w1[e];
  for (int e = t; e < MLP_H * MLP_H; e += nt) {
    *reinterpret_cast<__nv_bfloat16 *>(w2 + kmaj(e / MLP_H, e % MLP_H, MLP_H)) = m.w2[e];
    *reinterpret_cast<__nv_bfloat16 *>(w3 + kmaj(e / MLP_H, e % MLP_H, MLP_H)) = m.w3[e];
  }
  for (int e = t; e < TC_N4 * MLP_H; e += nt) {
    const int n = e / MLP_H, k = e % MLP_H;
    *reinterpret_cast<__nv_bfloat16 *>(w4 + kmaj(n, k, MLP_H)) =
        n < 2 ? m.w4[n * MLP_H + k] : __float2bfloat16(0.0f);
  }
  for (int e = t; e < MLP_H; e += nt) {
    S.b1[e] = m.b1[e];
    S.b2[e] = m.b2[e];
    S.b3[e] = m.b3[e];
  }
  if (t < 2)
    S.b4[t] = m.b4[t];
  if (t == 0)
    S.act = m.act;
}

// One layer's product into tensor memory: thread 0 issues K/16 MMAs and the
// commit; every thread waits for the result.  Returns false on a timeout.
AXB_D bool tc_layer(const TcSmem &S, const void *A, const void *B, int K, int N, unsigned tmem,
                    unsigned &parity) {
  const unsigned bar = smem_u32(&S.bar);
  if (threadIdx.x == 0) {
    fence_after_sync();
    const unsigned sbo = unsigned(K * 16);
    const unsigned id = idesc_bf16(N);
    for (int kk = 0; kk < K / 16; ++kk)
      umma(tmem, smem_desc(static_cast<const char *>(A) + kk * 256, sbo),
           smem_desc(static_cast<const char *>(B) + kk * 256, sbo), id, kk > 0);
    umma_commit(bar);
  }
  const bool ok = mbar_wait(bar, parity);
  parity ^= 1u;
  fence_after_sync();
  return ok;
}

// This thread's row of a 64-column accumulator + bias, activated, rounded to
// BF16 and stored as row `r` of the hidden operand.
AXB_D void tc_hidden_out(TcSmem &S, unsigned trow, const float *bias, int r) {
  char *ah = reinterpret_cast<char *>(S.ah);
#pragma unroll
  for (int c16 = 0; c16 < MLP_H / 16; ++c16) {
    float v[16];
    tmem_ld16(trow + unsigned(c16 * 16), v);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint4 pk;
      unsigned *p = reinterpret_cast<unsigned *>(&pk);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = c16 * 16 + h * 8 + 2 * q;
        p[q] = pack_bf16x2(mlp_act(v[h * 8 + 2 * q] + bias[j], S.act),
                           mlp_act(v[h * 8 + 2 * q + 1] + bias[j + 1], S.act));
      }
      *reinterpret_cast<uint4 *>(ah + kmaj(r, c16 * 16 + h * 8, MLP_H)) = pk;
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
  bool ok = tc_layer(S, S.a1, S.w1, MLP_K1, MLP_H, tmem, parity);
  if (__syncthreads_or(!ok))
    return false;
  const float *bias[3] = {S.b1, S.b2, S.b3};
  const __nv_bfloat16 *w[2] = {S.w2, S.w3};
  for (int l = 0; l < 3; ++l) {
    tc_hidden_out(S, trow, bias[l], r);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    ok = tc_layer(S, S.ah, l < 2 ? static_cast<const void *>(w[l]) : S.w4, MLP_H,
                  l < 2 ? MLP_H : TC_N4, tmem, parity);
    if (__syncthreads_or(!ok))
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
AXB_D void tc_put_features(TcSmem &S, const float (&f)[MLP_K1]) {
  char *a1 = reinterpret_cast<char *>(S.a1);
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

// The learned guess of independent cells (x = h W and W per cell, decoded as
// mlp_cell_guess decodes it), ahead of the recovery.
__global__ void __launch_bounds__(TC_M) k_mlp_guess_tc(const axb_cells c, const MlpDev m,
                                                        float2 *guess, DevStatus *status) {
  __shared__ TcSmem S;
  const unsigned tmem = tc_setup(m, S);
  unsigned parity = 0;
  bool failed = false;
  const long long ntiles = (c.n + TC_M - 1) / TC_M;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long i = tile * TC_M + threadIdx.x;
    const bool valid = i < c.n;
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
      mlp_features(inv, m.nf, f);
    }
    tc_put_features(S, f);
    float y0, y1;
    if (!tc_forward(S, tmem, parity, y0, y1)) {
      failed = true;
      break;
    }
    if (valid) {
      const double lo = fmax(1e-10, 1.0 + inv.q - inv.s), hi = 2.0 + 2.0 * inv.q - inv.s;
      guess[i] = make_float2(float(lo + double(y0) * (hi - lo)),
                             float(fmax(exp(double(y1)), 1.0)));
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
  k_mlp_guess_tc<<<blocks, TC_M, 0, s>>>(c, m, guess, status);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

} // namespace axb
