// Launch helper for k_flux_pass, instantiated per reconstruction scheme in
// its own translation unit (axb_flux_<scheme>.cu) to keep builds parallel.
#pragma once

#include "axb_batch.cuh"
#include "axb_internal.hxx"
#include "axb_rhs_kernels.cuh"

namespace axb {

template <int RECON, class EOS, bool UCT>
int launch_flux_pass_uct(int dir, const RhsArgs &a, const EOS &eos, int seglen,
                         cudaStream_t s) {
  const BoxDev &b = a.b;
  if (dir == 0) {
    // one warp per (y, z) row of the transverse range [ng-te, ng+n+te-1]^2
    const long long warps = (long long)(b.n[1] + 2 * a.text) * (b.n[2] + 2 * a.text);
    const long long blocks = (warps * 32 + 127) / 128;
    if (blocks > 0x7fffffffLL)
      return AXB_ERR_TOO_LARGE;
    k_flux_x<RECON, EOS, UCT><<<(unsigned)blocks, 128, 0, s>>>(a, eos);
    return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
  }
  const int T0 = 0, T1 = dir == 2 ? 1 : 2;
  const dim3 block(32, 4);
  // Thread layout: 32 columns x 4 rows of the transverse plane per block,
  // or the plane walked row after row (no lane idle on the n+2-wide rows).
  // Measured at 256^3: the packed walk is 7-9 % faster for WENO-Z and PPM,
  // while MP5 is 30 % faster on the 32 x 4 blocks (each block's four rows
  // share the face metric's second vertex row in L1).
  constexpr bool packed = RECON != AXB_RECON_MP5;
  if (!packed) {
    const dim3 grid((b.n[T0] + 2 * a.text + 31) / 32, (b.n[T1] + 2 * a.text + 3) / 4,
                    (b.n[dir] + seglen - 1) / seglen);
    if (dir == 1)
      k_flux_pass<1, RECON, EOS, UCT><<<grid, block, 0, s>>>(a, eos, seglen);
    else
      k_flux_pass<2, RECON, EOS, UCT><<<grid, block, 0, s>>>(a, eos, seglen);
    return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
  }
  // the threads walk the transverse plane [ng-1, ng+n]^2 row after row
  // (as in the batched kernels), so the 2 extra columns of the plane do
  // not leave most of a warp idle
  RhsArgs ap = a;
  ap.b.packed = 1;
  const long long plane = (long long)(b.n[T0] + 2 * a.text) * (b.n[T1] + 2 * a.text);
  const dim3 grid(unsigned((plane + 127) / 128), 1, (b.n[dir] + seglen - 1) / seglen);
  if (dir == 1)
    k_flux_pass<1, RECON, EOS, UCT><<<grid, block, 0, s>>>(ap, eos, seglen);
  else
    k_flux_pass<2, RECON, EOS, UCT><<<grid, block, 0, s>>>(ap, eos, seglen);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

// the upwind-CT face data and the wider transverse range are a separate
// instantiation, so the flux-CT passes carry none of it
template <int RECON, class EOS>
int launch_flux_pass_eos(int dir, const RhsArgs &a, const EOS &eos, int seglen,
                         cudaStream_t s) {
  if (a.use_uct)
    return launch_flux_pass_uct<RECON, EOS, true>(dir, a, eos, seglen, s);
  return launch_flux_pass_uct<RECON, EOS, false>(dir, a, eos, seglen, s);
}

template <int RECON>
int launch_flux_pass_t(int dir, const RhsArgs &a, const axb_eos &eos,
                       int seglen, cudaStream_t s) {
  if (eos.kind == 0)
    return launch_flux_pass_eos<RECON>(dir, a, eos.ideal, seglen, s);
  if (eos.kind == 1)
    return launch_flux_pass_eos<RECON>(dir, a, tab_for_launch(eos, a.status), seglen, s);
  return AXB_ERR_UNSUPPORTED;
}

// Batched flux passes over the boxes of a batch (tile tables built by the
// batch with the grids of launch_flux_pass_eos).
template <int DIR, int RECON, class EOS>
__global__ void __launch_bounds__(128, AXB_FLUX_MINB)
    k_flux_pass_batch(const RhsArgs *args, const TileTable t, unsigned long long *ctr, const EOS eos, const int seglen) {
  batch_loop(args, t, ctr, [&](const RhsArgs &a, const uint3 bid) {
    flux_pass_body<DIR, RECON, EOS>(a, eos, seglen, bid);
  });
}

template <int RECON, class EOS>
__global__ void __launch_bounds__(128, AXB_FLUX_X_MINB)
    k_flux_x_batch(const RhsArgs *args, const TileTable t, unsigned long long *ctr, const EOS eos) {
  batch_loop(args, t, ctr, [&](const RhsArgs &a, const uint3 bid) {
    flux_x_body<RECON, EOS>(a, eos, bid);
  });
}

template <int RECON, class EOS>
int launch_flux_batch_eos(int dir, const RhsArgs *args, const TileTable &t,
                          unsigned long long *ctr, const EOS &eos, int seglen, int nblocks,
                          cudaStream_t s) {
  if (t.total == 0)
    return AXB_OK;
  if (dir == 0)
    k_flux_x_batch<RECON, EOS><<<nblocks, 128, 0, s>>>(args, t, ctr, eos);
  else if (dir == 1)
    k_flux_pass_batch<1, RECON, EOS><<<nblocks, dim3(32, 4), 0, s>>>(args, t, ctr, eos, seglen);
  else
    k_flux_pass_batch<2, RECON, EOS><<<nblocks, dim3(32, 4), 0, s>>>(args, t, ctr, eos, seglen);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

template <int RECON>
int launch_flux_batch_t(int dir, const RhsArgs *args, const TileTable &t,
                        unsigned long long *ctr, const axb_eos &eos, DevStatus *status,
                        int seglen, int nblocks, cudaStream_t s) {
  if (eos.kind == 0)
    return launch_flux_batch_eos<RECON>(dir, args, t, ctr, eos.ideal, seglen, nblocks, s);
  if (eos.kind == 1)
    return launch_flux_batch_eos<RECON>(dir, args, t, ctr, tab_for_launch(eos, status), seglen,
                                        nblocks, s);
  return AXB_ERR_UNSUPPORTED;
}

int launch_flux_batch(int recon, int dir, const RhsArgs *args, const TileTable &t,
                      unsigned long long *ctr, const axb_eos &eos, DevStatus *status,
                      int seglen, int nblocks, cudaStream_t s);

int launch_flux_ppm(int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);
int launch_flux_wenoz(int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);
int launch_flux_mp5(int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);
int launch_flux_low(int recon, int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);

} // namespace axb
