// Launch helper for k_flux_pass, instantiated per reconstruction scheme in
// its own translation unit (axb_flux_<scheme>.cu) to keep builds parallel.
#pragma once

#include "axb_internal.hxx"
#include "axb_rhs_kernels.cuh"

namespace axb {

template <int RECON, class EOS>
int launch_flux_pass_eos(int dir, const RhsArgs &a, const EOS &eos, int seglen,
                         cudaStream_t s) {
  const BoxDev &b = a.b;
  if (dir == 0) {
    // one warp per (y, z) row of the transverse range [ng-1, ng+n]^2
    const long long warps = (long long)(b.n[1] + 2) * (b.n[2] + 2);
    const long long blocks = (warps * 32 + 127) / 128;
    if (blocks > 0x7fffffffLL)
      return AXB_ERR_TOO_LARGE;
    k_flux_x<RECON, EOS><<<(unsigned)blocks, 128, 0, s>>>(a, eos);
    return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
  }
  const int T0 = 0, T1 = dir == 2 ? 1 : 2;
  const dim3 block(32, 4);
  const dim3 grid((b.n[T0] + 2 + 31) / 32, (b.n[T1] + 2 + 3) / 4,
                  (b.n[dir] + seglen - 1) / seglen);
  if (dir == 1)
    k_flux_pass<1, RECON, EOS><<<grid, block, 0, s>>>(a, eos, seglen);
  else
    k_flux_pass<2, RECON, EOS><<<grid, block, 0, s>>>(a, eos, seglen);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
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

int launch_flux_ppm(int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);
int launch_flux_wenoz(int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);
int launch_flux_mp5(int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);
int launch_flux_low(int recon, int dir, const RhsArgs &a, const axb_eos &eos, int seglen, cudaStream_t s);

} // namespace axb
