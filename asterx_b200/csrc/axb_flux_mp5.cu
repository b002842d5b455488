// k_flux_pass instantiations for the mp5 reconstruction.
#include "axb_flux_launch.cuh"
namespace axb {
int launch_flux_mp5(int dir, const RhsArgs &a, const axb_eos &eos, int seglen,
                   cudaStream_t s) {
  return launch_flux_pass_t<AXB_RECON_MP5>(dir, a, eos, seglen, s);
}
int launch_flux_batch_mp5(int dir, const RhsArgs *args, const TileTable &t,
                          unsigned long long *ctr, const axb_eos &eos, DevStatus *st,
                          int seglen, int nblocks, cudaStream_t s) {
  return launch_flux_batch_t<AXB_RECON_MP5>(dir, args, t, ctr, eos, st, seglen, nblocks, s);
}
} // namespace axb
