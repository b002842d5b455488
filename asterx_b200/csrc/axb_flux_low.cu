// k_flux_pass instantiations for the low-order reconstructions (Godunov,
// minmod, monocentral).
#include "axb_flux_launch.cuh"
namespace axb {
int launch_flux_low(int recon, int dir, const RhsArgs &a, const axb_eos &eos,
                    int seglen, cudaStream_t s) {
  switch (recon) {
  case AXB_RECON_GODUNOV:
    return launch_flux_pass_t<AXB_RECON_GODUNOV>(dir, a, eos, seglen, s);
  case AXB_RECON_MINMOD:
    return launch_flux_pass_t<AXB_RECON_MINMOD>(dir, a, eos, seglen, s);
  case AXB_RECON_MONOCENTRAL:
    return launch_flux_pass_t<AXB_RECON_MONOCENTRAL>(dir, a, eos, seglen, s);
  }
  return AXB_ERR_UNSUPPORTED;
}
int launch_flux_batch_low(int recon, int dir, const RhsArgs *args, const TileTable &t,
                          unsigned long long *ctr, const axb_eos &eos, DevStatus *st,
                          int seglen, int nblocks, cudaStream_t s) {
  switch (recon) {
  case AXB_RECON_GODUNOV:
    return launch_flux_batch_t<AXB_RECON_GODUNOV>(dir, args, t, ctr, eos, st, seglen, nblocks, s);
  case AXB_RECON_MINMOD:
    return launch_flux_batch_t<AXB_RECON_MINMOD>(dir, args, t, ctr, eos, st, seglen, nblocks, s);
  case AXB_RECON_MONOCENTRAL:
    return launch_flux_batch_t<AXB_RECON_MONOCENTRAL>(dir, args, t, ctr, eos, st, seglen, nblocks,
                                                      s);
  }
  return AXB_ERR_UNSUPPORTED;
}
} // namespace axb
