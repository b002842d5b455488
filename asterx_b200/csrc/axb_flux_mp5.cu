// k_flux_pass instantiations for the mp5 reconstruction.
#include "axb_flux_launch.cuh"
namespace axb {
int launch_flux_mp5(int dir, const RhsArgs &a, const axb_eos &eos, int seglen,
                   cudaStream_t s) {
  return launch_flux_pass_t<AXB_RECON_MP5>(dir, a, eos, seglen, s);
}
} // namespace axb
