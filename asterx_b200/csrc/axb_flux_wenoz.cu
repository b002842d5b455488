// k_flux_pass instantiations for the wenoz reconstruction.
#include "axb_flux_launch.cuh"
namespace axb {
int launch_flux_wenoz(int dir, const RhsArgs &a, const axb_eos &eos, int seglen,
                   cudaStream_t s) {
  return launch_flux_pass_t<AXB_RECON_WENOZ>(dir, a, eos, seglen, s);
}
} // namespace axb
