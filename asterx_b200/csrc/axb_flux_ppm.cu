// k_flux_pass instantiations for the ppm reconstruction.
#include "axb_flux_launch.cuh"
namespace axb {
int launch_flux_ppm(int dir, const RhsArgs &a, const axb_eos &eos, int seglen,
                   cudaStream_t s) {
  return launch_flux_pass_t<AXB_RECON_PPM>(dir, a, eos, seglen, s);
}
} // namespace axb
