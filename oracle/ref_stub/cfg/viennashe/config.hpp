// Stand-in for viennashe/config.hpp in the oracle's pinning library (oracle/_ref): the real one
// pulls in the simulator's quantities and with them ViennaGrid's meshes.  The scattering models
// read only conf.scattering() (she/scattering/*_phonon_scattering.hpp constructors), which this
// container provides with the reference's own parameter class (she/scattering/config.hpp).
// Test infrastructure only.
#ifndef VSHE_REF_STUB_CONFIG
#define VSHE_REF_STUB_CONFIG
#include "viennashe/forwards.h"
#include "viennashe/she/scattering/config.hpp"
namespace viennashe {
class config {
 public:
  she::scatter_config const &scattering() const { return scatter_; }

 private:
  she::scatter_config scatter_;
};
}  // namespace viennashe
#endif
