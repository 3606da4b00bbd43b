// ref_physics.cpp -- TEST INFRASTRUCTURE, not product code.
//
// The reference's own scalar physics, compiled from its headers where they lie (oracle/build_ref.sh,
// into oracle/_ref, never committed): the Modena dispersion (viennashe/physics/dispersion.hpp:207-286)
// for silicon electrons (materials/all.hpp), the equilibrium helpers of viennashe/physics/physics.hpp,
// and the acoustic and optical phonon scattering models (she/scattering/acoustic_phonon_scattering.hpp,
// optical_phonon_scattering.hpp) with their default parameters (she/scattering/config.hpp), evaluated
// through a stand-in device that reports the lattice temperature.  tests/test_oracle_ref.py pins the
// oracle's restatement (she_oracle.cpp vsheo_physics_probe) to it; the probe numbering is shared.
#include "viennashe/config.hpp"
#include "viennashe/physics/dispersion.hpp"
#include "viennashe/physics/physics.hpp"
#include "viennashe/she/scattering/acoustic_phonon_scattering.hpp"
#include "viennashe/she/scattering/optical_phonon_scattering.hpp"

namespace {
struct StandInMesh {};
struct StandInDevice {
  typedef StandInMesh mesh_type;
  double T;
  template <typename E> double get_lattice_temperature(E const &) const { return T; }
};
}  // namespace

extern "C" {

// what: 0 DOS(in[0]); 1 velocity(in[0]); 2 optical phonon number(in[0] energy, in[1] T);
// 3 built-in potential(in[0] T, in[1] N_D, in[2] N_A); 4 ohmic contact electron density(T, N_D,
// N_A); 5 acoustic phonon rate(in[0] T); 6 optical phonon processes(in[0] grid spacing, in[1] T,
// in[2] kinetic energy) -> out[0..3] rates of the four processes, out[4] the snapped phonon energy
// (final energy of the emission minus the initial one); 7 band weight(in[0] T).
int vsheref_physics_probe(int what, const double *in, double *out) {
  using namespace viennashe;
  physics::modena_dispersion<materials::si> disp(ELECTRON_TYPE_ID);
  switch (what) {
    case 0: out[0] = disp.density_of_states(in[0]); return 0;
    case 1: out[0] = disp.velocity(in[0]); return 0;
    case 2: out[0] = physics::get_optical_phonon_number(in[0], in[1]); return 0;
    case 3: out[0] = physics::built_in_potential(in[0], in[1], in[2]); return 0;
    case 4: out[0] = physics::contact_carrier_ohm(in[0], in[1], in[2], ELECTRON_TYPE_ID); return 0;
    case 5: {
      config conf;
      StandInDevice dev{in[0]};
      she::acoustic_phonon_scattering<StandInDevice> ac(dev, conf);
      viennagrid::result_of::cell<StandInMesh>::type c;
      out[0] = ac(c, 1e-20, ELECTRON_TYPE_ID)[0].rate();
      return 0;
    }
    case 6: {
      config conf;
      StandInDevice dev{in[1]};
      she::optical_phonon_scattering<StandInDevice> op(dev, conf, in[0]);
      viennagrid::result_of::cell<StandInMesh>::type c;
      const auto r = op(c, in[2], ELECTRON_TYPE_ID);
      for (int k = 0; k < 4; ++k) out[k] = r[size_t(k)].rate();
      out[4] = r[0].initial_energy() - r[0].final_energy();
      return 0;
    }
    case 7: out[0] = physics::get_band_weight(in[0], ELECTRON_TYPE_ID); return 0;
  }
  return -1;
}

}  // extern "C"
