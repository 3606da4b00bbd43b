// Stand-in for ViennaGrid's forwards.hpp (ViennaGrid is not part of the viennashe-dev tree), so
// that the reference's own headers compile for the oracle's pinning library (oracle/_ref) and for
// the drop-in adapter's test harness: the names viennashe/forwards.h uses (:70, :78, :85) and the
// mesh element traits the scattering models name (she/scattering/common.hpp:82-87), with the
// standard headers the real one brings in.  Test infrastructure only.
#ifndef VSHE_REF_STUB_VIENNAGRID_FORWARDS
#define VSHE_REF_STUB_VIENNAGRID_FORWARDS
#include <iostream>
#include <vector>
namespace viennagrid {
template <int N> struct simplex_tag {};
template <int N> struct hypercube_tag {};
namespace result_of {
template <typename MeshT> struct cell_tag { typedef void type; };
template <typename MeshT> struct point { typedef double type; };
template <typename MeshT> struct vertex { struct type {}; };
template <typename MeshT> struct facet { struct type {}; };
template <typename MeshT> struct cell { struct type {}; };
}  // namespace result_of
}  // namespace viennagrid
#endif
