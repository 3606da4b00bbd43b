// Stand-in for ViennaGrid's forwards.hpp (ViennaGrid is not part of the viennashe-dev tree):
// the three names viennashe/forwards.h uses (:70, :78, :85) and the standard headers the real
// one brings in, so that the reference's own headers the drop-in adapter includes compile.
// Test infrastructure only.
#ifndef VSHE_TEST_VIENNAGRID_FORWARDS_STUB
#define VSHE_TEST_VIENNAGRID_FORWARDS_STUB
#include <iostream>
#include <vector>
namespace viennagrid {
template <int N> struct simplex_tag {};
template <int N> struct hypercube_tag {};
namespace result_of {
template <typename MeshT> struct cell_tag { typedef void type; };
}  // namespace result_of
}  // namespace viennagrid
#endif
