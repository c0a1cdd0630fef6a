// Stand-in declarations for the libigl v2.6.0 calls the reference's CPU sources name outside the
// dual-contouring path (marching cubes, closest points on a mesh, the AABB tree: used by the
// refinement method and the viewer). TEST INFRASTRUCTURE ONLY: they throw if ever called.
#pragma once
#include <stdexcept>
namespace igl {
template <typename... A> inline void marching_cubes(A&&...) {
    throw std::logic_error("igl::marching_cubes is not part of this harness");
}
}  // namespace igl
