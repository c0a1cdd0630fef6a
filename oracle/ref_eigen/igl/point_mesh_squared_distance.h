// See marching_cubes.h. TEST INFRASTRUCTURE ONLY.
#pragma once
#include <stdexcept>
namespace igl {
template <typename... A> inline void point_mesh_squared_distance(A&&...) {
    throw std::logic_error("igl::point_mesh_squared_distance is not part of this harness");
}
}  // namespace igl
