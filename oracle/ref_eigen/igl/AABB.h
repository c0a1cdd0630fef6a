// See marching_cubes.h. TEST INFRASTRUCTURE ONLY.
#pragma once
#include <stdexcept>
namespace igl {
template <typename DerivedV, int DIM>
class AABB {
public:
    template <typename... A> void init(A&&...) { throw std::logic_error("igl::AABB is not part of this harness"); }
    template <typename... A> double squared_distance(A&&...) const {
        throw std::logic_error("igl::AABB is not part of this harness");
    }
};
}  // namespace igl
