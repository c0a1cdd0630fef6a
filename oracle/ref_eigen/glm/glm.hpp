// Stand-in for the one GLM type the reference's viewer code names (glm::vec3 colours).
// TEST INFRASTRUCTURE ONLY.
#pragma once
namespace glm {
struct vec3 {
    float x = 0, y = 0, z = 0;
    vec3() = default;
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};
}  // namespace glm
