// Test infrastructure: the subset of GLM's vec3 that the reference's sources use
// (include/common/dom_types.h:78-79, src/common/kernel/predict.cu:33-34,
// ego_motion_compensation.cu:14-16, init_new_particles.cu:101-102). GLM is not installed here.
#pragma once
namespace glm {
struct vec3 {
    float x, y, z;
    __host__ __device__ vec3() : x(0.f), y(0.f), z(0.f) {}
    __host__ __device__ vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    __host__ __device__ float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    __host__ __device__ const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    __host__ __device__ vec3& operator+=(const vec3& o) {
        x += o.x;
        y += o.y;
        z += o.z;
        return *this;
    }
};
__host__ __device__ inline vec3 operator*(const vec3& v, float s) { return vec3(v.x * s, v.y * s, v.z * s); }
__host__ __device__ inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
}  // namespace glm
