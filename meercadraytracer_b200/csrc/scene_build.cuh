// GPU scene compilation: binned-SAH BVH build and the geometry compile step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mcrt {

// Device buffers reused across builds.
struct BuildBuffers;

class SceneBuilder {
 public:
  SceneBuilder();
  ~SceneBuilder();
  SceneBuilder(const SceneBuilder&) = delete;
  SceneBuilder& operator=(const SceneBuilder&) = delete;

  // buildBvh on device arrays: d_tris holds 9 floats per triangle; d_bounds /
  // d_nodes / d_order are sized for max(1, 2n - 1) nodes and n triangles.
  // Returns the node count. Throws on CUDA errors (caught at the ABI).
  int build_device(const float* d_tris, int n, float* d_bounds, int* d_nodes, uint32_t* d_order, cudaStream_t s);

  // buildBvh from and to host arrays.
  int build_bvh_host(const float* tris, int n, float* bounds, int* nodes, uint32_t* order, cudaStream_t s);

  // compileGeometry after the flatten, from and to host arrays.
  void compile_host(int n, const double* p, const double* nrm, const double* uv, const double* colors,
                    const uint8_t* has_color, const uint32_t* materials, const uint8_t* flags, const uint8_t* sides,
                    float* triangles_out, float* normals_out, float* uvs_out, float* tangents_out, float* colors_out,
                    uint32_t* materials_out, uint8_t* flags_out, uint8_t* sides_out, float* bounds_out,
                    int* nodes_out, uint32_t* order_out, int* node_count_out, double* epsilon_out, int* any_colors,
                    cudaStream_t s);

  // Levels of the last build (for tests and benchmarks).
  int last_levels() const { return last_levels_; }

 private:
  BuildBuffers* b_;
  int last_levels_ = 0;
};

}  // namespace mcrt
