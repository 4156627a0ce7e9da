// GPU scene compilation: binned-SAH BVH build and the geometry compile step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mcrt {

// Device buffers reused across builds.
struct BuildBuffers;

// A mesh of instanced geometry, as host arrays (three.js BufferGeometry
// attributes): 3 floats per vertex position (and normal), 2 per uv.
struct MeshInput {
  int vertex_count;
  const float* position;
  const float* normal;    // or nullptr: face normals
  const float* uv;        // or nullptr: zeros
  int index_count;        // 0: not indexed
  const uint32_t* index;
};

// One instance: a mesh under a column-major world matrix, with the words every
// one of its triangles gets.
struct InstanceInput {
  double world[16];
  int mesh;
  uint32_t material;
  int flags, side, flat_shading;
};

// A compiled geometry left in the builder's device buffers (CompiledGeometry
// layout, BVH order), valid until the next build.
struct DeviceGeometry {
  int n, node_count, root_count, levels;
  double epsilon;
  const float *triangles, *normals, *uvs, *tangents, *bounds;
  const uint32_t *materials, *order;
  const uint8_t *flags, *sides;
  const int* nodes;
};

class SceneBuilder {
 public:
  SceneBuilder();
  ~SceneBuilder();
  SceneBuilder(const SceneBuilder&) = delete;
  SceneBuilder& operator=(const SceneBuilder&) = delete;

  // buildBvh on device arrays: d_tris holds 9 floats per triangle; d_bounds /
  // d_nodes / d_order are sized for max(1, 2n - 1) nodes and n triangles.
  // Returns the node count. Throws on CUDA errors (caught at the ABI).
  // `bins`: SAH bins per axis (the reference's 16; at most 32).
  int build_device(const float* d_tris, int n, float* d_bounds, int* d_nodes, uint32_t* d_order, cudaStream_t s,
                   int bins = 16);

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

  // Meshes for compile_instances, kept on the device until replaced.
  void upload_meshes(int count, const MeshInput* meshes, cudaStream_t s);
  // Triangles the instances make (-1 if one names no uploaded mesh).
  long long instance_triangles(int count, const InstanceInput* inst) const;
  // compileGeometry of the instances entirely on the device: the flatten of
  // addMesh (src/compile.ts:212-306), the BVH with `bins` bins, the reorder,
  // tangents and epsilon. times_ms (3 floats, or null): flatten, build, finish.
  void compile_instances(int count, const InstanceInput* inst, int bins, cudaStream_t s, DeviceGeometry* out,
                         float* times_ms);
  // Device memory the builder holds between builds.
  size_t device_bytes() const;

 private:
  BuildBuffers* b_;
  int last_levels_ = 0;
};

// Exclusive prefix sums of `in` into `out` (n ints) on stream `s`, with the
// builder's two-kernel scan; `sums` is scratch of exclusive_scan_scratch()
// ints.
void exclusive_scan(const int* in, int* out, int n, int* sums, cudaStream_t s);
int exclusive_scan_scratch();

}  // namespace mcrt
