// Internal declarations shared by the host builder and the CUDA side of
// libpfxtrace.  Not part of the C ABI.
#pragma once
#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfxt.h"
#include "pfxt_math.h"
#include "pfxt_types.h"

#define PFXT_PI_F 3.14159265358979323846f

namespace pfxt {

struct Invalid : std::runtime_error {
  explicit Invalid(const std::string& m) : std::runtime_error(m) {}
};
struct Refused : std::runtime_error {
  explicit Refused(const std::string& m) : std::runtime_error(m) {}
};

// Levels and emitter candidates of a built scene, kept for moving instances
// afterwards (the `placing` state of Trace, gpu.rs:530-540); build.cpp.
struct Placing;

// The packed buffers of one scene (SceneBuffers, gpu.rs:412-436).
struct SceneBlobs {
  std::vector<GpuTriangle> triangles;
  std::vector<GpuNode> nodes;
  std::vector<GpuHot> materials;
  std::vector<std::array<float, 4>> uv;
  std::vector<GpuSurface> surfaces;
  std::vector<GpuEmitter> emitters;
  std::vector<float> emitter_cdf;
  std::vector<GpuLight> lights;
  std::vector<uint32_t> order;
  std::vector<float> sky_rows, sky_columns;
  uint32_t sky_width = 1, sky_height = 1;
  float sky_radiance[3] = {0, 0, 0};
  std::vector<float> sobol;
  uint32_t sobol_length = 0;
  uint32_t triangle_count = 0, light_count = 0, emitter_count = 0;
  uint32_t max_depth = 0;
  std::shared_ptr<Placing> placing;  // null when the scene has no instances
  // Builds (gpu.rs:400-403): bottom-level BVHs built (the world's and one per
  // distinct mesh) and top-level BVHs laid (1 with instances, +1 per move).
  uint32_t bottom_builds = 0, top_builds = 0;
  uint32_t gpu_builds = 0;  // bottom-level BVHs built on the GPU
};

SceneBlobs* build_scene(const pfxt_scene& scene, const pfxt_settings& settings);

// Trace::move_instances (gpu.rs:2433-2530) on the host buffers: new transforms
// for the first `count` instances (16 floats each, column-major).  Rewrites the
// moved instances' surface records, their emitters and the top-level BVH in
// place (no buffer changes size) and returns whether anything moved.
bool move_instances(SceneBlobs& blobs, const float* transforms, size_t count);

// The binned-SAH BVH build on the GPU (bvh_gpu.cu): the host build's nodes and
// order byte for byte, for boxes with no NaN and no -0.0 coordinate.
bool gpu_bvh_available();
void gpu_bvh_build(const float* boxes, uint32_t n, uint32_t leaf, uint32_t most, std::vector<GpuNode>& nodes,
                   std::vector<uint32_t>& order);
// Whether large triangle BVHs are built on the GPU when one is present (1, the
// default) or always on the host (0); returns the previous setting.
int set_gpu_bvh(int on);

// slice::select_nth_unstable_by as the light tree runs it, on bare keys (tests).
void select_nth_for_test(const float* keys, uint32_t n, uint32_t index, int rounds, uint32_t* order);

// Thread-local last error of the C ABI.
void set_error(const std::string& message);

// Convert reference nodes into the B200 traversal layout (layout.cpp).
struct TraversalLayout {
  std::vector<WideNode> wide;
  std::vector<TravTri> tris;
  std::vector<InstRec> insts;
  uint32_t root = REF_NONE;  // wide node whose child 0 is the scene root
  bool small = false;        // every box coordinate 0 or within 2^-70..2^79 in magnitude (SceneView::small)
};
TraversalLayout make_layout(const pfxt_buffers& buffers);

}  // namespace pfxt
