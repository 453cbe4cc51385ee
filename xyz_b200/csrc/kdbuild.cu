// Device kd-tree builder (XYZGPU_BUILD_DEVICE).
#include "scene.h"

namespace xyzgpu {

int kd_build_device(SceneImpl &, const float4 *, int, const BuildConfig &, cudaStream_t) {
  return set_error(XYZGPU_E_INVALID, "scene_create: the device kd-tree builder is not available in this build");
}

}  // namespace xyzgpu
