// camera.cu -- host-side camera records (20 floats) for bajo_trace_camera.
// Restates Camera.__init__ / Camera.from_vfov (bajo/bvh/camera.mojo:77-116)
// with the reference's fma-based cross/dot (bajo/core/vec.mojo:440,522-539);
// compiled with -ffp-contract=off so every other operation rounds as written.
#include <cmath>
#include <cstring>

#include "../../include/bajo_b200.h"

namespace {
struct v3 {
  float x, y, z;
};
v3 sub(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
float dot(v3 a, v3 b) { return std::fmaf(a.x, b.x, std::fmaf(a.y, b.y, a.z * b.z)); }
v3 cross(v3 a, v3 b) {
  return {std::fmaf(a.y, b.z, -(a.z * b.y)), std::fmaf(a.z, b.x, -(a.x * b.z)), std::fmaf(a.x, b.y, -(a.y * b.x))};
}
v3 normalize(v3 v) {
  float l = std::sqrt(dot(v, v));
  float inv_l = (l > 1.0e-20f) ? 1.0f / l : 0.0f;
  return {v.x * inv_l, v.y * inv_l, v.z * inv_l};
}
}  // namespace

extern "C" {

int32_t bajo_camera_make(const float* origin, const float* target, const float* world_up, float fov_scale,
                         float* out20) {
  if (!origin || !target || !world_up || !out20) return BAJO_ERR_INVALID_ARGUMENT;
  v3 o{origin[0], origin[1], origin[2]}, t{target[0], target[1], target[2]};
  v3 up{world_up[0], world_up[1], world_up[2]};
  v3 fwd = normalize(sub(t, o));
  v3 right = normalize(cross(fwd, up));
  v3 u = normalize(cross(right, fwd));
  std::memset(out20, 0, 20 * sizeof(float));
  float* c = out20;
  c[0] = o.x; c[1] = o.y; c[2] = o.z;
  c[3] = fwd.x; c[4] = fwd.y; c[5] = fwd.z;
  c[6] = right.x; c[7] = right.y; c[8] = right.z;
  c[9] = u.x; c[10] = u.y; c[11] = u.z;
  c[12] = fov_scale;
  c[13] = 1.0f;  // focus distance; defocus disk vectors stay zero (angle 0)
  return BAJO_OK;
}

int32_t bajo_camera_from_vfov(const float* origin, const float* target, const float* world_up, float vfov_deg,
                              float* out20) {
  float theta = vfov_deg * (float)(3.14159265358979323846 / 180.0);
  return bajo_camera_make(origin, target, world_up, std::tan(theta / 2.0f), out20);
}

}  // extern "C"
