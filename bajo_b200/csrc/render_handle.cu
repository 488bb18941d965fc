// render_handle.cu -- handle-based rendering: create / enqueue / download /
// destroy around bajo_render and bajo_render_guided (the host side of
// render_gpu_triangles, bajo/rt/gpu/triangle_path.mojo:143-172, and of
// GpuRtRenderTarget's download, bajo/rt/gpu/resources.mojo:275).
//
// The caller still owns every device buffer (workspace, pixels, scene).  A
// handle owns only host state: the settings, the workspace it renders into,
// and a CUDA graph of the last enqueued render.  The first enqueue on a
// capturable stream records the whole chunked launch sequence (memsets,
// primary / trace / shade / shadow kernels per bounce, resolve) into a graph;
// later enqueues with the same arguments replay it with one launch.  The
// graph reads buffer contents at replay time, so a new camera or new scene
// data in the same buffers needs no new graph; other pointers, or other
// scene, guide or settings values, record a new one.  The legacy default
// stream (NULL) cannot be captured: renders there are enqueued directly.
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/bajo_b200.h"

struct BajoRenderer {
  BajoRenderSettings settings;
  void* workspace;
  size_t workspace_bytes;
  // the arguments the graph was recorded with
  bool have_graph;
  BajoRtScene scene;
  BajoLbvh bvh;
  BajoGuide guide;
  bool guided;
  const float* camera;
  float* pixels;
  double* pixels64;
  cudaStream_t stream;
  cudaGraphExec_t exec;
  uint32_t graph_launches;
};

namespace {

int32_t render_now(BajoRenderer* r, const BajoRtScene* scene, const float* cam, float* px, double* px64,
                   const BajoGuide* guide, cudaStream_t st) {
  if (guide)
    return bajo_render_guided(scene, cam, &r->settings, guide, px, px64, r->workspace, r->workspace_bytes, st);
  return bajo_render(scene, cam, &r->settings, px, px64, r->workspace, r->workspace_bytes, st);
}

void drop_graph(BajoRenderer* r) {
  if (r->have_graph) cudaGraphExecDestroy(r->exec);
  r->have_graph = false;
}

bool same_args(const BajoRenderer* r, const BajoRtScene* scene, const float* cam, float* px, double* px64,
               const BajoGuide* guide, cudaStream_t st) {
  if (!r->have_graph || r->camera != cam || r->pixels != px || r->pixels64 != px64 || r->stream != st ||
      r->guided != (guide != nullptr))
    return false;
  if (std::memcmp(&r->scene, scene, sizeof(BajoRtScene)) != 0 ||
      std::memcmp(&r->bvh, scene->bvh, sizeof(BajoLbvh)) != 0)
    return false;
  return !guide || std::memcmp(&r->guide, guide, sizeof(BajoGuide)) == 0;
}

}  // namespace

extern "C" {

int32_t bajo_render_create(const BajoRenderSettings* settings, void* d_workspace, size_t workspace_bytes,
                           BajoRenderer** out) {
  if (!settings || !d_workspace || !out) return BAJO_ERR_INVALID_ARGUMENT;
  size_t need = 0;
  const int32_t rc = bajo_render_workspace_size(settings, &need);
  if (rc != BAJO_OK) return rc;
  if (workspace_bytes < need) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  BajoRenderer* r = static_cast<BajoRenderer*>(std::calloc(1, sizeof(BajoRenderer)));
  if (!r) return BAJO_ERR_CUDA;
  r->settings = *settings;
  r->workspace = d_workspace;
  r->workspace_bytes = workspace_bytes;
  *out = r;
  return BAJO_OK;
}

int32_t bajo_render_enqueue(BajoRenderer* r, const BajoRtScene* scene, const float* d_camera, const BajoGuide* guide,
                            float* d_pixels, double* d_pixels64, void* stream) {
  if (!r || !scene || !scene->bvh || !d_camera || !d_pixels) return BAJO_ERR_INVALID_ARGUMENT;
  if ((guide != nullptr) != (r->settings.algorithm == BAJO_RENDER_GUIDED)) return BAJO_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread)
    return render_now(r, scene, d_camera, d_pixels, d_pixels64, guide, st);
  if (!same_args(r, scene, d_camera, d_pixels, d_pixels64, guide, st)) {
    drop_graph(r);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return BAJO_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusNone)  // already inside the caller's capture: just record into it
      return render_now(r, scene, d_camera, d_pixels, d_pixels64, guide, st);
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return BAJO_ERR_CUDA;
    const int32_t rc = render_now(r, scene, d_camera, d_pixels, d_pixels64, guide, st);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != BAJO_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return rc != BAJO_OK ? rc : BAJO_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&r->exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return BAJO_ERR_CUDA;
    r->have_graph = true;
    r->scene = *scene;
    r->bvh = *scene->bvh;
    r->guided = guide != nullptr;
    if (guide) r->guide = *guide;
    r->camera = d_camera;
    r->pixels = d_pixels;
    r->pixels64 = d_pixels64;
    r->stream = st;
  }
  if (cudaGraphLaunch(r->exec, st) != cudaSuccess) return BAJO_ERR_CUDA;
  ++r->graph_launches;
  return BAJO_OK;
}

int32_t bajo_render_download(BajoRenderer* r, const float* d_pixels, float* h_pixels, uint64_t* rays,
                             uint64_t* shadow_rays, uint32_t* status, void* stream) {
  if (!r || (h_pixels && !d_pixels)) return BAJO_ERR_INVALID_ARGUMENT;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return BAJO_ERR_CUDA;
  if (h_pixels) {
    const size_t bytes = (size_t)r->settings.width * r->settings.height * 3 * sizeof(float);
    if (cudaMemcpy(h_pixels, d_pixels, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return BAJO_ERR_CUDA;
  }
  // workspace header: status word, then the two 64-bit ray totals at byte 8
  unsigned char head[24];
  if (cudaMemcpy(head, r->workspace, sizeof(head), cudaMemcpyDeviceToHost) != cudaSuccess) return BAJO_ERR_CUDA;
  if (status) std::memcpy(status, head, 4);
  if (rays) std::memcpy(rays, head + 8, 8);
  if (shadow_rays) std::memcpy(shadow_rays, head + 16, 8);
  return BAJO_OK;
}

int32_t bajo_render_graph_launches(const BajoRenderer* r, uint32_t* launches) {
  if (!r || !launches) return BAJO_ERR_INVALID_ARGUMENT;
  *launches = r->graph_launches;
  return BAJO_OK;
}

int32_t bajo_render_destroy(BajoRenderer* r) {
  if (!r) return BAJO_ERR_INVALID_ARGUMENT;
  drop_graph(r);
  std::free(r);
  return BAJO_OK;
}

}  // extern "C"
