// C-ABI implementation (include/appearance_cuda.h): handle, scene upload and
// BVH build, camera, frame encode and readback.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/appearance_cuda.h"
#include "bvh_build.h"
#include "dev_common.cuh"
#include "device_scope.h"
#include "dev_shade.cuh"
#include "frame.cuh"
#include "spectral.cuh"
#include "spectral_fit.h"
#include "traverse.cuh"
#include "traverse2.cuh"
#include "world.h"

namespace {

using namespace ap;

static_assert(sizeof(ap_frame_config) == sizeof(FrameConfig), "config layout");
static_assert(sizeof(ap_material) == sizeof(MaterialDev), "material layout");

struct DeviceScene {
  void* nodes = nullptr;
  void* tris = nullptr;
  void* positions = nullptr;
  void* normals = nullptr;
  void* normals_f = nullptr;  // float vertex normals (the spectral mode's shading normals)
  void* indices = nullptr;
  void* tri_material = nullptr;
  void* tri_instance = nullptr;
  void* instances = nullptr;
  void* materials = nullptr;
  void* emissive_instances = nullptr;
  void* emissive_cdf = nullptr;
  void* emissive_tris = nullptr;
  void* emissive_tri_base = nullptr;
  void* emissive_info = nullptr;
  void* env = nullptr;
  DevScene view{};
  // host copies for the spectral tables (ap_spectral_setup)
  std::vector<float> host_materials;  // 26 floats per material
  std::vector<float> host_env;        // RGB per texel
  BvhStats stats{};
  size_t bytes = 0;  // device memory held
  bool valid = false;
  void release() {
    void** all[] = {&nodes, &tris, &positions, &normals, &normals_f, &indices, &tri_material, &tri_instance,
                    &instances, &materials, &emissive_instances, &emissive_cdf, &emissive_tris,
                    &emissive_tri_base, &emissive_info, &env};
    for (void** p : all) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    bytes = 0;
    valid = false;
  }
};

// The device copy of a world's two-level form (World::build_two_level),
// used by the ray queries when the world has spawned instances.
struct DeviceTwoLevel {
  void *nodes = nullptr, *tris = nullptr, *tlas_nodes = nullptr, *tlas_leaves = nullptr, *insts = nullptr;
  void *positions = nullptr, *normals = nullptr, *indices = nullptr, *tri_mat = nullptr, *model_tri0 = nullptr,
       *tri_inst = nullptr, *env = nullptr;
  DevScene view{};  // nodes / tris: the BLAS pool; env: the base scene's environment
  TwoLevel tl{};
  ModelGeo mg{};
  std::vector<ap_material> materials;  // the models' materials, as tri_mat indexes them
  uint64_t version = ~0ull;
  bool valid = false;
  void release() {
    void** all[] = {&nodes, &tris, &tlas_nodes, &tlas_leaves, &insts, &positions, &normals, &indices, &tri_mat,
                    &model_tri0, &tri_inst, &env};
    for (void** p : all) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    valid = false;
    version = ~0ull;
  }
};

struct Handle {
  FrameConfig cfg{};
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  FrameStreams fs;  // second stream of the frame (DI shadow rays beside the next extension)
  std::string err;
  DeviceScene scene;
  void* frame_mem = nullptr;
  size_t frame_bytes = 0;
  uint32_t W = 0, H = 0;
  FrameBuffers fb{};
  uint32_t frame_idx = 0;
  // camera
  bool explicit_mats = false;
  Mats mats{};
  double cam_transform[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  float fov = 60.0f, znear = 0.1f, zfar = 300.0f;  // Camera::default (appearance-camera/src/lib.rs)
  bool have_prev = false;
  double prev_vp[16] = {0};
  // scratch for ap_trace_rays
  void* trace_mem = nullptr;
  size_t trace_bytes = 0;
  uint64_t ext_rays = 0;
  FrameProfiler prof;
  uint32_t accum_count = 0;  // frames in the display accumulation (resolve.wgsl accum_frame_count)
  // radiance cache mode (ap_rc_attach)
  RcFrame rc{};
  void* rc_mem = nullptr;
  uint32_t rc_w = 0, rc_h = 0;
  // spectral mode (ap_spectral_setup / ap_render_spectral)
  void* spec_mats = nullptr;
  void* spec_env = nullptr;  // the environment's compensated sampling distribution
  void* spec_tab = nullptr;  // illuminant upsampling table (cache mode's predictions)
  void* spec_out = nullptr;
  size_t spec_out_bytes = 0;
  SpectralView spec{};
  bool spec_ready = false;
  uint64_t spec_version = 0;  // the world the spectral tables were built for
  // base scene, registered models and spawned instances (world actions)
  World world;
  DeviceTwoLevel two_level;
  void spec_release() {
    if (spec_mats) cudaFree(spec_mats);
    if (spec_env) cudaFree(spec_env);
    if (spec_tab) cudaFree(spec_tab);
    spec_mats = spec_env = spec_tab = nullptr;
    spec_ready = false;
  }
};

int fail(Handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int check_cuda(Handle* h, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return AP_OK;
  if (e == cudaErrorMemoryAllocation) return fail(h, AP_E_OOM, std::string(what) + ": " + cudaGetErrorString(e));
  return fail(h, AP_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
int upload(Handle* h, void** dst, const T* src, size_t count) {
  size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  int rc = check_cuda(h, cudaMalloc(dst, bytes), "cudaMalloc");
  if (rc) return rc;
  h->scene.bytes += bytes;
  if (count) rc = check_cuda(h, cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice), "upload");
  return rc;
}

__global__ void k_sun_derive(SunDev* s) { sun_derive(*s); }

// The sun's derived fields, computed on the device like every other use of
// the sun functions' arithmetic (run once per scene upload).
int derive_sun(Handle* h, SunDev* sun) {
  void* d = nullptr;
  int rc = check_cuda(h, cudaMalloc(&d, sizeof(SunDev)), "sun");
  if (rc) return rc;
  rc = check_cuda(h, cudaMemcpy(d, sun, sizeof(SunDev), cudaMemcpyHostToDevice), "sun");
  if (!rc) {
    k_sun_derive<<<1, 1, 0, h->stream>>>(static_cast<SunDev*>(d));
    rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sun derive");
  }
  if (!rc) rc = check_cuda(h, cudaMemcpy(sun, d, sizeof(SunDev), cudaMemcpyDeviceToHost), "sun");
  cudaFree(d);
  return rc;
}

// Fills the emissive-triangle table (run once per scene upload).
__global__ void k_build_emissive_tris(DevScene s, EmissiveTri* out, uint32_t total) {
  uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  uint32_t lo = 0, hi = s.num_emissive_instances;  // instance whose range holds g
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (s.emissive_tri_base[mid] <= g) lo = mid;
    else hi = mid;
  }
  const InstanceDev in = s.instances[s.emissive_instances[lo]];
  uint32_t tri = g - s.emissive_tri_base[lo];
  float3 p0, p1, p2;
  tri_positions(s, in, tri, &p0, &p1, &p2);
  float3 cr = cross(p1 - p0, p2 - p0);
  float3 n = normalize(cr);
  const MaterialDev* m = s.materials + in.material_idx + s.tri_material[in.first_index / 3 + tri];
  EmissiveTri e;
  e.p0[0] = p0.x; e.p0[1] = p0.y; e.p0[2] = p0.z; e.area = len(cr) * 0.5f;
  e.p1[0] = p1.x; e.p1[1] = p1.y; e.p1[2] = p1.z; e.pad0 = 0.0f;
  e.p2[0] = p2.x; e.p2[1] = p2.y; e.p2[2] = p2.z; e.pad1 = 0.0f;
  e.n[0] = n.x; e.n[1] = n.y; e.n[2] = n.z; e.pad2 = 0.0f;
  e.emission[0] = m->emission[0]; e.emission[1] = m->emission[1]; e.emission[2] = m->emission[2]; e.pad3 = 0.0f;
  out[g] = e;
}

__global__ void k_pack_normals(const float* n, uint32_t count, uint32_t* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] = pack_oct30(f3(n[3 * i], n[3 * i + 1], n[3 * i + 2]));
}

// ---- camera: glam perspective_rh / look_to_rh in double, rounded once ----
void mat_mul(const double* a, const double* b, double* out) {  // column-major
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += a[k * 4 + r] * b[c * 4 + k];
      out[c * 4 + r] = s;
    }
}
bool mat_inv(const double* m, double* out) {  // Gauss-Jordan, column-major in/out
  double a[4][8];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      a[r][c] = m[c * 4 + r];
      a[r][c + 4] = r == c ? 1.0 : 0.0;
    }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (std::fabs(a[piv][c]) < 1e-300) return false;
    for (int k = 0; k < 8; ++k) std::swap(a[c][k], a[piv][k]);
    double inv = 1.0 / a[c][c];
    for (int k = 0; k < 8; ++k) a[c][k] *= inv;
    for (int r = 0; r < 4; ++r)
      if (r != c) {
        double f = a[r][c];
        for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
      }
  }
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out[c * 4 + r] = a[r][c + 4];
  return true;
}

void camera_from_transform(Handle* hd, uint32_t w, uint32_t h, double* view, double* proj) {
  // CameraUpdate (lib.rs:285-294): rotation + translation of the transform;
  // Transform::get_view_matrix = look_to_rh(t, R*(0,0,-1), R*(0,1,0)).
  const double* m = hd->cam_transform;
  double cx[3] = {m[0], m[1], m[2]}, cy[3] = {m[4], m[5], m[6]}, cz[3] = {m[8], m[9], m[10]};
  auto nrm = [](double* v) {
    double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > 0) { v[0] /= l; v[1] /= l; v[2] /= l; }
  };
  nrm(cx); nrm(cy); nrm(cz);
  double t[3] = {m[12], m[13], m[14]};
  // view = inverse(rigid(R, t)): rows of R, translation -R^T t
  double v[16] = {cx[0], cy[0], cz[0], 0, cx[1], cy[1], cz[1], 0, cx[2], cy[2], cz[2], 0,
                  -(cx[0] * t[0] + cx[1] * t[1] + cx[2] * t[2]),
                  -(cy[0] * t[0] + cy[1] * t[1] + cy[2] * t[2]),
                  -(cz[0] * t[0] + cz[1] * t[1] + cz[2] * t[2]), 1};
  std::memcpy(view, v, sizeof(v));
  double f = 1.0 / std::tan(0.5 * (double)hd->fov * M_PI / 180.0);
  double aspect = (double)w / (double)h;
  double r = (double)hd->zfar / ((double)hd->znear - (double)hd->zfar);
  double p[16] = {f / aspect, 0, 0, 0, 0, f, 0, 0, 0, 0, r, -1, 0, 0, r * hd->znear, 0};
  std::memcpy(proj, p, sizeof(p));
}

void compute_mats(Handle* hd, uint32_t w, uint32_t h) {
  if (hd->explicit_mats) return;
  double view[16], proj[16], vp[16], iv[16], ip[16];
  camera_from_transform(hd, w, h, view, proj);
  mat_mul(proj, view, vp);
  mat_inv(view, iv);
  mat_inv(proj, ip);
  const double* pvp = hd->have_prev ? hd->prev_vp : vp;
  for (int i = 0; i < 16; ++i) {
    hd->mats.inv_view[i] = (float)iv[i];
    hd->mats.inv_proj[i] = (float)ip[i];
    hd->mats.view_proj[i] = (float)vp[i];
    hd->mats.prev_view_proj[i] = (float)pvp[i];
  }
  std::memcpy(hd->prev_vp, vp, sizeof(vp));
  hd->have_prev = true;
}

int ensure_frame(Handle* h, uint32_t w, uint32_t hgt) {
  if (h->frame_mem && h->W == w && h->H == hgt) return AP_OK;
  if (h->frame_mem) cudaFree(h->frame_mem);
  h->frame_mem = nullptr;
  size_t bytes = frame_buffer_bytes(w, hgt);
  int rc = check_cuda(h, cudaMalloc(&h->frame_mem, bytes), "frame buffers");
  if (rc) return rc;
  rc = check_cuda(h, cudaMemsetAsync(h->frame_mem, 0, bytes, h->stream), "frame buffers");
  if (rc) return rc;
  h->frame_bytes = bytes;
  frame_buffers_carve(h->frame_mem, w, hgt, &h->fb);
  h->W = w;
  h->H = hgt;
  h->frame_idx = 0;  // SizedResources::new restarts the temporal state
  h->accum_count = 0;
  return AP_OK;
}

int world_sync(Handle* h);

int render_common(Handle* h, uint32_t w, uint32_t hgt, ap_frame_stats* stats, FrameProfiler* prof = nullptr) {
  if (w == 0 || hgt == 0 || (uint64_t)w * hgt > (1ull << 28)) return fail(h, AP_E_INVALID, "bad resolution");
  if (int wrc = world_sync(h)) return wrc;
  if (!h->scene.valid) return fail(h, AP_E_NO_SCENE, "no scene uploaded");
  const FrameConfig& c = h->cfg;
  if (c.sample_count == 0 || c.max_bounces == 0 || c.max_bounces > 64 || c.di_area_samples > 1024 ||
      c.di_bsdf_samples > 16 || c.svgf_atrous_passes > 8 || c.di_spatial_samples > 64 || c.gi_spatial_samples > 64 ||
      c.di_spatial_passes > 16 || c.gi_spatial_passes > 16)
    return fail(h, AP_E_INVALID, "frame config out of range");
  int rc = ensure_frame(h, w, hgt);
  if (rc) return rc;
  if (h->rc.cache && (h->rc_w != w || h->rc_h != hgt)) {
    if (h->rc_mem) cudaFree(h->rc_mem);
    h->rc_mem = nullptr;
    h->rc_w = h->rc_h = 0;
    rc = check_cuda(h, cudaMalloc(&h->rc_mem, rc_frame_bytes(w, hgt, h->rc.stride, h->rc.batch)), "radiance cache buffers");
    if (rc) return rc;
    rc_frame_carve(h->rc_mem, w, hgt, h->rc.stride, h->rc.batch, &h->rc);
    h->rc_w = w;
    h->rc_h = hgt;
  }
  compute_mats(h, w, hgt);
  cudaEventRecord(h->ev0, h->stream);
  int launches = encode_frame(h->scene.view, h->fb, h->cfg, h->mats, w, hgt, h->frame_idx, h->num_sms, h->stream, prof,
                              h->rc.cache ? &h->rc : nullptr, &h->fs);
  cudaEventRecord(h->ev1, h->stream);
  uint32_t rays = 0;
  cudaMemcpyAsync(&rays, h->fb.counters + 3, 4, cudaMemcpyDeviceToHost, h->stream);
  rc = check_cuda(h, cudaGetLastError(), "frame launch");
  if (rc) return rc;
  rc = check_cuda(h, cudaEventSynchronize(h->ev1), "frame");
  if (rc) return rc;
  if (h->rc.cache) {
    std::string msg;
    if ((rc = rc_take_status(h->rc.cache, &msg))) return fail(h, rc, "radiance cache: " + msg);
  }
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (stats) {
    stats->gpu_ms = ms;
    stats->extension_rays = rays;
    stats->kernel_launches = (uint32_t)launches;
    stats->width = w;
    stats->height = hgt;
    stats->frame_idx = h->frame_idx;
  }
  h->frame_idx += 1;
  return AP_OK;
}

int validate_scene(Handle* h, const ap_scene_desc* d) {
  if (!d->positions || !d->normals || !d->indices || !d->tri_material || !d->meshes || !d->materials)
    return fail(h, AP_E_INVALID, "scene: null array");
  if (d->num_meshes == 0 || d->num_materials == 0) return fail(h, AP_E_INVALID, "scene: no meshes or materials");
  // validate mesh ranges
  uint64_t tri_total = 0;
  for (uint32_t m = 0; m < d->num_meshes; ++m) {
    const ap_mesh& me = d->meshes[m];
    if (me.num_indices % 3 != 0 || (uint64_t)me.first_index + me.num_indices > 3ull * d->num_tris ||
        (uint64_t)me.first_vertex + me.num_vertices > d->num_vertices || me.material_idx >= d->num_materials)
      return fail(h, AP_E_INVALID, "scene: mesh " + std::to_string(m) + " out of range");
    if (me.first_index != 3 * tri_total) return fail(h, AP_E_INVALID, "scene: meshes must be contiguous in index order");
    tri_total += me.num_indices / 3;
  }
  if (tri_total != d->num_tris) return fail(h, AP_E_INVALID, "scene: meshes do not cover all triangles");
  for (uint32_t m = 0; m < d->num_meshes; ++m) {
    const ap_mesh& me = d->meshes[m];
    for (uint32_t i = 0; i < me.num_indices; ++i)
      if (d->indices[me.first_index + i] >= me.num_vertices) return fail(h, AP_E_INVALID, "scene: index out of range");
    for (uint32_t t = 0; t < me.num_indices / 3; ++t)
      if (me.material_idx + d->tri_material[me.first_index / 3 + t] >= d->num_materials)
        return fail(h, AP_E_INVALID, "scene: triangle material out of range");
  }
  return AP_OK;
}

// Replaces the device scene with `d` (validated) and builds its BVH.
int upload_scene(Handle* h, const ap_scene_desc* d) {
  ap::DeviceScope device_scope(h->device);
  cudaStreamSynchronize(h->stream);
  h->scene.release();
  h->spec_release();
  // flattened world triangles, instances, emissive list and CDF (vertex_pool.rs:307-348)
  std::vector<float> tv(9 * (size_t)d->num_tris);
  std::vector<InstanceDev> inst(d->num_meshes);
  std::vector<uint32_t> tri_inst(d->num_tris);
  std::vector<uint32_t> emissive;
  uint32_t num_emissive_tris = 0;
  uint32_t g = 0;
  for (uint32_t m = 0; m < d->num_meshes; ++m) {
    const ap_mesh& me = d->meshes[m];
    InstanceDev& in = inst[m];
    std::memset(&in, 0, sizeof(in));
    in.first_vertex = me.first_vertex;
    in.first_index = me.first_index;
    in.num_indices = me.num_indices;
    in.material_idx = me.material_idx;
    in.emissive_idx = 0xFFFFFFFFu;
    in.first_global_tri = g;
    if (me.emissive) {
      in.emissive_idx = (uint32_t)emissive.size();
      emissive.push_back(m);
      num_emissive_tris += me.num_indices / 3;
    }
    for (uint32_t t = 0; t < me.num_indices / 3; ++t, ++g) {
      tri_inst[g] = m;
      for (int k = 0; k < 3; ++k) {
        const float* p = d->positions + 3 * (size_t)(me.first_vertex + d->indices[me.first_index + 3 * t + k]);
        tv[9 * (size_t)g + 3 * k + 0] = p[0];
        tv[9 * (size_t)g + 3 * k + 1] = p[1];
        tv[9 * (size_t)g + 3 * k + 2] = p[2];
      }
    }
  }
  std::vector<uint32_t> tri_base;
  {
    uint32_t b = 0;
    for (uint32_t e : emissive) {
      tri_base.push_back(b);
      b += inst[e].num_indices / 3;
    }
  }
  std::vector<float> cdf;
  float acc = 0.0f;
  for (uint32_t e : emissive) {
    float pdf = (float)(inst[e].num_indices / 3) / (float)num_emissive_tris;
    acc = acc + pdf;
    cdf.push_back(acc);
  }
  std::vector<uint4> info(emissive.size());
  for (size_t e = 0; e < emissive.size(); ++e) {
    uint32_t cb;
    std::memcpy(&cb, &cdf[e], 4);
    info[e] = make_uint4(cb, tri_base[e], inst[emissive[e]].num_indices / 3, 0u);
  }
  WideBvh bvh;
  std::string berr;
  if (!build_wide_bvh(tv.data(), d->num_tris, (uint32_t)kTraversalStack, &bvh, &berr))
    return fail(h, AP_E_INVALID, "BVH build: " + berr);
  std::vector<float4> pos4(d->num_vertices);
  for (uint32_t i = 0; i < d->num_vertices; ++i)
    pos4[i] = make_float4(d->positions[3 * i], d->positions[3 * i + 1], d->positions[3 * i + 2], 0.0f);
  DeviceScene& s = h->scene;
  int rc = 0;
  if ((rc = upload(h, &s.nodes, bvh.nodes.data(), bvh.nodes.size())) ||
      (rc = upload(h, &s.tris, bvh.tris.data(), bvh.tris.size())) ||
      (rc = upload(h, &s.positions, pos4.data(), pos4.size())) ||
      (rc = upload(h, &s.normals_f, d->normals, 3 * (size_t)d->num_vertices)) ||
      (rc = check_cuda(h, cudaMalloc(&s.normals, std::max<size_t>(4 * (size_t)d->num_vertices, 16)), "normals")) ||
      (rc = upload(h, &s.indices, d->indices, 3 * (size_t)d->num_tris)) ||
      (rc = upload(h, &s.tri_material, d->tri_material, d->num_tris)) ||
      (rc = upload(h, &s.tri_instance, tri_inst.data(), tri_inst.size())) ||
      (rc = upload(h, &s.instances, inst.data(), inst.size())) ||
      (rc = upload(h, &s.materials, reinterpret_cast<const MaterialDev*>(d->materials), d->num_materials)) ||
      (rc = upload(h, &s.emissive_instances, emissive.data(), emissive.size())) ||
      (rc = upload(h, &s.emissive_cdf, cdf.data(), cdf.size())) ||
      (rc = upload(h, &s.emissive_tri_base, tri_base.data(), tri_base.size())) ||
      (rc = upload(h, &s.emissive_info, info.data(), info.size())) ||
      (rc = check_cuda(h, cudaMalloc(&s.emissive_tris, std::max<size_t>(sizeof(EmissiveTri) * num_emissive_tris, 16)),
                       "emissive triangles"))) {
    s.release();
    return rc;
  }
  if (d->num_vertices)
    k_pack_normals<<<(d->num_vertices + 255) / 256, 256, 0, h->stream>>>(static_cast<const float*>(s.normals_f),
                                                                           d->num_vertices,
                                                                           static_cast<uint32_t*>(s.normals));
  rc = check_cuda(h, cudaStreamSynchronize(h->stream), "pack normals");
  if (rc) {
    s.release();
    return rc;
  }
  if (d->env && d->env_w && d->env_h) {
    if ((rc = upload(h, &s.env, d->env, 3 * (size_t)d->env_w * d->env_h))) {
      s.release();
      return rc;
    }
  }
  DevScene& v = s.view;
  v.nodes = static_cast<const uint4*>(s.nodes);
  v.tris = static_cast<const float4*>(s.tris);
  v.positions = static_cast<const float4*>(s.positions);
  v.normals = static_cast<const uint32_t*>(s.normals);
  v.normals_f = static_cast<const float*>(s.normals_f);
  v.indices = static_cast<const uint32_t*>(s.indices);
  v.tri_material = static_cast<const uint32_t*>(s.tri_material);
  v.tri_instance = static_cast<const uint32_t*>(s.tri_instance);
  v.instances = static_cast<const InstanceDev*>(s.instances);
  v.materials = static_cast<const MaterialDev*>(s.materials);
  v.emissive_instances = static_cast<const uint32_t*>(s.emissive_instances);
  v.emissive_cdf = static_cast<const float*>(s.emissive_cdf);
  v.num_emissive_instances = (uint32_t)emissive.size();
  v.num_emissive_tris = num_emissive_tris;
  v.env = static_cast<const float*>(s.env);
  v.env_w = s.env ? d->env_w : 0;
  v.env_h = s.env ? d->env_h : 0;
  std::memset(&v.sun, 0, sizeof(SunDev));
  std::memcpy(&v.sun, d->sun, 8 * sizeof(float));  // direction, size, color, intensity
  if ((rc = derive_sun(h, &v.sun))) {
    s.release();
    return rc;
  }
  v.num_tris = d->num_tris;
  v.emissive_tri_base = static_cast<const uint32_t*>(s.emissive_tri_base);
  v.emissive_info = static_cast<const uint4*>(s.emissive_info);
  v.emissive_tris = static_cast<const EmissiveTri*>(s.emissive_tris);
  if (num_emissive_tris) {
    k_build_emissive_tris<<<(num_emissive_tris + 255) / 256, 256, 0, h->stream>>>(
        v, static_cast<EmissiveTri*>(s.emissive_tris), num_emissive_tris);
    rc = check_cuda(h, cudaStreamSynchronize(h->stream), "emissive triangles");
    if (rc) {
      s.release();
      return rc;
    }
  }
  {
    const float* mf = reinterpret_cast<const float*>(d->materials);
    s.host_materials.assign(mf, mf + 26 * (size_t)d->num_materials);
  }
  if (s.env) s.host_env.assign(d->env, d->env + 3 * (size_t)d->env_w * d->env_h);
  else s.host_env.clear();
  s.stats = bvh.stats;
  s.bytes += std::max<size_t>(4 * (size_t)d->num_vertices, 16) + std::max<size_t>(sizeof(EmissiveTri) * num_emissive_tris, 16);
  s.valid = true;
  return AP_OK;
}

// Re-uploads the world after world actions changed it (the reference rebuilds
// its TLAS before every frame, scene_resources/mod.rs:218-276).
int world_sync(Handle* h) {
  if (!h->world.dirty) return AP_OK;
  h->world.dirty = false;
  HostScene flat;
  h->world.flatten(&flat);
  if (flat.meshes.empty()) {
    ap::DeviceScope device_scope(h->device);
    cudaStreamSynchronize(h->stream);
    h->scene.release();
    h->spec_release();
    return AP_OK;
  }
  const ap_scene_desc d = flat.desc();
  int rc = validate_scene(h, &d);
  if (rc) return rc;
  return upload_scene(h, &d);
}

// The two-level form of a world with spawned instances (null without
// instances: the flat scene is the world), rebuilt after a change.
int two_level_sync(Handle* h, const TwoLevel** out) {
  *out = nullptr;
  if (h->world.instances.empty()) {
    h->two_level.release();
    return AP_OK;
  }
  DeviceTwoLevel& t = h->two_level;
  if (t.valid && t.version == h->world.version) {
    *out = &t.tl;
    return AP_OK;
  }
  ap::DeviceScope device_scope(h->device);
  cudaStreamSynchronize(h->stream);
  t.release();
  TwoLevelHost host;
  std::string err;
  if (!h->world.build_two_level((uint32_t)kTraversalStack, &host, &err)) return fail(h, AP_E_INVALID, err);
  auto put = [&](void** dst, const void* src, size_t bytes, const char* what) {
    int rc = check_cuda(h, cudaMalloc(dst, std::max<size_t>(bytes, 16)), what);
    if (!rc && bytes) rc = check_cuda(h, cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), what);
    return rc;
  };
  int rc = 0;
  if ((rc = put(&t.nodes, host.nodes.data(), sizeof(WideNode) * host.nodes.size(), "BLAS nodes")) ||
      (rc = put(&t.tris, host.tris.data(), sizeof(TriRec) * host.tris.size(), "BLAS triangles")) ||
      (rc = put(&t.tlas_nodes, host.tlas_nodes.data(), sizeof(WideNode) * host.tlas_nodes.size(), "TLAS nodes")) ||
      (rc = put(&t.tlas_leaves, host.tlas_leaves.data(), sizeof(TriRec) * host.tlas_leaves.size(), "TLAS leaves")) ||
      (rc = put(&t.insts, host.insts.data(), sizeof(InstRec) * host.insts.size(), "instances")) ||
      (rc = put(&t.positions, host.positions4.data(), sizeof(float) * host.positions4.size(), "model vertices")) ||
      (rc = put(&t.normals, host.normals.data(), sizeof(float) * host.normals.size(), "model normals")) ||
      (rc = put(&t.indices, host.indices.data(), sizeof(uint32_t) * host.indices.size(), "model indices")) ||
      (rc = put(&t.tri_mat, host.tri_material.data(), sizeof(uint32_t) * host.tri_material.size(), "model materials")) ||
      (rc = put(&t.model_tri0, host.model_tri0.data(), sizeof(uint32_t) * host.model_tri0.size(), "model table")) ||
      (rc = put(&t.tri_inst, host.tri_inst.data(), sizeof(uint32_t) * host.tri_inst.size(), "triangle instances")) ||
      (rc = put(&t.env, h->world.base.env.data(), sizeof(float) * h->world.base.env.size(), "environment"))) {
    t.release();
    return rc;
  }
  std::memset(&t.view, 0, sizeof(t.view));
  t.view.nodes = static_cast<const uint4*>(t.nodes);
  t.view.tris = static_cast<const float4*>(t.tris);
  t.view.env = h->world.base.env_w ? static_cast<const float*>(t.env) : nullptr;
  t.view.env_w = h->world.base.env_w;
  t.view.env_h = h->world.base.env_h;
  t.mg.positions = static_cast<const float4*>(t.positions);
  t.mg.normals = static_cast<const float*>(t.normals);
  t.mg.indices = static_cast<const uint32_t*>(t.indices);
  t.mg.tri_mat = static_cast<const uint32_t*>(t.tri_mat);
  t.mg.model_tri0 = static_cast<const uint32_t*>(t.model_tri0);
  t.mg.tri_inst = static_cast<const uint32_t*>(t.tri_inst);
  t.materials = host.materials;
  t.tl.tlas_nodes = static_cast<const uint4*>(t.tlas_nodes);
  t.tl.tlas_leaves = static_cast<const float4*>(t.tlas_leaves);
  t.tl.insts = static_cast<const InstRec*>(t.insts);
  t.tl.num_insts = (uint32_t)host.insts.size();
  t.version = h->world.version;
  t.valid = true;
  *out = &t.tl;
  return AP_OK;
}

}  // namespace

namespace ap {
// Scene, stream and error slot of a handle, for entry points defined in other
// translation units (noalloc.cu).  Returns AP_E_NO_SCENE when no scene is loaded.
int handle_trace_context(void* hp, const DevScene** scene, const TwoLevel** two_level, cudaStream_t* stream,
                         int* num_sms, int* device, std::string** err) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  *err = &h->err;
  if (h->world.instances.empty()) {
    if (int rc = world_sync(h)) return rc;
    if (!h->scene.valid) {
      h->err = "no scene uploaded";
      return AP_E_NO_SCENE;
    }
  }
  if (int rc = two_level_sync(h, two_level)) return rc;
  *scene = *two_level ? &h->two_level.view : &h->scene.view;
  *stream = h->stream;
  *num_sms = h->num_sms;
  *device = h->device;
  return AP_OK;
}

// Device bytes held by a handle's scene (0 without one).
size_t handle_scene_bytes(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  return (h && h->scene.valid) ? h->scene.bytes : 0;
}
}  // namespace ap

extern "C" {

void ap_frame_config_default(ap_frame_config* c) {
  if (!c) return;
  c->max_bounces = 2;
  c->sample_count = 1;
  c->restir_di = 1;
  c->restir_gi = 1;
  c->svgf = 0;
  c->firefly_filter = 1;
  c->taa = 0;
  c->di_area_samples = 4;
  c->di_bsdf_samples = 1;
  c->di_temporal_m_factor = 20.0f;
  c->di_spatial_passes = 1;
  c->di_spatial_samples = 3;
  c->di_unbiased = 1;
  c->gi_temporal_m_cap = 30.0f;
  c->gi_spatial_passes = 0;
  c->gi_spatial_samples = 5;
  c->gi_unbiased = 1;
  c->svgf_max_history = 24;
  c->svgf_atrous_passes = 5;
  c->taa_history_influence = 0.8f;
}

void* ap_create(const ap_frame_config* cfg, int device, int* err) {
  int dummy;
  if (!err) err = &dummy;
  *err = AP_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    *err = AP_E_CUDA;
    return nullptr;
  }
  Handle* h = new Handle();
  h->device = device;
  if (cfg) std::memcpy(&h->cfg, cfg, sizeof(FrameConfig));
  else ap_frame_config_default(reinterpret_cast<ap_frame_config*>(&h->cfg));
  ap::DeviceScope device_scope(device);
  if (device_scope.status() != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess ||
      frame_streams_create(&h->fs) != 0) {
    *err = AP_E_CUDA;
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return nullptr;
  }
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  return h;
}

void ap_destroy(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return;
  ap::DeviceScope device_scope(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  h->scene.release();
  h->two_level.release();
  if (h->frame_mem) cudaFree(h->frame_mem);
  if (h->trace_mem) cudaFree(h->trace_mem);
  if (h->rc_mem) cudaFree(h->rc_mem);
  h->spec_release();
  if (h->spec_out) cudaFree(h->spec_out);
  if (h->prof.created)
    for (int i = 0; i <= FrameProfiler::kMax; ++i) cudaEventDestroy(h->prof.ev[i]);
  frame_streams_destroy(&h->fs);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

const char* ap_last_error(const void* hp) {
  const Handle* h = static_cast<const Handle*>(hp);
  return h ? h->err.c_str() : "null handle";
}

int ap_set_config(void* hp, const ap_frame_config* cfg) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !cfg) return AP_E_INVALID;
  std::memcpy(&h->cfg, cfg, sizeof(FrameConfig));
  // a new configuration starts a new frame sequence: drop the temporal state
  ap::DeviceScope device_scope(h->device);
  cudaStreamSynchronize(h->stream);
  if (h->frame_mem) cudaFree(h->frame_mem);
  h->frame_mem = nullptr;
  h->W = h->H = 0;
  h->frame_idx = 0;
  h->have_prev = false;
  return AP_OK;
}

int ap_world_action(void* hp, uint32_t ty, const void* bytes, size_t len) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  switch (ty) {
    case 0: {  // CameraUpdateData {Mat4, fov, near, far, pad}
      if (!bytes || len != 80) return fail(h, AP_E_INVALID, "CameraUpdate expects 80 bytes");
      const float* f = static_cast<const float*>(bytes);
      for (int i = 0; i < 16; ++i) h->cam_transform[i] = f[i];
      h->fov = f[16];
      h->znear = f[17];
      h->zfar = f[18];
      h->explicit_mats = false;
      return AP_OK;
    }
    case 4: {  // Clear
      if (!bytes || len != 4) return fail(h, AP_E_INVALID, "Clear expects 4 bytes");
      h->world.clear();
      return world_sync(h);
    }
    case 1:
    case 2:
    case 3: {
      const uint8_t* b = static_cast<const uint8_t*>(bytes);
      std::string msg;
      const int rc = ty == 1 ? h->world.spawn(b, len, &msg)
                             : (ty == 2 ? h->world.transform(b, len, &msg) : h->world.destroy(b, len, &msg));
      return rc ? fail(h, rc, msg) : AP_OK;
    }
    default:
      return fail(h, AP_E_INVALID, "unknown world action type");
  }
}

int ap_scene_upload(void* hp, const ap_scene_desc* d) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !d) return AP_E_INVALID;
  int rc = validate_scene(h, d);
  if (rc) return rc;
  h->world.base.assign(*d);
  h->world.instances.clear();
  h->world.dirty = false;
  ++h->world.version;
  return upload_scene(h, d);
}

int ap_model_register(void* hp, const char* asset_path, const ap_scene_desc* d) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !d || !asset_path) return AP_E_INVALID;
  const std::string path(asset_path);
  if (path.empty() || path.size() >= 256) return fail(h, AP_E_INVALID, "model: asset path must have 1..255 bytes");
  int rc = validate_scene(h, d);
  if (rc) return rc;
  h->world.models[path].assign(*d);
  ++h->world.version;
  for (const World::Instance& in : h->world.instances)
    if (in.path == path) h->world.dirty = true;
  return AP_OK;
}


int ap_set_camera_matrices(void* hp, const float* m) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !m) return AP_E_INVALID;
  std::memcpy(&h->mats, m, sizeof(Mats));
  h->explicit_mats = true;
  return AP_OK;
}

int ap_render_hdr(void* hp, uint32_t w, uint32_t hgt, uint32_t row_start, uint32_t row_end, float* out,
                  size_t out_bytes, ap_frame_stats* stats) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  if (row_start >= row_end || row_end > hgt) return fail(h, AP_E_INVALID, "bad row range");
  size_t need = (size_t)(row_end - row_start) * w * 3 * sizeof(float);
  if (!out || out_bytes < need) return fail(h, AP_E_INVALID, "output buffer too small");
  ap::DeviceScope device_scope(h->device);
  int rc = render_common(h, w, hgt, stats);
  if (rc) return rc;
  rc = check_cuda(h, cudaMemcpyAsync(out, h->fb.out_rgb + (size_t)row_start * w * 3, need, cudaMemcpyDeviceToHost, h->stream),
                  "readback");
  if (rc) return rc;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "readback");
}

int ap_rc_attach(void* hp, void* cache, uint32_t prefix_bounces, uint32_t train_stride, uint32_t train_batch, float lr,
                 int train) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  if (cache && (prefix_bounces == 0 || prefix_bounces >= kRcMaxBounces || train_stride == 0 || train_batch == 0 ||
                train_batch > (1u << 22) || !(lr >= 0.0f)))
    return fail(h, AP_E_INVALID, "radiance cache: parameters out of range");
  ap::DeviceScope device_scope(h->device);
  cudaStreamSynchronize(h->stream);
  if (h->rc_mem) cudaFree(h->rc_mem);
  h->rc_mem = nullptr;
  h->rc_w = h->rc_h = 0;
  h->rc = RcFrame{};
  if (cache) {
    h->rc.cache = cache;
    h->rc.prefix = prefix_bounces;
    h->rc.stride = train_stride;
    h->rc.batch = train_batch;
    h->rc.lr = lr;
    h->rc.train = train;
  }
  return AP_OK;
}

int ap_render_rgba8(void* hp, uint32_t w, uint32_t hgt, uint32_t row_start, uint32_t row_end, int accumulate,
                    uint8_t* out, size_t out_bytes, ap_frame_stats* stats) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  if (row_start >= row_end || row_end > hgt) return fail(h, AP_E_INVALID, "bad row range");
  size_t need = (size_t)(row_end - row_start) * w * 4;
  if (!out || out_bytes < need) return fail(h, AP_E_INVALID, "output buffer too small");
  ap::DeviceScope device_scope(h->device);
  int rc = render_common(h, w, hgt, stats);
  if (rc) return rc;
  // lib.rs:349-352: a moved camera or accumulation off restarts the average
  if (!accumulate || std::memcmp(h->mats.view_proj, h->mats.prev_view_proj, sizeof(h->mats.view_proj)) != 0) {
    cudaMemsetAsync(h->fb.accum, 0, (size_t)w * hgt * sizeof(float4), h->stream);
    h->accum_count = 0;
  }
  encode_resolve_rgba8(h->fb, w, hgt, h->cfg.sample_count, h->accum_count, h->stream);
  h->accum_count += 1;  // SizedResources::end_frame (lib.rs:209-216)
  rc = check_cuda(h, cudaGetLastError(), "resolve");
  if (rc) return rc;
  rc = check_cuda(h, cudaMemcpyAsync(out, h->fb.rgba + (size_t)row_start * w, need, cudaMemcpyDeviceToHost, h->stream),
                  "readback");
  if (rc) return rc;
  return check_cuda(h, cudaStreamSynchronize(h->stream), "readback");
}

int ap_render_device(void* hp, uint32_t w, uint32_t hgt, ap_frame_stats* stats) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  ap::DeviceScope device_scope(h->device);
  return render_common(h, w, hgt, stats);
}

const float* ap_device_framebuffer(const void* hp) {
  const Handle* h = static_cast<const Handle*>(hp);
  return h ? h->fb.out_rgb : nullptr;
}

int ap_trace_rays(void* hp, const float* origins_tmax, const float* dirs, uint32_t n, int any_hit, uint32_t* out4) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  if (h->world.instances.empty()) {  // a world of instances is queried in its two-level form
    if (int wrc = world_sync(h)) return wrc;
    if (!h->scene.valid) return fail(h, AP_E_NO_SCENE, "no scene uploaded");
  }
  if (!origins_tmax || !dirs || !out4) return fail(h, AP_E_INVALID, "null buffer");
  if (n == 0) return AP_OK;
  ap::DeviceScope device_scope(h->device);
  const TwoLevel* tl = nullptr;
  if (int trc = two_level_sync(h, &tl)) return trc;
  size_t need = (size_t)n * 48 + 256;
  if (h->trace_bytes < need) {
    if (h->trace_mem) cudaFree(h->trace_mem);
    h->trace_mem = nullptr;
    int rc = check_cuda(h, cudaMalloc(&h->trace_mem, need), "trace scratch");
    if (rc) return rc;
    h->trace_bytes = need;
  }
  char* p = static_cast<char*>(h->trace_mem);
  float4* o = reinterpret_cast<float4*>(p);
  float4* dd = reinterpret_cast<float4*>(p + (size_t)n * 16);
  uint4* out = reinterpret_cast<uint4*>(p + (size_t)n * 32);
  uint32_t* cursor = reinterpret_cast<uint32_t*>(p + (size_t)n * 48);
  cudaMemcpyAsync(o, origins_tmax, (size_t)n * 16, cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(dd, dirs, (size_t)n * 16, cudaMemcpyHostToDevice, h->stream);
  launch_trace_batch(tl ? h->two_level.view : h->scene.view, o, dd, n, any_hit, out, cursor, h->num_sms, h->stream,
                     tl);
  int rc = check_cuda(h, cudaGetLastError(), "trace launch");
  if (rc) return rc;
  cudaMemcpyAsync(out4, out, (size_t)n * 16, cudaMemcpyDeviceToHost, h->stream);
  return check_cuda(h, cudaStreamSynchronize(h->stream), "trace");
}

int ap_read_buffer(void* hp, uint32_t which, uint32_t* out, size_t out_bytes) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !out) return AP_E_INVALID;
  if (!h->frame_mem) return fail(h, AP_E_INVALID, "no frame rendered");
  size_t P = (size_t)h->W * h->H;
  uint32_t cur = (h->frame_idx + 1) & 1u;  // parity of the last rendered frame
  ap::DeviceScope device_scope(h->device);
  struct Part { const void* ptr; size_t stride; };
  std::vector<Part> parts;
  size_t words = 0;
  switch (which) {
    case 0: parts = {{h->fb.radiance, 4}}; words = 1; break;
    case 1: parts = {{h->fb.payload, 16}}; words = 4; break;
    case 2: parts = {{h->fb.gb_a[cur], 16}, {h->fb.gb_b[cur], 16}}; words = 8; break;
    case 3: parts = {{h->fb.di_a, 16}, {h->fb.di_b, 16}}; words = 8; break;
    case 4: parts = {{h->fb.gi_a, 16}, {h->fb.gi_b, 16}}; words = 8; break;
    case 5: parts = {{h->fb.ctx, 16}}; words = 4; break;
    case 7: parts = {{h->fb.rays, 16}}; words = 4; break;
    case 8: parts = {{h->fb.hit_bsdf, 16}}; words = 4; break;
    case 9: parts = {{h->fb.hit_gi, 16}}; words = 4; break;
    case 10: parts = {{h->fb.rq_o[Q_GI_CAND], 16}, {h->fb.rq_d[Q_GI_CAND], 16}}; words = 8; break;
    case 11: parts = {{h->fb.st_a, 16}, {h->fb.st_b, 16}}; words = 8; break;
    case 12: parts = {{h->fb.st_c, 16}, {h->fb.st_d, 16}}; words = 8; break;
    default: return fail(h, AP_E_INVALID, "unknown buffer");
  }
  if (out_bytes < P * words * 4) return fail(h, AP_E_INVALID, "output buffer too small");
  size_t col = 0;
  for (const Part& pt : parts) {
    size_t pw = pt.stride / 4;
    int rc = check_cuda(h, cudaMemcpy2DAsync(out + col, words * 4, pt.ptr, pt.stride, pt.stride, P,
                                             cudaMemcpyDeviceToHost, h->stream),
                        "read buffer");
    if (rc) return rc;
    col += pw;
  }
  return check_cuda(h, cudaStreamSynchronize(h->stream), "read buffer");
}

int ap_profile_frame(void* hp, uint32_t w, uint32_t hgt, double* kind_ms, uint32_t* kind_count, const char** names,
                     uint32_t max_kinds, uint32_t* num_kinds, int count_visits, uint64_t* visits,
                     ap_frame_stats* stats) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !kind_ms || !kind_count || !num_kinds) return AP_E_INVALID;
  ap::DeviceScope device_scope(h->device);
  if (!h->prof.created) {
    for (int i = 0; i <= FrameProfiler::kMax; ++i)
      if (cudaEventCreate(&h->prof.ev[i]) != cudaSuccess) return fail(h, AP_E_CUDA, "profiler events");
    h->prof.created = true;
  }
  h->prof.count_visits = count_visits != 0;
  int rc = render_common(h, w, hgt, stats, &h->prof);
  h->prof.count_visits = false;
  if (rc) return rc;
  uint32_t nk = std::min<uint32_t>(max_kinds, (uint32_t)K_NUM_KINDS);
  if (visits) {
    std::vector<unsigned long long> v(3 * K_NUM_KINDS, 0ull);
    if (count_visits) {
      rc = check_cuda(h, cudaMemcpy(v.data(), h->fb.visits, v.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
                      "visits");
      if (rc) return rc;
    }
    for (uint32_t k = 0; k < 3 * nk; ++k) visits[k] = v[k];
  }
  for (uint32_t k = 0; k < nk; ++k) {
    kind_ms[k] = 0.0;
    kind_count[k] = 0;
    if (names) names[k] = kernel_kind_name((int)k);
  }
  for (int i = 0; i < h->prof.n; ++i) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, h->prof.ev[i], h->prof.ev[i + 1]);
    int k = h->prof.kind[i];
    if (k >= 0 && (uint32_t)k < nk) {
      kind_ms[k] += ms;
      kind_count[k] += 1;
    }
  }
  *num_kinds = nk;
  return AP_OK;
}

int ap_spectral_setup(void* hp, const float* sun_dir3, const float* sun_rgb3, float sun_scale, float scene_radius,
                      float env_scale) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !sun_dir3 || !sun_rgb3) return AP_E_INVALID;
  const bool two = !h->world.instances.empty();  // a world of instances renders in its two-level form
  const TwoLevel* tl = nullptr;
  if (two) {
    if (int trc = two_level_sync(h, &tl)) return trc;
  } else {
    if (int wrc = world_sync(h)) return wrc;
    if (!h->scene.valid) return fail(h, AP_E_NO_SCENE, "no scene uploaded");
  }
  if (!(scene_radius > 0.0f) || !(sun_scale >= 0.0f) || !(env_scale >= 0.0f) ||
      !(sun_dir3[0] * sun_dir3[0] + sun_dir3[1] * sun_dir3[1] + sun_dir3[2] * sun_dir3[2] > 0.0f))
    return fail(h, AP_E_INVALID, "spectral setup: bad light parameters");
  ap::DeviceScope device_scope(h->device);
  cudaStreamSynchronize(h->stream);
  h->spec_release();
  const DeviceScene& sc = h->scene;
  const float* mat26 = two ? reinterpret_cast<const float*>(h->two_level.materials.data()) : sc.host_materials.data();
  const uint32_t nm = two ? (uint32_t)h->two_level.materials.size() : (uint32_t)(sc.host_materials.size() / 26);
  std::vector<spec::Material> mats(nm);
  spec::upsample_materials(mat26, nm, mats.data());
  const std::vector<float>& env_rgb = two ? h->world.base.env : sc.host_env;
  const uint32_t env_w = two ? h->world.base.env_w : sc.view.env_w, env_h = two ? h->world.base.env_h : sc.view.env_h;
  const size_t texels = env_rgb.size() / 3;
  std::vector<float> env_pdf(texels);
  float env_integral = 0.0f;
  if (texels) spectral_env_distribution(env_rgb.data(), env_w, env_h, env_pdf.data(), &env_integral);
  int rc = check_cuda(h, cudaMalloc(&h->spec_mats, sizeof(spec::Material) * std::max<uint32_t>(nm, 1)), "spectral materials");
  if (!rc) rc = check_cuda(h, cudaMalloc(&h->spec_env, std::max<size_t>(sizeof(float) * texels, 16)), "spectral env");
  if (!rc) rc = check_cuda(h, cudaMemcpy(h->spec_mats, mats.data(), sizeof(spec::Material) * nm, cudaMemcpyHostToDevice),
                           "spectral materials");
  if (!rc && texels)
    rc = check_cuda(h, cudaMemcpy(h->spec_env, env_pdf.data(), sizeof(float) * texels, cudaMemcpyHostToDevice),
                    "spectral env");
  const spec::IlluminantTable& tab = spec::illuminant_table();
  if (!rc) rc = check_cuda(h, cudaMalloc(&h->spec_tab, sizeof(float) * tab.coef.size()), "spectral table");
  if (!rc)
    rc = check_cuda(h, cudaMemcpy(h->spec_tab, tab.coef.data(), sizeof(float) * tab.coef.size(), cudaMemcpyHostToDevice),
                    "spectral table");
  if (rc) {
    h->spec_release();
    return rc;
  }
  h->spec.mats = static_cast<const spec::Material*>(h->spec_mats);
  h->spec.env_pdf = static_cast<const float*>(h->spec_env);
  h->spec.env_pdf_integral = env_integral;
  h->spec.env_w = texels ? env_w : 0;
  h->spec.env_h = texels ? env_h : 0;
  h->spec.two_level = two ? 1 : 0;
  if (two) {
    h->spec.tl = *tl;
    h->spec.mg = h->two_level.mg;
  }
  h->spec_version = h->world.version;
  h->spec.env_scale = env_scale;
  h->spec.sun = spec::make_sun(sun_dir3, sun_rgb3, sun_scale, scene_radius);
  h->spec.illum_tab = static_cast<const float*>(h->spec_tab);
  h->spec.illum_norm = (float)spec::illuminant_norm();
  h->spec_ready = true;
  return AP_OK;
}

namespace {
int render_spectral(void* hp, uint32_t w, uint32_t hgt, uint32_t row_start, uint32_t row_end, uint32_t spp,
                    uint32_t max_depth, uint32_t seed, float* out_rgb, size_t out_bytes, ap_frame_stats* stats,
                    uint64_t* visits6) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h) return AP_E_INVALID;
  const bool two = !h->world.instances.empty();
  const TwoLevel* tl = nullptr;
  if (two) {
    if (int trc = two_level_sync(h, &tl)) return trc;
  } else {
    if (int wrc = world_sync(h)) return wrc;
    if (!h->scene.valid) return fail(h, AP_E_NO_SCENE, "no scene uploaded");
  }
  if (!h->spec_ready || h->spec_version != h->world.version)
    return fail(h, AP_E_INVALID, "spectral mode not set up for this world (ap_spectral_setup)");
  if (two && h->rc.cache) return fail(h, AP_E_UNSUPPORTED, "the radiance cache takes flat scenes (no spawned instances)");
  if (w == 0 || hgt == 0 || w > 65536 || row_start >= row_end || row_end > hgt || spp == 0 || max_depth == 0 ||
      max_depth > (uint32_t)kSpectralMaxDepth || (uint64_t)w * (row_end - row_start) > (1ull << 26))
    return fail(h, AP_E_INVALID, "spectral render: bad arguments");
  const size_t need = (size_t)(row_end - row_start) * w * 3 * sizeof(float);
  if (out_rgb && out_bytes < need) return fail(h, AP_E_INVALID, "output buffer too small");
  ap::DeviceScope device_scope(h->device);
  // the image, then the wavefront's work area
  const uint32_t P = w * (row_end - row_start);
  SpectralCache cache_mode{};
  const SpectralCache* rcp = nullptr;
  if (h->rc.cache) {  // radiance-cache mode (ap_rc_attach)
    cache_mode = SpectralCache{h->rc.cache, h->rc.prefix, h->rc.stride, h->rc.batch, h->rc.lr, h->rc.train};
    rcp = &cache_mode;
  }
  const size_t need_a = (need + 255) & ~(size_t)255;
  const size_t total = need_a + spectral_work_bytes(P, rcp);
  if (h->spec_out_bytes < total) {
    if (h->spec_out) cudaFree(h->spec_out);
    h->spec_out = nullptr;
    h->spec_out_bytes = 0;
    int rc = check_cuda(h, cudaMalloc(&h->spec_out, total), "spectral buffers");
    if (rc) return rc;
    h->spec_out_bytes = total;
  }
  compute_mats(h, w, hgt);
  SpectralCamera cam;
  std::memcpy(cam.inv_view, h->mats.inv_view, sizeof(cam.inv_view));
  std::memcpy(cam.inv_proj, h->mats.inv_proj, sizeof(cam.inv_proj));
  void* work = static_cast<char*>(h->spec_out) + need_a;
  const unsigned long long* counter = spectral_stats(work, P, rcp);
  cudaEventRecord(h->ev0, h->stream);
  const int launches = launch_spectral(two ? h->two_level.view : h->scene.view, h->spec, cam, w, hgt, row_start,
                                       row_end, spp, (int)max_depth,
                                       seed, static_cast<float*>(h->spec_out), work, h->num_sms, visits6 != nullptr,
                                       rcp, h->stream, &h->fs);
  cudaEventRecord(h->ev1, h->stream);
  int rc = check_cuda(h, cudaGetLastError(), "spectral launch");
  if (rc) return rc;
  unsigned long long cnt[6] = {0, 0, 0, 0, 0, 0};
  rc = check_cuda(h, cudaMemcpyAsync(cnt, counter, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream), "ray count");
  if (rc) return rc;
  if (out_rgb) {
    rc = check_cuda(h, cudaMemcpyAsync(out_rgb, h->spec_out, need, cudaMemcpyDeviceToHost, h->stream), "spectral readback");
    if (rc) return rc;
  }
  rc = check_cuda(h, cudaStreamSynchronize(h->stream), "spectral render");
  if (rc) return rc;
  if (rcp) {
    std::string msg;
    if ((rc = rc_take_status(rcp->cache, &msg))) return fail(h, rc, "radiance cache: " + msg);
  }
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->gpu_ms = ms;
    stats->extension_rays = cnt[0] + cnt[3];
    stats->kernel_launches = (uint32_t)launches;
    stats->width = w;
    stats->height = hgt;
    stats->frame_idx = h->frame_idx;
  }
  if (visits6)
    for (int i = 0; i < 6; ++i) visits6[i] = cnt[i];
  return AP_OK;
}
}  // namespace

int ap_render_spectral(void* hp, uint32_t w, uint32_t hgt, uint32_t row_start, uint32_t row_end, uint32_t spp,
                       uint32_t max_depth, uint32_t seed, float* out_rgb, size_t out_bytes, ap_frame_stats* stats) {
  return render_spectral(hp, w, hgt, row_start, row_end, spp, max_depth, seed, out_rgb, out_bytes, stats, nullptr);
}

int ap_profile_spectral(void* hp, uint32_t w, uint32_t hgt, uint32_t row_start, uint32_t row_end, uint32_t spp,
                        uint32_t max_depth, uint32_t seed, uint64_t* visits6, ap_frame_stats* stats) {
  if (!visits6) return AP_E_INVALID;
  return render_spectral(hp, w, hgt, row_start, row_end, spp, max_depth, seed, nullptr, 0, stats, visits6);
}

int ap_bvh_stats(void* hp, uint32_t* out8) {
  Handle* h = static_cast<Handle*>(hp);
  if (!h || !out8) return AP_E_INVALID;
  if (int wrc = world_sync(h)) return wrc;
  if (!h->scene.valid) return fail(h, AP_E_NO_SCENE, "no scene uploaded");
  const BvhStats& s = h->scene.stats;
  out8[0] = s.num_nodes;
  out8[1] = s.num_tris;
  out8[2] = s.max_depth;
  out8[3] = s.max_stack;
  std::memcpy(&out8[4], &s.build_ms, 8);
  out8[6] = 0;
  out8[7] = 0;
  return AP_OK;
}

}  // extern "C"
