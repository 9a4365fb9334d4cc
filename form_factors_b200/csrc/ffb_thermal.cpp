// ffb_thermal.cpp -- the reference's two ray-traced thermal equations on the
// B200 path (include/ffb.h):
//   * the radiance equation (thermal_equation/radiance_cpu.cpp:96-190):
//     Malley emission weighted by temperature and emissivity, every hit
//     absorbed by the hit face's mesh;
//   * the distant source of parallel rays (thermal_equation/parallel_rays_cpu.cpp:66-131):
//     a disc of parallel rays in front of the scene's bounding sphere, every
//     hit absorbed by the hit face's mesh with the absorbance of the side hit.
// The host arithmetic -- face areas, emission weights and ray budgets,
// per-ray powers, the bounding sphere -- follows the reference operation for
// operation in float; the rays are emitted, traced and tallied on the GPU
// (ffb_radiance_absorption, ffb_parallel_rays).  Sums over rays are exact
// (integer counts, or integers in 64-bit fixed point) and rounded to float
// once, where the reference adds one float per ray.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ffb.h"

int ffb_set_error(int code, const char* msg);  // ffb_api.cu: records the message for ffb_last_error

namespace {

const float kSigma = 5.670400e-8f;  // thermal_equation/radiance_cpu.cpp:28

// math::triangle_area (math/triangle.cpp:86-92)
float triangle_area(const float* t)
{
  const float vx = t[3] - t[0], vy = t[4] - t[1], vz = t[5] - t[2];
  const float wx = t[6] - t[0], wy = t[7] - t[1], wz = t[8] - t[2];
  const float nx = vy * wz - vz * wy, ny = vz * wx - vx * wz, nz = vx * wy - vy * wx;
  return sqrtf(nx * nx + ny * ny + nz * nz) / 2;
}

// malley_emission::emitted_front / emitted_rear (emission/malley_emission.cpp:50-60)
int emitted(int n_rays, float weight, float total_weight)
{
  return weight > 0 ? std::max<int>(1, (int)(n_rays * (weight / total_weight))) : 0;
}

// subject::build_face_to_mesh_index (subject/system.cpp:93-108); every face
// must belong to exactly one mesh here (the reference leaves the entry of a
// face outside every mesh unset).
int face_to_mesh(int n_faces, const ffb_mesh* meshes, int n_meshes, std::vector<int32_t>& out)
{
  out.assign((size_t)n_faces, -1);
  for (int m = 0; m < n_meshes; ++m) {
    const ffb_mesh& mesh = meshes[m];
    if (mesh.first_idx < 0 || mesh.n_faces < 0 || mesh.first_idx + mesh.n_faces > n_faces)
      return FFB_ERR_ARG;
    for (int f = mesh.first_idx; f < mesh.first_idx + mesh.n_faces; ++f) {
      if (out[(size_t)f] >= 0)
        return FFB_ERR_ARG;
      out[(size_t)f] = m;
    }
  }
  for (int f = 0; f < n_faces; ++f)
    if (out[(size_t)f] < 0)
      return FFB_ERR_ARG;
  return FFB_OK;
}

int check_materials(const ffb_mesh* meshes, int n_meshes, int n_materials)
{
  for (int m = 0; m < n_meshes; ++m)
    if (meshes[m].material_idx < 0 || meshes[m].material_idx >= n_materials)
      return FFB_ERR_ARG;
  return FFB_OK;
}

}  // namespace

extern "C" int ffb_bounding_sphere(const float* faces9, int n_faces, float* center3, float* radius)
{
  if (!faces9 || n_faces <= 0 || !center3 || !radius)
    return FFB_ERR_ARG;
  // math::triangles_bsphere (math/triangle.cpp:361-384)
  float cx = 0, cy = 0, cz = 0;
  for (int i = 0; i < n_faces; ++i) {
    const float* t = faces9 + 9 * (size_t)i;
    // triangle_center: (p0 + p1 + p2) / 3.f, math/triangle.cpp:81-84
    cx += ((t[0] + t[3]) + t[6]) / 3.f;
    cy += ((t[1] + t[4]) + t[7]) / 3.f;
    cz += ((t[2] + t[5]) + t[8]) / 3.f;
  }
  // vec3 /= float multiplies by the reciprocal (math/operations.h:144-150)
  const float inv = 1.f / (float)n_faces;
  cx *= inv;
  cy *= inv;
  cz *= inv;
  float r = 0;
  for (int i = 1; i < n_faces; ++i) {  // the reference starts at 1
    const float* t = faces9 + 9 * (size_t)i;
    for (int k = 0; k < 3; ++k) {
      const float dx = cx - t[3 * k], dy = cy - t[3 * k + 1], dz = cz - t[3 * k + 2];
      const float d = sqrtf(dx * dx + dy * dy + dz * dz);
      if (d > r)
        r = d;
    }
  }
  center3[0] = cx;
  center3[1] = cy;
  center3[2] = cz;
  *radius = r;
  return FFB_OK;
}

extern "C" int ffb_radiance_step(ffb_ctx* ctx, const float* faces9, int n_faces, const ffb_mesh* meshes, int n_meshes,
                                 const ffb_optics* materials, int n_materials, const float* temperatures, int n_rays,
                                 uint64_t seed, uint32_t epoch, int flags, float* emission, float* absorption)
{
  if (!faces9 || n_faces <= 0 || !meshes || n_meshes <= 0 || !materials || !temperatures || !emission ||
      !absorption || n_rays < 0)
    return ffb_set_error(FFB_ERR_ARG, "bad radiance step arguments");
  if (check_materials(meshes, n_meshes, n_materials) < 0)
    return ffb_set_error(FFB_ERR_ARG, "mesh material index out of range");
  std::vector<int32_t> f2m;
  if (face_to_mesh(n_faces, meshes, n_meshes, f2m) < 0)
    return ffb_set_error(FFB_ERR_ARG, "meshes must cover every face exactly once");
  std::vector<float> area((size_t)n_faces);
  for (int f = 0; f < n_faces; ++f)
    area[(size_t)f] = triangle_area(faces9 + 9 * (size_t)f);
  // calculate_weights (radiance_cpu.cpp:96-123): density T (not T^4) times emissivity and area
  std::vector<float> w(2 * (size_t)n_faces, 0.f);
  float total = 0;
  for (int m = 0; m < n_meshes; ++m) {
    const ffb_optics& mat = materials[meshes[m].material_idx];
    const float density = temperatures[m];
    const float front_density = density * mat.front_emissivity;
    const float rear_density = density * mat.rear_emissivity;
    for (int f = meshes[m].first_idx; f != meshes[m].first_idx + meshes[m].n_faces; ++f) {
      const float front = front_density * area[(size_t)f];
      const float rear = rear_density * area[(size_t)f];
      total += front + rear;
      w[2 * (size_t)f] = front;
      w[2 * (size_t)f + 1] = rear;
    }
  }
  std::vector<int32_t> front_rays((size_t)n_faces), rear_rays((size_t)n_faces);
  for (int f = 0; f < n_faces; ++f) {
    front_rays[(size_t)f] = emitted(n_rays, w[2 * (size_t)f], total);
    rear_rays[(size_t)f] = emitted(n_rays, w[2 * (size_t)f + 1], total);
  }
  // emission and per-ray powers (radiance_cpu.cpp:149-175)
  std::vector<float> power_front((size_t)n_faces, 0.f), power_rear((size_t)n_faces, 0.f);
  for (int m = 0; m < n_meshes; ++m) {
    const ffb_optics& mat = materials[meshes[m].material_idx];
    const float T = temperatures[m];
    const float power_density = kSigma * (T * T * T * T);
    const float front_density = power_density * mat.front_emissivity;
    const float rear_density = power_density * mat.rear_emissivity;
    for (int f = meshes[m].first_idx; f != meshes[m].first_idx + meshes[m].n_faces; ++f) {
      const float front_emission = front_density * area[(size_t)f];
      const float rear_emission = rear_density * area[(size_t)f];
      emission[m] += front_emission + rear_emission;
      if (front_rays[(size_t)f] > 0)
        power_front[(size_t)f] = front_emission / front_rays[(size_t)f];
      if (rear_rays[(size_t)f] > 0)
        power_rear[(size_t)f] = rear_emission / rear_rays[(size_t)f];
    }
  }
  std::vector<double> absorbed((size_t)n_meshes);
  const int rc = ffb_radiance_absorption(ctx, front_rays.data(), rear_rays.data(), power_front.data(),
                                         power_rear.data(), f2m.data(), n_meshes, seed, epoch, flags,
                                         absorbed.data());
  if (rc < 0)
    return rc;
  for (int m = 0; m < n_meshes; ++m)
    absorption[m] += (float)absorbed[(size_t)m];
  return FFB_OK;
}

extern "C" int ffb_distant_source_step(ffb_ctx* ctx, const float* faces9, int n_faces, const ffb_mesh* meshes,
                                       int n_meshes, const ffb_optics* materials, int n_materials, int n_rays,
                                       float power, const float* direction3, uint64_t seed, uint32_t epoch,
                                       float* absorption)
{
  if (!faces9 || n_faces <= 0 || !meshes || n_meshes <= 0 || !materials || !direction3 || !absorption || n_rays <= 0)
    return ffb_set_error(FFB_ERR_ARG, "bad distant-source step arguments");
  if (check_materials(meshes, n_meshes, n_materials) < 0)
    return ffb_set_error(FFB_ERR_ARG, "mesh material index out of range");
  std::vector<int32_t> f2m;
  if (face_to_mesh(n_faces, meshes, n_meshes, f2m) < 0)
    return ffb_set_error(FFB_ERR_ARG, "meshes must cover every face exactly once");
  // the disc in front of the bounding sphere (parallel_rays_cpu.cpp:96-101)
  float center[3], bradius;
  int rc = ffb_bounding_sphere(faces9, n_faces, center, &bradius);
  if (rc < 0)
    return ffb_set_error(rc, "bounding sphere");
  const float radius = bradius * 1.1f;
  ffb_disc_source src;
  for (int k = 0; k < 3; ++k) {
    src.direction[k] = direction3[k];
    src.center[k] = center[k];
  }
  src.distance = 1.1f + radius;
  src.radius = radius;
  std::vector<uint32_t> side((size_t)2 * n_faces);
  rc = ffb_parallel_rays(ctx, &src, n_rays, seed, epoch, side.data());
  if (rc < 0)
    return rc;
  // ray power and the absorbed sums (parallel_rays_cpu.cpp:108-122)
  const float ray_power = power * (float(M_PI) * radius * radius) / n_rays;
  std::vector<double> absorbed((size_t)n_meshes, 0.0);
  for (int f = 0; f < n_faces; ++f) {
    const ffb_optics& mat = materials[meshes[f2m[(size_t)f]].material_idx];
    absorbed[(size_t)f2m[(size_t)f]] += (double)side[2 * (size_t)f] * (double)(mat.front_absorbance * ray_power) +
                                         (double)side[2 * (size_t)f + 1] * (double)(mat.rear_absorbance * ray_power);
  }
  for (int m = 0; m < n_meshes; ++m)
    absorption[m] += (float)absorbed[(size_t)m];
  return FFB_OK;
}
