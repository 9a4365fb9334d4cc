// ref_shim.cpp -- extern "C" entry points into the reference's own CPU code.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with the
// reference's CPU sources (compiled where they lie, never copied) into
// oracle/_ref/libffref.so.  Tests use it to pin the oracle restatement
// (oracle/ffo.c) and to produce golden vectors; bench.py's reference arm uses
// it to time the reference's zgrid_cpu path on the host cores.
//
// Reference interfaces called here:
//   ray_caster::system_create / set_scene / prepare / cast   ray_caster/system.cpp:65-126
//   emission::system_create / set_scene / calculate          emission/system.cpp:29-75
//   malley_emission::emitted_front / emitted_rear           emission/malley_emission.cpp:50-60
//   form_factors::system_create / set_scene / prepare / calculate  form_factors/system.cpp:45-106
//   math::triangle_intersect                                  math/triangle.cpp:28-79
//   math::rotate_towards                                      math/mat.cpp:25-49
//   csv_export::export_csv                                    import_export/csv_export.cpp:26-46
//   radiance_equation::system_create / calculate              thermal_equation/radiance_cpu.cpp:96-190
//   parallel_rays_cpu::system_create / calculate              thermal_equation/parallel_rays_cpu.cpp:66-131
//   parallel_rays_emission_cpu::system_create                 emission/parallel_rays_cpu.cpp:88-138
//   math::triangles_bsphere                                   math/triangle.cpp:361-384
//   obj_import::scene                                         import_export/obj_import.cpp:167-340
#include "ray_caster/system.h"
#include "import_export/csv_export.h"
#include "subject/system.h"
#include "thermal_equation/system.h"
#include "thermal_equation/radiance_cpu.h"
#include "thermal_equation/parallel_rays_cpu.h"
#include "emission/parallel_rays_cpu.h"
#include "import_export/obj_import.h"
#include "emission/system.h"
#include "emission/malley_emission.h"
#include "form_factors/system.h"
#include "math/triangle.h"
#include "math/mat.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

// ray_caster/system.cpp:25,74-83 links the two CUDA caster factories; the
// CUDA sources are not built for the oracle, so both report "unavailable".
namespace naive_cuda_ray_caster { ray_caster::system_t* system_create() { return 0; } }
namespace zgrid_cuda_ray_caster { ray_caster::system_t* system_create() { return 0; } }

namespace
{
  // A caster that does nothing: lets the reference emission produce its ray
  // batch without casting it.
  int null_init(ray_caster::system_t*) { return 0; }
  int null_shutdown(ray_caster::system_t*) { return 0; }
  int null_set_scene(ray_caster::system_t*, ray_caster::scene_t*) { return 0; }
  int null_prepare(ray_caster::system_t*) { return 0; }
  int null_cast(ray_caster::system_t*, ray_caster::task_t* t)
  {
    for (int i = 0; i < t->n_tasks; ++i) t->hit_face[i] = 0;
    return 0;
  }
  const ray_caster::system_methods_t null_methods = {null_init, null_shutdown, null_set_scene,
                                                     null_prepare, null_cast};

  double now_s()
  {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }

  // Casts rays [0, n) of `task` on `n_threads` threads that take slices of
  // 2048 rays from a shared cursor (the reference casters keep no per-cast
  // state, so slices are independent; dynamic slices keep every core busy
  // when ray cost varies across the batch).
  int cast_threads(ray_caster::system_t* sys, ray_caster::task_t* task, int n_threads)
  {
    if (n_threads <= 1)
      return ray_caster::system_cast(sys, task);
    const long n = task->n_tasks;
    const long slice = 2048;
    std::atomic<long> cursor(0);
    std::atomic<int> status(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < n_threads; ++t) {
      pool.emplace_back([&]() {
        for (;;) {
          long b = cursor.fetch_add(slice);
          if (b >= n) break;
          long e = std::min(n, b + slice);
          ray_caster::task_t sub = {(int)(e - b), task->ray + b, task->hit_face + b, task->hit_point + b};
          int r = ray_caster::system_cast(sys, &sub);
          if (r < 0) status = r;
        }
      });
    }
    for (auto& th : pool) th.join();
    return status.load();
  }
}

extern "C" {

int ffref_triangle_intersect(const float* ray6, const float* tri9, float* point3)
{
  math::ray_t ray;
  std::memcpy(&ray, ray6, sizeof ray);
  math::triangle_t tri;
  std::memcpy(&tri, tri9, sizeof tri);
  math::vec3 p = {0, 0, 0};
  int r = math::triangle_intersect(ray, tri, &p);
  point3[0] = p.x; point3[1] = p.y; point3[2] = p.z;
  return r;
}

void ffref_rotate_towards(const float* s3, const float* t3, float* m9)
{
  math::mat33 m = math::rotate_towards(math::make_vec3(s3[0], s3[1], s3[2]),
                                       math::make_vec3(t3[0], t3[1], t3[2]));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m9[3 * i + j] = m.p[i][j];
}

int ffref_emitted(int n_rays, float weight, float total_weight)
{
  float w[2] = {weight, weight};
  malley_emission::task_t task(n_rays, total_weight, w);
  return malley_emission::emitted_front(&task, 0);
}

// Casts a ray batch with reference caster `type` (1 naive_cpu, 3 zgrid_cpu).
// hit[i] = face index or -1.  hit_pt is written for hits only.  Returns the
// reference status; *prepare_s / *cast_s receive wall seconds when non-null.
int ffref_cast(int type, int n_faces, const float* faces9, long n_rays, const float* rays6,
               int32_t* hit, float* hit_pt, int n_threads, double* prepare_s, double* cast_s)
{
  ray_caster::system_t* sys = ray_caster::system_create(type);
  if (!sys) return -1000;
  ray_caster::scene_t scene = {n_faces, (math::triangle_t*)faces9};
  double t0 = now_s();
  int r = ray_caster::system_set_scene(sys, &scene);
  if (r >= 0) r = ray_caster::system_prepare(sys);
  double t1 = now_s();
  if (r < 0) { ray_caster::system_free(sys); return r; }
  std::vector<math::triangle_t*> hf((size_t)n_rays, nullptr);
  std::vector<math::vec3> hp((size_t)n_rays);
  if (hit_pt)
    std::memcpy(hp.data(), hit_pt, sizeof(float) * 3 * (size_t)n_rays);
  ray_caster::task_t task = {(int)n_rays, (math::ray_t*)rays6, hf.data(), hp.data()};
  r = cast_threads(sys, &task, n_threads);
  double t2 = now_s();
  for (long i = 0; i < n_rays; ++i)
    hit[i] = hf[i] ? (int32_t)(hf[i] - scene.faces) : -1;
  if (hit_pt)
    std::memcpy(hit_pt, hp.data(), sizeof(float) * 3 * (size_t)n_rays);
  if (prepare_s) *prepare_s = t1 - t0;
  if (cast_s) *cast_s = t2 - t1;
  ray_caster::system_free(sys);
  return r;
}

// Reference Malley emission (malley_cpu, mt19937 seeds 1..4) for per-face
// weights weights2[2*f] (front) and weights2[2*f+1] (rear).  Writes up to
// `cap` rays and returns the batch size (negative on error).  The emitter is
// created fresh, so its generators restart from their seeds each call.
long ffref_emit(int n_faces, const float* faces9, int n_rays, const float* weights2,
                float total_weight, float* rays6, long cap)
{
  ray_caster::system_t null_caster = {&null_methods};
  emission::system_t* em = emission::system_create(EMISSION_MALLEY_CPU, &null_caster);
  ray_caster::scene_t scene = {n_faces, (math::triangle_t*)faces9};
  int r = emission::system_set_scene(em, &scene);
  if (r < 0) { emission::system_free(em); return r; }
  std::vector<float> w(weights2, weights2 + 2 * (size_t)n_faces);
  malley_emission::task_t task(n_rays, total_weight, w.data());
  r = emission::system_calculate(em, &task);
  long n = 0;
  if (r >= 0 && task.rays) {
    n = task.rays->n_tasks;
    long m = n < cap ? n : cap;
    if (rays6) std::memcpy(rays6, task.rays->ray, sizeof(float) * 6 * (size_t)m);
  }
  ray_caster::task_free(task.rays);
  emission::system_free(em);
  return r < 0 ? r : n;
}

// The reference form-factor calculator end to end (cpu_form_factors +
// malley_cpu + caster `caster_type`).  meshes3 holds {first_idx, n_faces, pad}
// per mesh; ff_out receives n_meshes^2 floats.  `n_calls` > 1 repeats
// set_scene/prepare/calculate on the same systems (the reference's
// total_area then keeps accumulating, cpu_system.cpp:126).
int ffref_form_factors(int n_faces, const float* faces9, int n_meshes, const int32_t* meshes3,
                       int n_rays, int caster_type, int n_calls, float* ff_out)
{
  ray_caster::system_t* rc = ray_caster::system_create(caster_type);
  if (!rc) return -1000;
  emission::system_t* em = emission::system_create(EMISSION_MALLEY_CPU, rc);
  form_factors::system_t* ff = form_factors::system_create(FORM_FACTORS_CPU, em);
  form_factors::scene_t scene = {n_faces, (math::triangle_t*)faces9, n_meshes,
                                 (form_factors::mesh_t*)meshes3};
  int r = 0;
  for (int c = 0; c < n_calls && r >= 0; ++c) {
    r = form_factors::system_set_scene(ff, &scene);
    if (r >= 0) r = form_factors::system_prepare(ff);
    form_factors::task_t task = {n_rays, ff_out};
    if (r >= 0) r = form_factors::system_calculate(ff, &task);
  }
  form_factors::system_free(ff);
  emission::system_free(em);
  ray_caster::system_free(rc);
  return r;
}

// One timed step of the reference path for a bounded sample: the reference
// Malley emission of the faces flagged in `sample_mask` (the others get zero
// weight, total weight unchanged, so each sampled face emits exactly as many
// rays as in a full run), the reference zgrid_cpu cast of that batch on
// `n_threads` threads over disjoint slices, and the per-(source, hit) count
// of cpu_system.cpp:167-196 (per-face meshes).  The grid is built once in
// ffref_step_open.  Returns the number of rays cast.
struct ffref_step_t
{
  ray_caster::system_t* caster;
  ray_caster::scene_t scene;
  std::vector<float> faces;
};

void* ffref_step_open(int caster_type, int n_faces, const float* faces9, double* prepare_s)
{
  ffref_step_t* s = new ffref_step_t;
  s->faces.assign(faces9, faces9 + 9 * (size_t)n_faces);
  s->scene = {n_faces, (math::triangle_t*)s->faces.data()};
  s->caster = ray_caster::system_create(caster_type);
  if (!s->caster) { delete s; return 0; }
  double t0 = now_s();
  ray_caster::system_set_scene(s->caster, &s->scene);
  if (ray_caster::system_prepare(s->caster) < 0) {
    ray_caster::system_free(s->caster);
    delete s;
    return 0;
  }
  if (prepare_s) *prepare_s = now_s() - t0;
  return s;
}

long ffref_step_run(void* handle, int n_rays, const float* weights2, float total_weight,
                    const uint8_t* sample_mask, int n_threads, uint32_t* counts_sparse_src,
                    double* emit_s, double* cast_s)
{
  ffref_step_t* s = (ffref_step_t*)handle;
  const int n = s->scene.n_faces;
  std::vector<float> w(2 * (size_t)n);
  for (int f = 0; f < n; ++f) {
    w[2 * f] = sample_mask[f] ? weights2[2 * f] : 0.f;
    w[2 * f + 1] = sample_mask[f] ? weights2[2 * f + 1] : 0.f;
  }
  double t0 = now_s();
  ray_caster::system_t null_caster = {&null_methods};
  emission::system_t* em = emission::system_create(EMISSION_MALLEY_CPU, &null_caster);
  emission::system_set_scene(em, &s->scene);
  malley_emission::task_t task(n_rays, total_weight, w.data());
  emission::system_calculate(em, &task);
  double t1 = now_s();
  long n_cast = 0;
  if (task.rays) {
    n_cast = task.rays->n_tasks;
    cast_threads(s->caster, task.rays, n_threads);
    // count hits per sampled source face, in emission order
    long k = 0;
    for (int f = 0; f < n; ++f) {
      int nf = malley_emission::emitted_front(&task, f) + malley_emission::emitted_rear(&task, f);
      for (int j = 0; j < nf && k < n_cast; ++j, ++k) {
        math::triangle_t* h = task.rays->hit_face[k];
        if (h && counts_sparse_src) counts_sparse_src[h - s->scene.faces] += 1;
      }
    }
  }
  double t2 = now_s();
  if (emit_s) *emit_s = t1 - t0;
  if (cast_s) *cast_s = t2 - t1;
  ray_caster::task_free(task.rays);
  task.rays = 0;
  emission::system_free(em);
  return n_cast;
}

// A subject scene: meshes3 = (first, count, material) per mesh; optics4 =
// (front emissivity, rear emissivity, front absorbance, rear absorbance)
// per material, the other properties those of the reference's black body.
static subject::scene_t make_subject(int n_faces, const float* faces9, int n_meshes, const int* meshes3,
                                     int n_materials, const float* optics4, std::vector<subject::mesh_t>& meshes,
                                     std::vector<subject::material_t>& materials)
{
  meshes.resize(n_meshes);
  for (int m = 0; m < n_meshes; ++m)
    meshes[m] = subject::make_mesh(meshes3[3 * m], meshes3[3 * m + 1], meshes3[3 * m + 2]);
  materials.resize(n_materials);
  for (int k = 0; k < n_materials; ++k) {
    materials[k] = subject::black_body();
    materials[k].front.emissivity = optics4[4 * k];
    materials[k].rear.emissivity = optics4[4 * k + 1];
    materials[k].front.absorbance = optics4[4 * k + 2];
    materials[k].rear.absorbance = optics4[4 * k + 3];
  }
  subject::scene_t s;
  s.n_faces = n_faces;
  s.faces = (subject::face_t*)faces9;
  s.n_meshes = n_meshes;
  s.meshes = meshes.data();
  s.n_materials = n_materials;
  s.materials = materials.data();
  return s;
}

// One calculate() of the reference's radiance equation with malley_cpu over
// caster `type`: emission and absorption per mesh (added to zeros).
int ffref_radiance(int type, int n_faces, const float* faces9, int n_meshes, const int* meshes3, int n_materials,
                   const float* optics4, const float* temperatures, int n_rays, float* emission_out,
                   float* absorption_out)
{
  std::vector<subject::mesh_t> meshes;
  std::vector<subject::material_t> materials;
  subject::scene_t scene = make_subject(n_faces, faces9, n_meshes, meshes3, n_materials, optics4, meshes, materials);
  ray_caster::system_t* caster = ray_caster::system_create(type);
  emission::system_t* emitter = emission::system_create(EMISSION_MALLEY_CPU, caster);
  radiance_equation::params_t params = {emitter, n_rays};
  // the factory (thermal_equation/factory.cpp) would pull in every equation type
  thermal_equation::system_t* eq = radiance_equation::system_create();
  int r = thermal_equation::system_init(eq, &params);
  if (r >= 0)
    r = thermal_equation::system_set_scene(eq, &scene);
  std::memset(emission_out, 0, sizeof(float) * n_meshes);
  std::memset(absorption_out, 0, sizeof(float) * n_meshes);
  if (r >= 0) {
    thermal_equation::task_t task = {temperatures, emission_out, absorption_out};
    r = thermal_equation::system_calculate(eq, &task);
  }
  thermal_equation::system_free(eq);
  emission::system_free(emitter);
  ray_caster::system_free(caster);
  return r;
}

struct ffref_source_param {
  float power;
  float direction[3];
};

static parallel_rays_cpu::source_t ffref_source(void* param)
{
  const ffref_source_param* p = (const ffref_source_param*)param;
  parallel_rays_cpu::source_t s;
  s.power = p->power;
  s.direction = math::make_vec3(p->direction[0], p->direction[1], p->direction[2]);
  return s;
}

// One calculate() of the reference's distant-source (parallel rays)
// equation: absorbed power per mesh.
int ffref_parallel_rays(int type, int n_faces, const float* faces9, int n_meshes, const int* meshes3,
                        int n_materials, const float* optics4, int n_rays, float power, const float* direction3,
                        float* absorption_out)
{
  std::vector<subject::mesh_t> meshes;
  std::vector<subject::material_t> materials;
  subject::scene_t scene = make_subject(n_faces, faces9, n_meshes, meshes3, n_materials, optics4, meshes, materials);
  ray_caster::system_t* caster = ray_caster::system_create(type);
  emission::system_t* emitter = emission::system_create(EMISSION_PARALLEL_RAYS_CPU, caster);
  ffref_source_param sp = {power, {direction3[0], direction3[1], direction3[2]}};
  parallel_rays_cpu::params_t params = {n_rays, emitter, &sp, &ffref_source};
  thermal_equation::system_t* eq = parallel_rays_cpu::system_create();
  int r = thermal_equation::system_init(eq, &params);
  if (r >= 0)
    r = thermal_equation::system_set_scene(eq, &scene);
  std::memset(absorption_out, 0, sizeof(float) * n_meshes);
  if (r >= 0) {
    std::vector<float> em(n_meshes, 0.f);
    std::vector<float> temps(n_meshes, 0.f);
    thermal_equation::task_t task = {temps.data(), em.data(), absorption_out};
    r = thermal_equation::system_calculate(eq, &task);
  }
  thermal_equation::system_free(eq);
  emission::system_free(emitter);
  ray_caster::system_free(caster);
  return r;
}

// obj_import::scene: status, and on success the scene (release with
// ffref_obj_free); counts3 = faces, meshes, materials.
int ffref_obj_load(const char* filename, void** scene_out, int* counts3)
{
  subject::scene_t* scene = 0;
  const int r = obj_import::scene(filename, &scene);
  *scene_out = scene;
  if (r == 0 && scene) {
    counts3[0] = scene->n_faces;
    counts3[1] = scene->n_meshes;
    counts3[2] = scene->n_materials;
  }
  return r;
}

void ffref_obj_copy(void* handle, float* faces9, int* meshes3, void* materials)
{
  subject::scene_t* s = (subject::scene_t*)handle;
  std::memcpy(faces9, s->faces, sizeof(subject::face_t) * (size_t)s->n_faces);
  std::memcpy(meshes3, s->meshes, sizeof(subject::mesh_t) * (size_t)s->n_meshes);
  std::memcpy(materials, s->materials, sizeof(subject::material_t) * (size_t)s->n_materials);
}

void ffref_obj_free(void* handle) { subject::scene_free((subject::scene_t*)handle); }

void ffref_bsphere(int n_faces, const float* faces9, float* center3, float* radius)
{
  math::sphere_t s = math::triangles_bsphere((const math::triangle_t*)faces9, n_faces);
  center3[0] = s.center.x;
  center3[1] = s.center.y;
  center3[2] = s.center.z;
  *radius = s.radius;
}

// The reference's CSV export of an n x n matrix (n meshes, row-major floats).
int ffref_export_csv(const char* filename, int n, const float* ff)
{
  form_factors::scene_t scene;
  scene.n_faces = 0;
  scene.faces = 0;
  scene.n_meshes = n;
  scene.meshes = 0;
  form_factors::task_t task;
  task.n_rays = 0;
  task.form_factors = const_cast<float*>(ff);
  return csv_export::export_csv(filename, &scene, &task);
}

void ffref_step_close(void* handle)
{
  ffref_step_t* s = (ffref_step_t*)handle;
  if (!s) return;
  ray_caster::system_free(s->caster);
  delete s;
}

}  // extern "C"
