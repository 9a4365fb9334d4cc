// ffb_systems.cpp -- the B200 ray caster, emission and form-factor systems
// behind the reference's C-style vtables (include/ffb_systems.h), on top of
// the C ABI of include/ffb.h.
//
// Host arithmetic that decides how many rays a face emits and how a matrix
// row is normalised is written with the reference's float operations in the
// reference's order (compiled with -ffp-contract=off), so that the same
// inputs spend the same rays and produce the same normalisation.
#include "ffb_systems.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ffb.h"

namespace {

// malley_emission::emitted_front / emitted_rear (emission/malley_emission.cpp:50-60).
int emitted(int n_rays, float weight, float total_weight)
{
  return weight > 0 ? std::max<int>(1, (int)(n_rays * (weight / total_weight))) : 0;
}

// math::triangle_area (math/triangle.cpp:86-92).
float triangle_area(const math::triangle_t& t)
{
  const math::vec3 a = t.points[0], b = t.points[1], c = t.points[2];
  const float vx = b.x - a.x, vy = b.y - a.y, vz = b.z - a.z;
  const float wx = c.x - a.x, wy = c.y - a.y, wz = c.z - a.z;
  const float nx = vy * wz - vz * wy, ny = vz * wx - vx * wz, nz = vx * wy - vy * wx;
  return sqrtf(nx * nx + ny * ny + nz * nz) / 2;
}

int device_from_env()
{
  const char* s = getenv("FFB_DEVICE");
  return s ? atoi(s) : 0;
}

// ray_caster::task_create / task_free (ray_caster/system.cpp:44-62): every
// array malloc'd so that the reference's task_free releases it.
ray_caster::task_t* task_alloc(int n)
{
  ray_caster::task_t* t = (ray_caster::task_t*)malloc(sizeof(ray_caster::task_t));
  t->n_tasks = n;
  t->ray = (math::ray_t*)malloc((size_t)n * sizeof(math::ray_t));
  t->hit_face = (ray_caster::face_t**)malloc((size_t)n * sizeof(ray_caster::face_t*));
  t->hit_point = (math::vec3*)malloc((size_t)n * sizeof(math::vec3));
  return t;
}

void task_release(ray_caster::task_t* t)
{
  if (!t)
    return;
  free(t->ray);
  free(t->hit_face);
  free(t->hit_point);
  free(t);
}

}  // namespace

// ===========================================================================
// Ray caster
// ===========================================================================
namespace b200_ray_caster {

struct caster_t : ray_caster::system_t {
  ffb_ctx* ctx;
  ray_caster::scene_t* scene;
  ffb_grid_params grid;
  int prepared;
  std::vector<int32_t>* idx;  // host staging
  std::vector<float>* pts;
};

static int init(caster_t* s)
{
  s->ctx = nullptr;
  s->scene = nullptr;
  s->grid = ffb_grid_params{0, 0, 0, 32.f, 1};
  s->prepared = 0;
  s->idx = new std::vector<int32_t>();
  s->pts = new std::vector<float>();
  return ffb_ctx_create(device_from_env(), &s->ctx);
}

static int shutdown(caster_t* s)
{
  ffb_ctx_destroy(s->ctx);
  s->ctx = nullptr;
  delete s->idx;
  delete s->pts;
  s->idx = nullptr;
  s->pts = nullptr;
  return RAY_CASTER_OK;
}

static int set_scene(caster_t* s, ray_caster::scene_t* scene)
{
  s->scene = scene;
  s->prepared = 0;
  return RAY_CASTER_OK;
}

static int prepare(caster_t* s)
{
  if (s->scene == 0 || s->scene->n_faces == 0)
    return -RAY_CASTER_ERROR;
  if (!s->ctx)
    return FFB_ERR_NO_DEVICE;
  int r = ffb_scene_set(s->ctx, &s->scene->faces[0].points[0].x, s->scene->n_faces);
  if (r < 0)
    return r;
  if ((r = ffb_grid_build(s->ctx, &s->grid)) < 0)
    return r;
  s->prepared = 1;
  return RAY_CASTER_OK;
}

static int cast(caster_t* s, ray_caster::task_t* task)
{
  if (!s->prepared)
    return -RAY_CASTER_ERROR;
  const int n = task->n_tasks;
  if (n <= 0)
    return RAY_CASTER_OK;
  s->idx->resize((size_t)n);
  s->pts->resize(3 * (size_t)n);
  int r = ffb_cast(s->ctx, &task->ray[0].origin.x, n, s->idx->data(), s->pts->data());
  if (r < 0)
    return r;
  const int32_t* idx = s->idx->data();
  const float* p = s->pts->data();
  for (int i = 0; i < n; ++i) {
    if (idx[i] >= 0) {
      task->hit_face[i] = &s->scene->faces[idx[i]];
      task->hit_point[i].x = p[3 * i];
      task->hit_point[i].y = p[3 * i + 1];
      task->hit_point[i].z = p[3 * i + 2];
    } else {
      task->hit_face[i] = 0;
    }
  }
  return RAY_CASTER_OK;
}

static const ray_caster::system_methods_t methods = {
    (int (*)(ray_caster::system_t*))&init,
    (int (*)(ray_caster::system_t*))&shutdown,
    (int (*)(ray_caster::system_t*, ray_caster::scene_t*))&set_scene,
    (int (*)(ray_caster::system_t*))&prepare,
    (int (*)(ray_caster::system_t*, ray_caster::task_t*))&cast,
};

ray_caster::system_t* system_create()
{
  caster_t* s = (caster_t*)malloc(sizeof(caster_t));
  s->methods = &methods;
  return s;
}

ray_caster::system_t* create()
{
  ray_caster::system_t* s = system_create();
  s->methods->init(s);
  return s;
}

void destroy(ray_caster::system_t* s)
{
  if (!s)
    return;
  s->methods->shutdown(s);
  free(s);
}

int set_grid(ray_caster::system_t* system, int nx, int ny, int nz, float cells_per_face)
{
  if (!system || system->methods != &methods)
    return FFB_ERR_ARG;
  caster_t* s = (caster_t*)system;
  s->grid.nx = nx;
  s->grid.ny = ny;
  s->grid.nz = nz;
  s->grid.cells_per_face = cells_per_face;
  s->prepared = 0;
  return FFB_OK;
}

}  // namespace b200_ray_caster

// ===========================================================================
// Emission
// ===========================================================================
namespace b200_emission {

struct emitter_t : emission::system_t {
  ray_caster::system_t* caster;
  ray_caster::scene_t* scene;
  ffb_ctx* ctx;
  uint64_t seed;
  uint32_t epoch;  // calls so far: every calculate draws fresh rays
  int flags;
};

static int init(emitter_t* s, ray_caster::system_t* caster)
{
  s->caster = caster;
  s->scene = nullptr;
  s->ctx = nullptr;
  s->seed = 1;
  s->epoch = 0;
  s->flags = 0;
  return ffb_ctx_create(device_from_env(), &s->ctx);
}

static int shutdown(emitter_t* s)
{
  ffb_ctx_destroy(s->ctx);
  s->ctx = nullptr;
  s->scene = nullptr;
  return EMISSION_OK;
}

// emission/malley_cpu.cpp:77-92: also sets and prepares the caster.
static int set_scene(emitter_t* s, ray_caster::scene_t* scene)
{
  if (scene == 0 || scene->n_faces == 0)
    return -EMISSION_ERROR;
  s->scene = scene;
  int r = 0;
  if (s->caster) {
    if ((r = s->caster->methods->set_scene(s->caster, scene)) < 0)
      return r;
    if ((r = s->caster->methods->prepare(s->caster)) < 0)
      return r;
  }
  if (!s->ctx)
    return FFB_ERR_NO_DEVICE;
  return ffb_scene_set(s->ctx, &scene->faces[0].points[0].x, scene->n_faces);
}

// emission/malley_cpu.cpp:142-211: the task's weights decide the rays per
// face side; the batch is packed face by face, front then rear.
static int calculate(emitter_t* s, emission::task_t* task)
{
  if (!s->scene || !s->ctx)
    return -EMISSION_ERROR;
  malley_emission::task_t* t = (malley_emission::task_t*)task;
  if (task->rays) {
    task_release(task->rays);
    task->rays = 0;
  }
  const int n = s->scene->n_faces;
  std::vector<int32_t> front((size_t)n), rear((size_t)n);
  long long total = 0;
  for (int f = 0; f < n; ++f) {
    front[f] = emitted(t->n_rays, t->weights[2 * f], t->total_weight);
    rear[f] = emitted(t->n_rays, t->weights[2 * f + 1], t->total_weight);
    total += (long long)front[f] + rear[f];
  }
  if (total == 0)
    return EMISSION_OK;
  if (total > 0x7FFFFFFF)
    return FFB_ERR_TOO_LARGE;
  ray_caster::task_t* rays = task_alloc((int)total);
  int r = ffb_emit(s->ctx, front.data(), rear.data(), s->seed, s->epoch++, s->flags, &rays->ray[0].origin.x);
  if (r < 0) {
    task_release(rays);
    return r;
  }
  task->rays = rays;
  if (s->caster && (r = s->caster->methods->cast(s->caster, rays)) < 0)
    return r;
  return EMISSION_OK;
}

const emission::system_methods_t methods = {
    (int (*)(emission::system_t*, ray_caster::system_t*))&init,
    (int (*)(emission::system_t*))&shutdown,
    (int (*)(emission::system_t*, ray_caster::scene_t*))&set_scene,
    (int (*)(emission::system_t*, emission::task_t*))&calculate,
};

emission::system_t* system_create()
{
  emitter_t* s = (emitter_t*)malloc(sizeof(emitter_t));
  s->methods = &methods;
  return s;
}

emission::system_t* create(ray_caster::system_t* caster)
{
  emission::system_t* s = system_create();
  s->methods->init(s, caster);
  return s;
}

void destroy(emission::system_t* s)
{
  if (!s)
    return;
  s->methods->shutdown(s);
  free(s);
}

int set_seed(emission::system_t* system, uint64_t seed)
{
  if (!system || system->methods != &methods)
    return FFB_ERR_ARG;
  emitter_t* s = (emitter_t*)system;
  s->seed = seed;
  s->epoch = 0;
  return FFB_OK;
}

int set_flags(emission::system_t* system, int flags)
{
  if (!system || system->methods != &methods)
    return FFB_ERR_ARG;
  ((emitter_t*)system)->flags = flags;
  return FFB_OK;
}

// seed/epoch/flags of a B200 emitter for the fused form-factor path.
bool draw_key(emission::system_t* system, uint64_t* seed, uint32_t* epoch, int* flags)
{
  if (!system || system->methods != &methods)
    return false;
  emitter_t* s = (emitter_t*)system;
  *seed = s->seed;
  *epoch = s->epoch++;
  *flags = s->flags;
  return true;
}

}  // namespace b200_emission

// ===========================================================================
// Form factors
// ===========================================================================
namespace b200_form_factors {

struct ff_t : form_factors::system_t {
  emission::system_t* emitter;
  form_factors::scene_t* scene;
  ray_caster::scene_t rc_scene;
  float total_area;
  float* face_weights;
  int* face_to_mesh;
  int mesh_layout_ok;  // meshes cover every face once, in face order
  ffb_ctx* ctx;
  ffb_grid_params grid;
  uint64_t seed;
  uint32_t epoch;
  int flags;
};

// Emission, trace and counting all run fused on the GPU, so the only
// emitters accepted are the B200 Malley emitter (whose seed, epoch and flags
// key the fused draws) and none at all.  Any other emitter is refused with
// -FORM_FACTORS_ERROR: there is no host counting path.
static int init(ff_t* s, emission::system_t* emitter)
{
  s->emitter = emitter;
  s->scene = 0;
  s->rc_scene = ray_caster::scene_t{0, 0};
  s->total_area = 0;
  s->face_weights = 0;
  s->face_to_mesh = 0;
  s->mesh_layout_ok = 0;
  s->ctx = nullptr;
  s->grid = ffb_grid_params{0, 0, 0, 32.f, 1};
  s->seed = 1;
  s->epoch = 0;
  s->flags = 0;
  if (emitter != 0 && emitter->methods != &b200_emission::methods)
    return -FORM_FACTORS_ERROR;
  const int rc = ffb_ctx_create(device_from_env(), &s->ctx);
  if (rc == FFB_OK)
    ffb_ctx_set_stats(s->ctx, 0);  // the calculator reports no counters
  return rc;
}

static int shutdown(ff_t* s)
{
  s->scene = 0;
  free(s->face_weights);
  s->face_weights = 0;
  free(s->face_to_mesh);
  s->face_to_mesh = 0;
  s->total_area = 0;
  ffb_ctx_destroy(s->ctx);
  s->ctx = nullptr;
  return FORM_FACTORS_OK;
}

// cpuFactorsCalculator/cpu_system.cpp:82-92: the scene is uploaded and the
// grid built here, where the reference's emitter prepares its caster.
static int set_scene(ff_t* s, form_factors::scene_t* scene)
{
  s->scene = scene;
  s->rc_scene = ray_caster::scene_t{scene->n_faces, scene->faces};
  if (scene->n_faces == 0)
    return -EMISSION_ERROR;
  if (!s->ctx)
    return FFB_ERR_NO_DEVICE;
  int r = ffb_scene_set(s->ctx, &scene->faces[0].points[0].x, scene->n_faces);
  if (r < 0)
    return r;
  return ffb_grid_build(s->ctx, &s->grid);
}

// cpuFactorsCalculator/cpu_system.cpp:95-136, total_area accumulating as there.
static int prepare(ff_t* s)
{
  if (s->scene == 0 || s->scene->n_faces == 0 || s->scene->n_meshes == 0)
    return -FORM_FACTORS_EMPTY_SCENE;
  const int n_faces = s->scene->n_faces;
  free(s->face_weights);
  s->face_weights = (float*)malloc(2 * (size_t)n_faces * sizeof(float));
  free(s->face_to_mesh);
  s->face_to_mesh = (int*)malloc((size_t)n_faces * sizeof(int));
  int next = 0;
  s->mesh_layout_ok = 1;
  for (int m = 0; m != s->scene->n_meshes; ++m) {
    const form_factors::mesh_t& mesh = s->scene->meshes[m];
    if (mesh.first_idx != next || mesh.n_faces < 0)
      s->mesh_layout_ok = 0;
    for (int f = 0; f != mesh.n_faces; ++f) {
      const int idx = mesh.first_idx + f;
      if (idx >= 0 && idx < n_faces)
        s->face_to_mesh[idx] = m;
    }
    next = mesh.first_idx + mesh.n_faces;
  }
  if (next != n_faces)
    s->mesh_layout_ok = 0;
  for (int i = 0; i != n_faces; ++i) {
    const float face_area = triangle_area(s->scene->faces[i]);
    s->total_area += 2.f * face_area;
    s->face_weights[2 * i] = face_area;
    s->face_weights[2 * i + 1] = face_area;
  }
  if (s->total_area < FLT_EPSILON)
    return -FORM_FACTORS_SCENE_TOO_SMALL;
  return FORM_FACTORS_OK;
}

static int calculate_fused(ff_t* s, form_factors::task_t* task)
{
  if (!s->mesh_layout_ok)
    return -FORM_FACTORS_ERROR;
  const int n_faces = s->scene->n_faces, n_meshes = s->scene->n_meshes;
  std::vector<int32_t> front((size_t)n_faces), rear((size_t)n_faces), outgoing((size_t)n_meshes, 0);
  for (int f = 0; f < n_faces; ++f) {
    front[f] = emitted(task->n_rays, s->face_weights[2 * f], s->total_area);
    rear[f] = emitted(task->n_rays, s->face_weights[2 * f + 1], s->total_area);
    outgoing[s->face_to_mesh[f]] += front[f] + rear[f];
  }
  uint64_t seed = s->seed;
  uint32_t epoch = 0;
  int flags = s->flags;
  if (!b200_emission::draw_key(s->emitter, &seed, &epoch, &flags))
    epoch = s->epoch++;
  return ffb_form_factors(s->ctx, front.data(), rear.data(), seed, epoch, flags, s->face_to_mesh, n_meshes,
                          outgoing.data(), task->form_factors);
}

static int calculate(ff_t* s, form_factors::task_t* task)
{
  if (!s->scene || !s->face_weights)
    return -FORM_FACTORS_EMPTY_SCENE;
  return calculate_fused(s, task);
}

static const form_factors::system_methods_t methods = {
    (int (*)(form_factors::system_t*, emission::system_t*))&init,
    (int (*)(form_factors::system_t*))&shutdown,
    (int (*)(form_factors::system_t*, form_factors::scene_t*))&set_scene,
    (int (*)(form_factors::system_t*))&prepare,
    (int (*)(form_factors::system_t*, form_factors::task_t*))&calculate,
};

form_factors::system_t* system_create()
{
  ff_t* s = (ff_t*)malloc(sizeof(ff_t));
  s->methods = &methods;
  return s;
}

form_factors::system_t* create(emission::system_t* emitter)
{
  form_factors::system_t* s = system_create();
  s->methods->init(s, emitter);
  return s;
}

void destroy(form_factors::system_t* s)
{
  if (!s)
    return;
  s->methods->shutdown(s);
  free(s);
}

static ff_t* as_ff(form_factors::system_t* system)
{
  return system && system->methods == &methods ? (ff_t*)system : nullptr;
}

int set_seed(form_factors::system_t* system, uint64_t seed)
{
  ff_t* s = as_ff(system);
  if (!s)
    return FFB_ERR_ARG;
  s->seed = seed;
  s->epoch = 0;
  return FFB_OK;
}

int set_flags(form_factors::system_t* system, int flags)
{
  ff_t* s = as_ff(system);
  if (!s)
    return FFB_ERR_ARG;
  s->flags = flags;
  return FFB_OK;
}

int set_grid(form_factors::system_t* system, int nx, int ny, int nz, float cells_per_face)
{
  ff_t* s = as_ff(system);
  if (!s)
    return FFB_ERR_ARG;
  s->grid.nx = nx;
  s->grid.ny = ny;
  s->grid.nz = nz;
  s->grid.cells_per_face = cells_per_face;
  return FFB_OK;
}

}  // namespace b200_form_factors

// ===========================================================================
// Parallel-rays emission
// ===========================================================================
namespace b200_parallel_rays_emission {

struct emitter_t : emission::system_t {
  ray_caster::system_t* caster;
  ray_caster::scene_t* scene;
  ffb_ctx* ctx;
  uint64_t seed;
  uint32_t epoch;  // calls so far: every calculate draws fresh rays
};

static int init(emitter_t* s, ray_caster::system_t* caster)
{
  s->caster = caster;
  s->scene = nullptr;
  s->ctx = nullptr;
  s->seed = 1;
  s->epoch = 0;
  return ffb_ctx_create(device_from_env(), &s->ctx);
}

static int shutdown(emitter_t* s)
{
  ffb_ctx_destroy(s->ctx);
  s->ctx = nullptr;
  s->scene = nullptr;
  return EMISSION_OK;
}

// emission/parallel_rays_cpu.cpp:64-80
static int set_scene(emitter_t* s, ray_caster::scene_t* scene)
{
  if (scene == 0 || scene->n_faces == 0)
    return -EMISSION_ERROR;
  s->scene = scene;
  int r = 0;
  if (s->caster) {
    if ((r = s->caster->methods->set_scene(s->caster, scene)) < 0)
      return r;
    if ((r = s->caster->methods->prepare(s->caster)) < 0)
      return r;
  }
  return EMISSION_OK;
}

// emission/parallel_rays_cpu.cpp:83-121
static int calculate(emitter_t* s, emission::task_t* task)
{
  if (!s->ctx)
    return -EMISSION_ERROR;
  parallel_rays_emission_cpu::task_t* t = (parallel_rays_emission_cpu::task_t*)task;
  if (task->rays) {
    task_release(task->rays);
    task->rays = 0;
  }
  if (t->n_rays <= 0)
    return EMISSION_OK;
  ffb_disc_source src;
  const math::vec3 d = t->direction, c = t->center;
  src.direction[0] = d.x;
  src.direction[1] = d.y;
  src.direction[2] = d.z;
  src.center[0] = c.x;
  src.center[1] = c.y;
  src.center[2] = c.z;
  src.distance = t->distance;
  src.radius = t->radius;
  ray_caster::task_t* rays = task_alloc(t->n_rays);
  int r = ffb_emit_parallel(s->ctx, &src, t->n_rays, s->seed, s->epoch++, &rays->ray[0].origin.x);
  if (r < 0) {
    task_release(rays);
    return r;
  }
  task->rays = rays;
  if (s->caster && (r = s->caster->methods->cast(s->caster, rays)) < 0)
    return r;
  return EMISSION_OK;
}

const emission::system_methods_t methods = {
    (int (*)(emission::system_t*, ray_caster::system_t*))&init,
    (int (*)(emission::system_t*))&shutdown,
    (int (*)(emission::system_t*, ray_caster::scene_t*))&set_scene,
    (int (*)(emission::system_t*, emission::task_t*))&calculate,
};

emission::system_t* system_create()
{
  emitter_t* s = (emitter_t*)malloc(sizeof(emitter_t));
  s->methods = &methods;
  return s;
}

emission::system_t* create(ray_caster::system_t* caster)
{
  emission::system_t* s = system_create();
  s->methods->init(s, caster);
  return s;
}

void destroy(emission::system_t* s)
{
  if (!s)
    return;
  s->methods->shutdown(s);
  free(s);
}

int set_seed(emission::system_t* system, uint64_t seed)
{
  if (!system || system->methods != &methods)
    return FFB_ERR_ARG;
  emitter_t* s = (emitter_t*)system;
  s->seed = seed;
  s->epoch = 0;
  return FFB_OK;
}

// seed and call number of a B200 parallel-rays emitter for the fused step
bool draw_key(emission::system_t* system, uint64_t* seed, uint32_t* epoch)
{
  if (!system || system->methods != &methods)
    return false;
  emitter_t* s = (emitter_t*)system;
  *seed = s->seed;
  *epoch = s->epoch++;
  return true;
}

}  // namespace b200_parallel_rays_emission

// ===========================================================================
// Ray-traced thermal equations (shared state)
// ===========================================================================
namespace {

struct thermal_t : thermal_equation::system_t {
  emission::system_t* emitter;
  int n_rays;
  subject::scene_t* scene;
  ray_caster::scene_t rc_scene;
  ffb_ctx* ctx;
  ffb_grid_params grid;
  uint64_t seed;
  uint32_t epoch;
  // distant source
  void* source_param;
  parallel_rays_cpu::source_t (*source)(void* param);
};

void mesh_tables(const subject::scene_t* scene, std::vector<ffb_mesh>& meshes, std::vector<ffb_optics>& optics)
{
  meshes.resize((size_t)scene->n_meshes);
  for (int m = 0; m < scene->n_meshes; ++m)
    meshes[m] = ffb_mesh{scene->meshes[m].first_idx, scene->meshes[m].n_faces, scene->meshes[m].material_idx};
  optics.resize((size_t)scene->n_materials);
  for (int k = 0; k < scene->n_materials; ++k) {
    const subject::material_t& mt = scene->materials[k];
    optics[k] = ffb_optics{mt.front.emissivity, mt.rear.emissivity, mt.front.absorbance, mt.rear.absorbance};
  }
}

// The step runs fused on the GPU (emission, trace and the absorbed-power
// scatter in one kernel), so the equation accepts only its own B200 emitter
// type (`accepted`) or none; any other emitter is refused with
// -THERMAL_EQUATION_ERROR: there is no host absorption path.
int thermal_init(thermal_t* s, emission::system_t* emitter, int n_rays, bool accepted)
{
  s->emitter = emitter;
  s->n_rays = n_rays;
  s->scene = 0;
  s->rc_scene = ray_caster::scene_t{0, 0};
  s->ctx = nullptr;
  s->grid = ffb_grid_params{0, 0, 0, 32.f, 1};
  s->seed = 1;
  s->epoch = 0;
  s->source_param = 0;
  s->source = 0;
  if (!accepted)
    return -THERMAL_EQUATION_ERROR;
  const int rc = ffb_ctx_create(device_from_env(), &s->ctx);
  if (rc == FFB_OK)
    ffb_ctx_set_stats(s->ctx, 0);
  return rc;
}

int thermal_shutdown(thermal_t* s)
{
  s->scene = 0;
  ffb_ctx_destroy(s->ctx);
  s->ctx = nullptr;
  return THERMAL_EQUATION_OK;
}

// radiance_cpu.cpp:78-94 / parallel_rays_cpu.cpp:66-78: the scene and its
// grid stay resident on the device.
int thermal_set_scene(thermal_t* s, subject::scene_t* scene)
{
  s->scene = scene;
  s->rc_scene = ray_caster::scene_t{scene->n_faces, scene->faces};
  if (scene->n_faces == 0)
    return -EMISSION_ERROR;
  if (!s->ctx)
    return FFB_ERR_NO_DEVICE;
  int r = ffb_scene_set(s->ctx, &scene->faces[0].points[0].x, scene->n_faces);
  if (r < 0)
    return r;
  return ffb_grid_build(s->ctx, &s->grid);
}

thermal_t* as_thermal(thermal_equation::system_t* system, const thermal_equation::system_methods_t* m)
{
  return system && system->methods == m ? (thermal_t*)system : nullptr;
}

}  // namespace

// ===========================================================================
// Radiance equation
// ===========================================================================
namespace b200_radiance_equation {

static int init(thermal_t* s, radiance_equation::params_t* params)
{
  emission::system_t* e = params ? params->emitter : 0;
  return thermal_init(s, e, params ? params->n_rays : 0, e == 0 || e->methods == &b200_emission::methods);
}

static int shutdown(thermal_t* s) { return thermal_shutdown(s); }

static int set_scene(thermal_t* s, subject::scene_t* scene) { return thermal_set_scene(s, scene); }

static int calculate_fused(thermal_t* s, thermal_equation::task_t* task)
{
  std::vector<ffb_mesh> meshes;
  std::vector<ffb_optics> optics;
  mesh_tables(s->scene, meshes, optics);
  uint64_t seed = s->seed;
  uint32_t epoch = 0;
  int flags = 0;
  if (!b200_emission::draw_key(s->emitter, &seed, &epoch, &flags))
    epoch = s->epoch++;
  return ffb_radiance_step(s->ctx, &s->scene->faces[0].points[0].x, s->scene->n_faces, meshes.data(),
                           s->scene->n_meshes, optics.data(), s->scene->n_materials, task->temperatures, s->n_rays,
                           seed, epoch, flags, task->emission, task->absorption);
}

static int calculate(thermal_t* s, thermal_equation::task_t* task)
{
  if (!s->scene)
    return -THERMAL_EQUATION_ERROR;
  return calculate_fused(s, task);
}

static const thermal_equation::system_methods_t methods = {
    (int (*)(thermal_equation::system_t*, void*))&init,
    (int (*)(thermal_equation::system_t*))&shutdown,
    (int (*)(thermal_equation::system_t*, subject::scene_t*))&set_scene,
    (int (*)(thermal_equation::system_t*, thermal_equation::task_t*))&calculate,
};

thermal_equation::system_t* system_create()
{
  thermal_t* s = (thermal_t*)malloc(sizeof(thermal_t));
  s->methods = &methods;
  return s;
}

thermal_equation::system_t* create(radiance_equation::params_t* params)
{
  thermal_equation::system_t* s = system_create();
  s->methods->init(s, params);
  return s;
}

void destroy(thermal_equation::system_t* s)
{
  if (!s)
    return;
  s->methods->shutdown(s);
  free(s);
}

int set_seed(thermal_equation::system_t* system, uint64_t seed)
{
  thermal_t* s = as_thermal(system, &methods);
  if (!s)
    return FFB_ERR_ARG;
  s->seed = seed;
  s->epoch = 0;
  return FFB_OK;
}

int set_grid(thermal_equation::system_t* system, int nx, int ny, int nz, float cells_per_face)
{
  thermal_t* s = as_thermal(system, &methods);
  if (!s)
    return FFB_ERR_ARG;
  s->grid = ffb_grid_params{nx, ny, nz, cells_per_face, 1};
  return FFB_OK;
}

}  // namespace b200_radiance_equation

// ===========================================================================
// Distant source (parallel rays)
// ===========================================================================
namespace b200_distant_source {

static int init(thermal_t* s, parallel_rays_cpu::params_t* params)
{
  emission::system_t* e = params ? params->emitter : 0;
  const int rc = thermal_init(s, e, params ? params->n_rays : 0,
                              e == 0 || e->methods == &b200_parallel_rays_emission::methods);
  s->source_param = params ? params->source_param : 0;
  s->source = params ? params->source : 0;
  return rc;
}

static int shutdown(thermal_t* s) { return thermal_shutdown(s); }

static int set_scene(thermal_t* s, subject::scene_t* scene) { return thermal_set_scene(s, scene); }

static int calculate_fused(thermal_t* s, thermal_equation::task_t* task, const parallel_rays_cpu::source_t& src)
{
  std::vector<ffb_mesh> meshes;
  std::vector<ffb_optics> optics;
  mesh_tables(s->scene, meshes, optics);
  uint64_t seed = s->seed;
  uint32_t epoch = 0;
  if (!b200_parallel_rays_emission::draw_key(s->emitter, &seed, &epoch))
    epoch = s->epoch++;
  const float dir[3] = {src.direction.x, src.direction.y, src.direction.z};
  return ffb_distant_source_step(s->ctx, &s->scene->faces[0].points[0].x, s->scene->n_faces, meshes.data(),
                                 s->scene->n_meshes, optics.data(), s->scene->n_materials, s->n_rays, src.power, dir,
                                 seed, epoch, task->absorption);
}

static int calculate(thermal_t* s, thermal_equation::task_t* task)
{
  if (!s->scene)
    return -THERMAL_EQUATION_ERROR;
  if (s->source == 0)  // parallel_rays_cpu.cpp:94-95
    return THERMAL_EQUATION_OK;
  const parallel_rays_cpu::source_t src = s->source(s->source_param);
  return calculate_fused(s, task, src);
}

static const thermal_equation::system_methods_t methods = {
    (int (*)(thermal_equation::system_t*, void*))&init,
    (int (*)(thermal_equation::system_t*))&shutdown,
    (int (*)(thermal_equation::system_t*, subject::scene_t*))&set_scene,
    (int (*)(thermal_equation::system_t*, thermal_equation::task_t*))&calculate,
};

thermal_equation::system_t* system_create()
{
  thermal_t* s = (thermal_t*)malloc(sizeof(thermal_t));
  s->methods = &methods;
  return s;
}

thermal_equation::system_t* create(parallel_rays_cpu::params_t* params)
{
  thermal_equation::system_t* s = system_create();
  s->methods->init(s, params);
  return s;
}

void destroy(thermal_equation::system_t* s)
{
  if (!s)
    return;
  s->methods->shutdown(s);
  free(s);
}

int set_seed(thermal_equation::system_t* system, uint64_t seed)
{
  thermal_t* s = as_thermal(system, &methods);
  if (!s)
    return FFB_ERR_ARG;
  s->seed = seed;
  s->epoch = 0;
  return FFB_OK;
}

int set_grid(thermal_equation::system_t* system, int nx, int ny, int nz, float cells_per_face)
{
  thermal_t* s = as_thermal(system, &methods);
  if (!s)
    return FFB_ERR_ARG;
  s->grid = ffb_grid_params{nx, ny, nz, cells_per_face, 1};
  return FFB_OK;
}

}  // namespace b200_distant_source

// ===========================================================================
// OBJ import
// ===========================================================================
namespace b200_obj_import {

int scene(const char* filename, subject::scene_t** out)
{
  if (!filename || !out)
    return FFB_ERR_ARG;
  ffb_ctx* ctx = nullptr;
  int rc = ffb_ctx_create(device_from_env(), &ctx);
  if (rc < 0)
    return rc;
  ffb_obj_info info;
  rc = ffb_obj_load(ctx, filename, &info);
  if (rc == FFB_ERR_FILE || rc == FFB_ERR_FORMAT) {
    ffb_ctx_destroy(ctx);
    return info.status;
  }
  if (rc < 0) {
    ffb_ctx_destroy(ctx);
    return rc;
  }
  // subject::scene_create layout; arrays malloc'd for subject::scene_free
  subject::scene_t* s = (subject::scene_t*)malloc(sizeof(subject::scene_t));
  s->n_faces = info.n_faces;
  s->faces = (subject::face_t*)malloc(sizeof(subject::face_t) * (size_t)std::max(info.n_faces, 1));
  s->n_meshes = info.n_meshes;
  s->meshes = (subject::mesh_t*)malloc(sizeof(subject::mesh_t) * (size_t)info.n_meshes);
  s->n_materials = info.n_materials;
  s->materials = (subject::material_t*)malloc(sizeof(subject::material_t) * (size_t)info.n_materials);
  static_assert(sizeof(subject::mesh_t) == sizeof(ffb_mesh), "mesh layout");
  static_assert(sizeof(subject::material_t) == sizeof(ffb_material), "material layout");
  rc = ffb_obj_result(ctx, &s->faces[0].points[0].x, (ffb_mesh*)s->meshes, (ffb_material*)s->materials);
  ffb_ctx_destroy(ctx);
  if (rc < 0) {
    free(s->faces);
    free(s->meshes);
    free(s->materials);
    free(s);
    return rc;
  }
  *out = s;
  return OBJ_IMPORT_OK;
}

}  // namespace b200_obj_import

// ===========================================================================
// CSV export
// ===========================================================================
namespace b200_csv_export {

int export_csv(const char* filename, form_factors::scene_t* scene, form_factors::task_t* task)
{
  if (!filename || !scene || !task || scene->n_meshes < 0 || (scene->n_meshes && !task->form_factors))
    return FFB_ERR_ARG;
  ffb_ctx* ctx = nullptr;
  int rc = ffb_ctx_create(device_from_env(), &ctx);
  if (rc == FFB_OK)
    rc = ffb_csv_export(ctx, filename, task->form_factors, scene->n_meshes);
  ffb_ctx_destroy(ctx);
  return rc == FFB_ERR_FILE ? -CSV_EXPORT_FILE_ERROR : rc;
}

}  // namespace b200_csv_export
