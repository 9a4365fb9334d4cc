/*
 * ffb_systems.h -- the B200 path as new selectable types behind the
 * reference's own C++ interfaces:
 *
 *   ray_caster::system_t    ray_caster/system.h:85-116     RAY_CASTER_B200      (5)
 *   emission::system_t      emission/system.h:77-93        EMISSION_MALLEY_B200 (3)
 *   form_factors::system_t  form_factors/system.h:95-119   FORM_FACTORS_B200    (2)
 *
 * Each system_create() mallocs the system and sets its method table, exactly
 * like the reference's implementation creators (e.g. ray_caster/naive_cpu.cpp
 * system_create): the reference's factory then calls init, and system_free
 * (shutdown + free) releases it.  create() does both steps for callers
 * without the reference's factory, destroy() is shutdown + free.  Built
 * inside the reference tree, define
 * FFB_USE_REFERENCE_HEADERS and put the reference root on the include path:
 * the reference's own headers then declare the interface types.  Otherwise
 * the layout-identical declarations below are used (same members, same order,
 * same method tables).
 */
#ifndef FFB_SYSTEMS_H
#define FFB_SYSTEMS_H

#include <stdint.h>

#ifdef FFB_USE_REFERENCE_HEADERS
#include "ray_caster/system.h"
#include "emission/system.h"
#include "emission/malley_emission.h"
#include "form_factors/system.h"
#include "import_export/csv_export.h"
#include "subject/system.h"
#include "thermal_equation/system.h"
#include "thermal_equation/radiance_cpu.h"
#include "thermal_equation/parallel_rays_cpu.h"
#include "emission/parallel_rays_cpu.h"
#include "import_export/obj_import.h"
#else

namespace math {
typedef float point_t;
struct vec3 {
  point_t x, y, z;
};
struct triangle_t {
  vec3 points[3];
};
typedef triangle_t face_t;
struct ray_t {
  vec3 origin;
  vec3 direction;  // the END point of the ray, not a direction
};
}  // namespace math

namespace ray_caster {
typedef math::triangle_t face_t;
typedef math::ray_t ray_t;
struct task_t {
  int n_tasks;
  math::ray_t* ray;
  face_t** hit_face;
  math::vec3* hit_point;
};
struct scene_t {
  int n_faces;
  face_t* faces;
};
struct system_t {
  const struct system_methods_t* methods;
};
#define RAY_CASTER_OK 0
#define RAY_CASTER_ERROR 1
#define RAY_CASTER_NOT_SUPPORTED 2
struct system_methods_t {
  int (*init)(system_t* system);
  int (*shutdown)(system_t* system);
  int (*set_scene)(system_t* system, scene_t* scene);
  int (*prepare)(system_t* system);
  int (*cast)(system_t* system, task_t* task);
};
}  // namespace ray_caster

namespace emission {
struct task_t {
  task_t(int n) : n_rays(n), rays(0) {}
  int n_rays;
  ray_caster::task_t* rays;
};
struct system_t {
  const struct system_methods_t* methods;
};
#define EMISSION_OK 0
#define EMISSION_ERROR 200
struct system_methods_t {
  int (*init)(system_t* system, ray_caster::system_t* ray_caster);
  int (*shutdown)(system_t* system);
  int (*set_scene)(system_t* system, ray_caster::scene_t* scene);
  int (*calculate)(system_t* system, task_t* task);
};
}  // namespace emission

namespace malley_emission {
struct task_t : emission::task_t {
  task_t(int n, float total, float* ws) : emission::task_t(n), total_weight(total), weights(ws) {}
  float total_weight;
  float* weights;  // two per face: front, rear
};
}  // namespace malley_emission

namespace form_factors {
typedef math::triangle_t face_t;
struct mesh_t {
  int first_idx;
  int n_faces;
  int padding0;
};
struct scene_t {
  int n_faces;
  face_t* faces;
  int n_meshes;
  mesh_t* meshes;
};
struct task_t {
  int n_rays;
  float* form_factors;
};
struct system_t {
  const struct system_methods_t* methods;
};
#define FORM_FACTORS_OK 0
#define FORM_FACTORS_ERROR 100
#define FORM_FACTORS_EMPTY_SCENE 101
#define FORM_FACTORS_SCENE_TOO_SMALL 102
struct system_methods_t {
  int (*init)(system_t* system, emission::system_t* emitter);
  int (*shutdown)(system_t* system);
  int (*set_scene)(system_t* system, scene_t* scene);
  int (*prepare)(system_t* system);
  int (*calculate)(system_t* system, task_t* task);
};
}  // namespace form_factors

/* import_export/csv_export.h:27-28 */
#define CSV_EXPORT_OK 0
#define CSV_EXPORT_FILE_ERROR 31

/* emission/parallel_rays_cpu.h:25-33 */
namespace parallel_rays_emission_cpu {
struct task_t : emission::task_t {
  task_t(int n) : emission::task_t(n) {}
  math::vec3 direction;  // the reference does not normalise it
  math::vec3 center;
  float distance;
  float radius;
};
}  // namespace parallel_rays_emission_cpu

/* subject/system.h:28-86 */
namespace subject {
typedef math::triangle_t face_t;
struct shell_properties_t {
  float density, heat_capacity, thermal_conductivity, thickness;
};
struct optical_properties_t {
  float specular_reflectance, diffuse_reflectance, absorbance, transmittance, emissivity;
};
struct material_t {
  shell_properties_t shell;
  optical_properties_t front;
  optical_properties_t rear;
  char name[128];
};
struct mesh_t {
  int first_idx;
  int n_faces;
  int material_idx;
};
struct scene_t {
  int n_faces;
  face_t* faces;
  int n_meshes;
  mesh_t* meshes;
  int n_materials;
  material_t* materials;
};
}  // namespace subject

/* import_export/obj_import.h:31-36 */
#define OBJ_IMPORT_OK 0
#define OBJ_IMPORT_FILE_ERROR 21
#define OBJ_IMPORT_FORMAT_ERROR 22
#define OBJ_IMPORT_MATERIAL_NOT_DEFINED 23
#define OBJ_IMPORT_MATERIAL_NOT_ENOUGH_PARAMETERS 24
#define OBJ_IMPORT_MATERIAL_INVALID_PARAMETER_VALUE 25

/* thermal_equation/system.h:26-78 */
namespace thermal_equation {
struct task_t {
  const float* temperatures;
  float* emission;
  float* absorption;
};
struct system_t {
  const struct system_methods_t* methods;
};
#define THERMAL_EQUATION_OK 0
#define THERMAL_EQUATION_ERROR 400
struct system_methods_t {
  int (*init)(system_t* system, void* params);
  int (*shutdown)(system_t* system);
  int (*set_scene)(system_t* system, subject::scene_t* scene);
  int (*calculate)(system_t* system, task_t* task);
};
}  // namespace thermal_equation

/* thermal_equation/radiance_cpu.h:29-33 */
namespace radiance_equation {
struct params_t {
  emission::system_t* emitter;
  int n_rays;
};
}  // namespace radiance_equation

/* thermal_equation/parallel_rays_cpu.h:27-40 */
namespace parallel_rays_cpu {
struct source_t {
  float power;  // W/m^2
  math::vec3 direction;
};
struct params_t {
  int n_rays;
  emission::system_t* emitter;
  void* source_param;
  source_t (*source)(void* param);
};
}  // namespace parallel_rays_cpu

#endif  // FFB_USE_REFERENCE_HEADERS

/* Type IDs beside the reference's (ray_caster/system.h:106-109,
 * emission/system.h:92-93, form_factors/system.h:119,
 * thermal_equation/system.h:71-75). */
#define RAY_CASTER_B200 5
#define EMISSION_MALLEY_B200 3
#define EMISSION_PARALLEL_RAYS_B200 4
#define FORM_FACTORS_B200 2
#define THERMAL_EQUATION_RADIANCE_B200 6
#define THERMAL_EQUATION_DISTANT_SOURCE_B200 7

namespace b200_ray_caster {
/* Grid nearest-hit caster on the GPU.  set_scene keeps the pointer (the
 * reference's casters do not own scenes); prepare uploads the faces and
 * builds the grid (-RAY_CASTER_ERROR without a scene or with no faces, as
 * ray_caster/zgrid_cpu.cpp:59-60); cast writes hit_face (a pointer into the
 * caller's faces, or 0) and, for hits only, hit_point. */
ray_caster::system_t* system_create();
ray_caster::system_t* create();
void destroy(ray_caster::system_t* system);
/* Grid resolution (0,0,0 = automatic from cells_per_face). */
int set_grid(ray_caster::system_t* system, int nx, int ny, int nz, float cells_per_face);
}  // namespace b200_ray_caster

namespace b200_emission {
/* Malley emission on the GPU with Philox draws keyed by (seed, call, face,
 * ray).  Works with any ray_caster::system_t: the rays are generated on the
 * device, copied into task->rays (malloc'd, freed by the caller with
 * ray_caster::task_free as in cpuFactorsCalculator/cpu_system.cpp:198) and
 * cast with the given caster.  set_scene also sets and prepares the caster
 * (emission/malley_cpu.cpp:77-92). */
emission::system_t* system_create();
emission::system_t* create(ray_caster::system_t* caster);
void destroy(emission::system_t* system);
/* Seed of the Philox stream (default 1); resets the per-call counter. */
int set_seed(emission::system_t* system, uint64_t seed);
/* FFB_EMIT_REF_NORMAL (1): rotate +z to the raw cross-product normal as the
 * reference does; 0 (default): the normalised normal. */
int set_flags(emission::system_t* system, int flags);
}  // namespace b200_emission

namespace b200_form_factors {
/* Form factors between meshes (cpuFactorsCalculator/cpu_system.cpp:149-201).
 * The whole calculation -- emission, grid trace, per-(mesh, mesh) counts and
 * the row normalisation -- runs fused on the GPU and no ray batch is ever
 * materialised.  The emitter must be a B200 Malley emitter (its seed and
 * flags key the draws) or NULL; init refuses any other emitter with
 * -FORM_FACTORS_ERROR, since there is no host counting path.  Weights, the
 * total area (accumulating over prepare calls, cpu_system.cpp:126) and the
 * per-face ray budget follow the reference.  The fused path needs meshes that
 * cover every face exactly once in face order (the layout the reference's
 * ray walk assumes, cpu_system.cpp:167-190); other layouts return
 * -FORM_FACTORS_ERROR. */
form_factors::system_t* system_create();
form_factors::system_t* create(emission::system_t* emitter);
void destroy(form_factors::system_t* system);
int set_seed(form_factors::system_t* system, uint64_t seed);
int set_flags(form_factors::system_t* system, int flags);
int set_grid(form_factors::system_t* system, int nx, int ny, int nz, float cells_per_face);
}  // namespace b200_form_factors

namespace b200_parallel_rays_emission {
/* Parallel rays from a disc (emission/parallel_rays_cpu.cpp): calculate reads
 * a parallel_rays_emission_cpu::task_t, emits its n_rays on the GPU (Philox
 * keyed by seed, call number and ray), copies them into task->rays (malloc'd,
 * released by ray_caster::task_free) and casts them with the given caster.
 * set_scene sets and prepares the caster as the reference does. */
emission::system_t* system_create();
emission::system_t* create(ray_caster::system_t* caster);
void destroy(emission::system_t* system);
int set_seed(emission::system_t* system, uint64_t seed);
}  // namespace b200_parallel_rays_emission

namespace b200_radiance_equation {
/* The radiance equation (thermal_equation/radiance_cpu.cpp) for
 * radiance_equation::params_t.  The step runs fused on the GPU
 * (ffb_radiance_step: the scene and grid stay resident from set_scene; needs
 * meshes covering every face once).  The emitter must be a B200 Malley
 * emitter or NULL; init refuses any other with -THERMAL_EQUATION_ERROR. */
thermal_equation::system_t* system_create();
thermal_equation::system_t* create(radiance_equation::params_t* params);
void destroy(thermal_equation::system_t* system);
int set_seed(thermal_equation::system_t* system, uint64_t seed);
int set_grid(thermal_equation::system_t* system, int nx, int ny, int nz, float cells_per_face);
}  // namespace b200_radiance_equation

namespace b200_distant_source {
/* The distant source of parallel rays (thermal_equation/parallel_rays_cpu.cpp)
 * for parallel_rays_cpu::params_t.  The step runs fused on the GPU
 * (ffb_distant_source_step).  The emitter must be a B200 parallel-rays emitter
 * or NULL; init refuses any other with -THERMAL_EQUATION_ERROR. */
thermal_equation::system_t* system_create();
thermal_equation::system_t* create(parallel_rays_cpu::params_t* params);
void destroy(thermal_equation::system_t* system);
int set_seed(thermal_equation::system_t* system, uint64_t seed);
int set_grid(thermal_equation::system_t* system, int nx, int ny, int nz, float cells_per_face);
}  // namespace b200_distant_source

namespace b200_obj_import {
/* obj_import::scene (import_export/obj_import.cpp:167-340) with the geometry
 * parsed on the GPU (ffb_obj_load): the same faces, meshes and materials, and
 * the same return codes (OBJ_IMPORT_OK or -OBJ_IMPORT_*).  On success *scene is
 * malloc'd as subject::scene_create does, for subject::scene_free.  Each call
 * uses its own context on device FFB_DEVICE (default 0). */
int scene(const char* filename, subject::scene_t** scene);
}  // namespace b200_obj_import

namespace b200_csv_export {
/* csv_export::export_csv (import_export/csv_export.cpp:26-46) with the text
 * formatted on the GPU: the same file, byte for byte, for the n_meshes x
 * n_meshes matrix task->form_factors (host memory).  Returns CSV_EXPORT_OK,
 * -CSV_EXPORT_FILE_ERROR when the file cannot be opened or written (as the
 * reference), or a negative FFB_ERR_* code of include/ffb.h for a device
 * failure.  Each call uses its own context on device FFB_DEVICE (default 0). */
int export_csv(const char* filename, form_factors::scene_t* scene, form_factors::task_t* task);
}  // namespace b200_csv_export

#endif /* FFB_SYSTEMS_H */
