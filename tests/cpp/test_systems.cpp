// test_systems.cpp -- the B200 system types driven through the reference's
// C-style interfaces, in the manner of the reference's typed gtest suites
// (test/ray_casting.cpp, test/form_factors.cpp): the same checks run for
// every engine type.
//
// Built two ways:
//  * standalone (include/ffb_systems.h declarations): B200 types only;
//  * with -DFFB_WITH_REFERENCE and the reference's headers/objects: the
//    reference's naive_cpu / zgrid_cpu casters, malley_cpu emitter and
//    cpu_form_factors calculator run beside the B200 types and mixed with
//    them (reference calculator over the B200 emitter and caster, B200
//    calculator over the reference emitter).
// Exit status 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <utility>
#include <vector>

#include "ffb_systems.h"

static int g_failures = 0;
static int g_checks = 0;
#define CHECK(cond)                                                              \
  do {                                                                           \
    ++g_checks;                                                                  \
    if (!(cond)) {                                                               \
      ++g_failures;                                                              \
      std::fprintf(stderr, "FAIL %s:%d: %s [%s]\n", __FILE__, __LINE__, #cond, g_case.c_str()); \
    }                                                                            \
  } while (0)

static std::string g_case;

using math::vec3;

static vec3 V(float x, float y, float z) { return vec3{x, y, z}; }
static vec3 add(vec3 a, vec3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static vec3 sub(vec3 a, vec3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static math::triangle_t T(vec3 a, vec3 b, vec3 c) { return math::triangle_t{{a, b, c}}; }
static vec3 center(const math::triangle_t& t)
{
  return V((t.points[0].x + t.points[1].x + t.points[2].x) / 3.f, (t.points[0].y + t.points[1].y + t.points[2].y) / 3.f,
           (t.points[0].z + t.points[1].z + t.points[2].z) / 3.f);
}
// math::ray_to_triangle: towards the centre, ending half way.
static math::ray_t ray_to(vec3 o, const math::triangle_t& t)
{
  vec3 c = center(t);
  vec3 h = sub(c, o);
  return math::ray_t{o, add(o, V(h.x / 2.f, h.y / 2.f, h.z / 2.f))};
}
// ray_caster::task_free for a task whose arrays were malloc'd by an emitter
static void task_free_all(ray_caster::task_t* t)
{
  if (!t)
    return;
  free(t->ray);
  free(t->hit_face);
  free(t->hit_point);
  free(t);
}

static bool near_enough(vec3 a, vec3 b)
{
  vec3 d = sub(a, b);
  return d.x * d.x + d.y * d.y + d.z * d.z < 1e-8;
}

// ---------------------------------------------------------------------------
// engines
// ---------------------------------------------------------------------------
struct Caster {
  const char* name;
  std::function<ray_caster::system_t*()> make;
  std::function<void(ray_caster::system_t*)> free_;
};

static std::vector<Caster> casters()
{
  std::vector<Caster> v;
  v.push_back({"B200", [] { return b200_ray_caster::create(); }, [](ray_caster::system_t* s) { b200_ray_caster::destroy(s); }});
#ifdef FFB_WITH_REFERENCE
  v.push_back({"NAIVE_CPU", [] { return ray_caster::system_create(RAY_CASTER_NAIVE_CPU); },
               [](ray_caster::system_t* s) { ray_caster::system_free(s); }});
  v.push_back({"ZGRID_CPU", [] { return ray_caster::system_create(RAY_CASTER_ZGRID_CPU); },
               [](ray_caster::system_t* s) { ray_caster::system_free(s); }});
#endif
  return v;
}

// ---------------------------------------------------------------------------
// ray caster checks (test/ray_casting.cpp:113-322)
// ---------------------------------------------------------------------------
static void ray_caster_suite(const Caster& E)
{
  auto floor1 = T(V(0, 0, 0), V(1, 0, 0), V(0, 1, 0));
  auto floor2 = T(V(1, 0, 0), V(0, 1, 0), V(1, 1, 0));
  auto stack = T(V(0, 0, -1), V(1, 0, -1), V(0, 1, -1));
  {
    g_case = std::string(E.name) + " empty scene";
    ray_caster::system_t* s = E.make();
    ray_caster::scene_t empty = {0, 0};
    CHECK(s->methods->set_scene(s, &empty) == RAY_CASTER_OK);
    CHECK(s->methods->prepare(s) == -RAY_CASTER_ERROR);
    E.free_(s);
  }
  {
    g_case = std::string(E.name) + " prepare without scene";
    ray_caster::system_t* s = E.make();
    CHECK(s->methods->prepare(s) == -RAY_CASTER_ERROR);
    E.free_(s);
  }
  {
    g_case = std::string(E.name) + " floor";
    ray_caster::system_t* s = E.make();
    math::triangle_t faces[2] = {floor1, floor2};
    ray_caster::scene_t scene = {2, faces};
    CHECK(s->methods->set_scene(s, &scene) == RAY_CASTER_OK);
    CHECK(s->methods->prepare(s) == RAY_CASTER_OK);
    math::ray_t rays[2] = {ray_to(add(center(faces[0]), V(0, 0, 1)), faces[0]),
                           ray_to(add(center(faces[1]), V(0, 0, -1)), faces[1])};
    ray_caster::face_t* hit[2] = {0, 0};
    vec3 pts[2];
    ray_caster::task_t task = {2, rays, hit, pts};
    CHECK(s->methods->cast(s, &task) == RAY_CASTER_OK);
    CHECK(hit[0] == &faces[0] && hit[1] == &faces[1]);
    CHECK(near_enough(pts[0], center(faces[0])) && near_enough(pts[1], center(faces[1])));
    E.free_(s);
  }
  {
    g_case = std::string(E.name) + " stack";
    ray_caster::system_t* s = E.make();
    math::triangle_t faces[2] = {floor1, stack};
    ray_caster::scene_t scene = {2, faces};
    s->methods->set_scene(s, &scene);
    CHECK(s->methods->prepare(s) == RAY_CASTER_OK);
    vec3 c0 = center(faces[0]), c1 = center(faces[1]);
    math::ray_t rays[4] = {
        math::ray_t{add(c0, V(0, 0, .5f)), sub(c0, V(0, 0, .5f))},  // HandleRayIntersectingTriangle
        ray_to(add(c0, V(0, 0, 1)), faces[0]),                     // FindNearestTriangle
        ray_to(add(c1, V(0, 0, .9f)), faces[1]),                   // SkipTriangleNearButInOppositeDirection
        ray_to(add(c1, V(2, 2, 2)), faces[1])};                    // IntersectTriganglesNotPlanes
    ray_caster::face_t* hit[4] = {0, 0, 0, 0};
    vec3 pts[4];
    ray_caster::task_t task = {4, rays, hit, pts};
    CHECK(s->methods->cast(s, &task) == RAY_CASTER_OK);
    CHECK(hit[0] == &faces[0] && hit[1] == &faces[0] && hit[2] == &faces[1] && hit[3] == &faces[1]);
    CHECK(near_enough(pts[0], c0) && near_enough(pts[1], c0) && near_enough(pts[2], c1) && near_enough(pts[3], c1));
    E.free_(s);
  }
  {
    g_case = std::string(E.name) + " large scene";
    ray_caster::system_t* s = E.make();
    std::vector<math::triangle_t> faces;
    for (int i = -500; i != 500; ++i) {
      vec3 sh = V(0, 0, .1f * (float)i);
      faces.push_back(T(add(floor1.points[0], sh), add(floor1.points[1], sh), add(floor1.points[2], sh)));
    }
    ray_caster::scene_t scene = {(int)faces.size(), faces.data()};
    s->methods->set_scene(s, &scene);
    CHECK(s->methods->prepare(s) == RAY_CASTER_OK);
    vec3 c = center(faces[0]);
    math::ray_t ray = ray_to(add(c, V(2, 2, -2)), faces[0]);
    ray_caster::face_t* hit = 0;
    vec3 pt;
    ray_caster::task_t task = {1, &ray, &hit, &pt};
    CHECK(s->methods->cast(s, &task) == RAY_CASTER_OK);
    CHECK(hit == &faces[0] && near_enough(pt, c));
    E.free_(s);
  }
}

// ---------------------------------------------------------------------------
// form factors (test/form_factors.cpp:192-298, two-sided semantics: F is half
// the one-sided analytic value)
// ---------------------------------------------------------------------------
static double vf_parallel(double a, double b, double c)
{
  double x = a / c, y = b / c, xq = x * x, yq = y * y;
  return 2.0 / M_PI / x / y *
         (std::log(std::sqrt((1 + xq) * (1 + yq) / (1 + xq + yq))) + x * std::sqrt(1 + yq) * std::atan(x / std::sqrt(1 + yq)) +
          y * std::sqrt(1 + xq) * std::atan(y / std::sqrt(1 + xq)) - x * std::atan(x) - y * std::atan(y));
}

static double vf_perpendicular(double H, double W, double L)
{
  double h = H / L, w = W / L;
  double a = (1 + h * h) * (1 + w * w) / (1 + h * h + w * w);
  double b = w * w * (1 + h * h + w * w) / (1 + w * w) / (h * h + w * w);
  double c = h * h * (1 + h * h + w * w) / (1 + h * h) / (h * h + w * w);
  return 1.0 / M_PI / w *
         (h * std::atan(1 / h) + w * std::atan(1 / w) - std::sqrt(h * h + w * w) * std::atan(1 / std::sqrt(h * h + w * w)) +
          0.25 * std::log(a * std::pow(b, w * w) * std::pow(c, h * h)));
}

static std::vector<math::triangle_t> square(vec3 o)
{
  return {T(add(V(0, 0, 0), o), add(V(1, 0, 0), o), add(V(0, 1, 0), o)),
          T(add(V(1, 0, 0), o), add(V(1, 1, 0), o), add(V(0, 1, 0), o))};
}

struct Calculator {
  const char* name;
  std::function<void(form_factors::system_t**, emission::system_t**, ray_caster::system_t**)> make;
  std::function<void(form_factors::system_t*, emission::system_t*, ray_caster::system_t*)> free_;
};

static std::vector<Calculator> calculators()
{
  std::vector<Calculator> v;
  // fused B200 path (B200 emitter, whose caster is the B200 caster)
  v.push_back({"B200 fused",
               [](form_factors::system_t** f, emission::system_t** e, ray_caster::system_t** r) {
                 *r = b200_ray_caster::create();
                 *e = b200_emission::create(*r);
                 *f = b200_form_factors::create(*e);
               },
               [](form_factors::system_t* f, emission::system_t* e, ray_caster::system_t* r) {
                 b200_form_factors::destroy(f);
                 b200_emission::destroy(e);
                 b200_ray_caster::destroy(r);
               }});
#ifdef FFB_WITH_REFERENCE
  // reference calculator over the B200 emitter and caster
  v.push_back({"CPU calculator + B200 emission/caster",
               [](form_factors::system_t** f, emission::system_t** e, ray_caster::system_t** r) {
                 *r = b200_ray_caster::create();
                 *e = b200_emission::create(*r);
                 *f = form_factors::system_create(FORM_FACTORS_CPU, *e);
               },
               [](form_factors::system_t* f, emission::system_t* e, ray_caster::system_t* r) {
                 form_factors::system_free(f);
                 b200_emission::destroy(e);
                 b200_ray_caster::destroy(r);
               }});
  // reference calculator and emitter over the B200 caster
  v.push_back({"CPU calculator + malley_cpu + B200 caster",
               [](form_factors::system_t** f, emission::system_t** e, ray_caster::system_t** r) {
                 *r = b200_ray_caster::create();
                 *e = emission::system_create(EMISSION_MALLEY_CPU, *r);
                 *f = form_factors::system_create(FORM_FACTORS_CPU, *e);
               },
               [](form_factors::system_t* f, emission::system_t* e, ray_caster::system_t* r) {
                 form_factors::system_free(f);
                 emission::system_free(e);
                 b200_ray_caster::destroy(r);
               }});
  // the reference alone, as the control
  v.push_back({"CPU reference",
               [](form_factors::system_t** f, emission::system_t** e, ray_caster::system_t** r) {
                 *r = ray_caster::system_create(RAY_CASTER_NAIVE_CPU);
                 *e = emission::system_create(EMISSION_MALLEY_CPU, *r);
                 *f = form_factors::system_create(FORM_FACTORS_CPU, *e);
               },
               [](form_factors::system_t* f, emission::system_t* e, ray_caster::system_t* r) {
                 form_factors::system_free(f);
                 emission::system_free(e);
                 ray_caster::system_free(r);
               }});
#endif
  return v;
}

static void form_factor_suite(const Calculator& C)
{
  const float distances[] = {.5f, 1, 2, 3, 10};
  for (float d : distances) {
    g_case = std::string(C.name) + " parallel d=" + std::to_string(d);
    form_factors::system_t* f;
    emission::system_t* e;
    ray_caster::system_t* r;
    C.make(&f, &e, &r);
    std::vector<math::triangle_t> faces = square(V(0, 0, 0));
    std::vector<math::triangle_t> top = square(V(0, 0, d));
    faces.insert(faces.end(), top.begin(), top.end());
    form_factors::mesh_t meshes[2] = {{0, 2, 0}, {2, 2, 0}};
    form_factors::scene_t scene = {4, faces.data(), 2, meshes};
    CHECK(f->methods->set_scene(f, &scene) >= 0);
    CHECK(f->methods->prepare(f) == FORM_FACTORS_OK);
    float ff[4];
    form_factors::task_t task = {40000, ff};
    CHECK(f->methods->calculate(f, &task) == FORM_FACTORS_OK);
    const double want = vf_parallel(1, 1, d) / 2;
    CHECK(std::fabs(ff[1] - want) < 0.01 && std::fabs(ff[2] - want) < 0.01);
    // a plate sees itself only through FP32 rounding of grazing rays
    CHECK(ff[0] < 1e-3f && ff[3] < 1e-3f);
    C.free_(f, e, r);
  }
  {
    g_case = std::string(C.name) + " perpendicular";
    form_factors::system_t* f;
    emission::system_t* e;
    ray_caster::system_t* r;
    C.make(&f, &e, &r);
    std::vector<math::triangle_t> faces = square(V(0, 0, 0));
    faces.push_back(T(V(0, 0, 0), V(0, 1, 0), V(0, 0, 1)));
    faces.push_back(T(V(0, 1, 0), V(0, 0, 1), V(0, 1, 1)));
    form_factors::mesh_t meshes[2] = {{0, 2, 0}, {2, 2, 0}};
    form_factors::scene_t scene = {4, faces.data(), 2, meshes};
    f->methods->set_scene(f, &scene);
    CHECK(f->methods->prepare(f) == FORM_FACTORS_OK);
    float ff[4];
    form_factors::task_t task = {40000, ff};
    CHECK(f->methods->calculate(f, &task) == FORM_FACTORS_OK);
    CHECK(std::fabs(ff[2] - vf_perpendicular(1, 1, 1) / 2) < 0.01);
    C.free_(f, e, r);
  }
  {
    g_case = std::string(C.name) + " box";
    form_factors::system_t* f;
    emission::system_t* e;
    ray_caster::system_t* r;
    C.make(&f, &e, &r);
    vec3 v[] = {V(0, 0, 0), V(1, 0, 0), V(1, 1, 0), V(0, 1, 0), V(0, 0, 1), V(1, 0, 1), V(1, 1, 1), V(0, 1, 1)};
    math::triangle_t faces[12];
    faces[0] = T(v[0], v[1], v[2]);
    faces[1] = T(v[0], v[3], v[2]);
    faces[8] = T(v[0], v[1], v[5]);
    faces[9] = T(v[0], v[4], v[5]);
    faces[4] = T(v[0], v[3], v[7]);
    faces[5] = T(v[0], v[4], v[7]);
    faces[6] = T(v[1], v[2], v[6]);
    faces[7] = T(v[1], v[5], v[6]);
    faces[2] = T(v[3], v[2], v[6]);
    faces[3] = T(v[3], v[7], v[6]);
    faces[10] = T(v[4], v[5], v[6]);
    faces[11] = T(v[4], v[7], v[6]);
    form_factors::mesh_t mesh = {0, 12, 0};
    form_factors::scene_t scene = {12, faces, 1, &mesh};
    f->methods->set_scene(f, &scene);
    CHECK(f->methods->prepare(f) == FORM_FACTORS_OK);
    float ff[1];
    form_factors::task_t task = {40000, ff};
    CHECK(f->methods->calculate(f, &task) == FORM_FACTORS_OK);
    CHECK(std::fabs(ff[0] - 0.5f) < 0.01);
    C.free_(f, e, r);
  }
  {
    g_case = std::string(C.name) + " empty scene";
    form_factors::system_t* f;
    emission::system_t* e;
    ray_caster::system_t* r;
    C.make(&f, &e, &r);
    form_factors::scene_t scene = {0, 0, 0, 0};
    f->methods->set_scene(f, &scene);
    CHECK(f->methods->prepare(f) == -FORM_FACTORS_EMPTY_SCENE);
    C.free_(f, e, r);
  }
}

// Emission: the batch layout of emission/malley_cpu.cpp:142-189 and the ray
// budget of emission/malley_emission.cpp:50-60.
static void emission_suite()
{
  g_case = "B200 emission";
  ray_caster::system_t* r = b200_ray_caster::create();
  emission::system_t* e = b200_emission::create(r);
  std::vector<math::triangle_t> faces = square(V(0, 0, 0));
  std::vector<math::triangle_t> top = square(V(0, 0, 1));
  faces.insert(faces.end(), top.begin(), top.end());
  ray_caster::scene_t scene = {4, faces.data()};
  CHECK(e->methods->set_scene(e, &scene) == EMISSION_OK);
  float w[8] = {1, 1, 2, 0, 0.5f, 0.5f, 0, 0};
  malley_emission::task_t task(1000, 5.f, w);
  CHECK(e->methods->calculate(e, &task) == EMISSION_OK);
  // 200+200, 400+0, 100+100, 0+0 rays
  CHECK(task.rays && task.rays->n_tasks == 1000);
  if (task.rays) {
    int hits = 0;
    for (int i = 0; i < task.rays->n_tasks; ++i) {
      math::ray_t ray = task.rays->ray[i];
      // origins lie on the emitting face (z = 0 for faces 0-1, z = 1 for face 2)
      const int face = i < 400 ? 0 : (i < 800 ? 1 : 2);
      const float z = face < 2 ? 0.f : 1.f;
      CHECK(std::fabs(ray.origin.z - z) < 2e-4f);
      // front rays of face 0 point up (+z), rear rays down
      if (face == 0)
        CHECK((i < 200) == (ray.direction.z > ray.origin.z));
      hits += task.rays->hit_face[i] != 0;
    }
    CHECK(hits > 50);
    free(task.rays->ray);
    free(task.rays->hit_face);
    free(task.rays->hit_point);
    free(task.rays);
  }
  b200_emission::destroy(e);
  b200_ray_caster::destroy(r);
}

// ---------------------------------------------------------------------------
// Ray-traced thermal equations (thermal_equation/radiance_cpu.cpp,
// thermal_equation/parallel_rays_cpu.cpp) and the parallel-rays emitter.
// ---------------------------------------------------------------------------
// The unit cube as 6 meshes of 2 triangles with inward normals.
static std::vector<math::triangle_t> cube_inward()
{
  const vec3 c = V(0.5f, 0.5f, 0.5f);
  const vec3 q[6][4] = {{V(0, 0, 0), V(1, 0, 0), V(1, 1, 0), V(0, 1, 0)}, {V(0, 0, 1), V(1, 0, 1), V(1, 1, 1), V(0, 1, 1)},
                        {V(0, 0, 0), V(1, 0, 0), V(1, 0, 1), V(0, 0, 1)}, {V(0, 1, 0), V(1, 1, 0), V(1, 1, 1), V(0, 1, 1)},
                        {V(0, 0, 0), V(0, 1, 0), V(0, 1, 1), V(0, 0, 1)}, {V(1, 0, 0), V(1, 1, 0), V(1, 1, 1), V(1, 0, 1)}};
  std::vector<math::triangle_t> out;
  for (int k = 0; k < 6; ++k) {
    math::triangle_t t[2] = {T(q[k][0], q[k][1], q[k][2]), T(q[k][0], q[k][2], q[k][3])};
    for (math::triangle_t& x : t) {
      const vec3 u = sub(x.points[1], x.points[0]), w = sub(x.points[2], x.points[0]);
      const vec3 n = V(u.y * w.z - u.z * w.y, u.z * w.x - u.x * w.z, u.x * w.y - u.y * w.x);
      const vec3 in = sub(c, x.points[0]);
      if (n.x * in.x + n.y * in.y + n.z * in.z < 0)
        std::swap(x.points[1], x.points[2]);
      out.push_back(x);
    }
  }
  return out;
}

static subject::material_t optics_material(float emis_front, float emis_rear, float abs_front, float abs_rear)
{
  subject::material_t m;
  std::memset(&m, 0, sizeof m);
  m.front.emissivity = emis_front;
  m.rear.emissivity = emis_rear;
  m.front.absorbance = abs_front;
  m.rear.absorbance = abs_rear;
  return m;
}

static bool within(float a, float b, float rel) { return std::fabs(a - b) <= rel * std::fabs(b); }

static parallel_rays_cpu::source_t sun_from_above(void*)
{
  parallel_rays_cpu::source_t s;
  s.power = 1000.f;
  s.direction = V(0, 0, -1);
  return s;
}

static void thermal_suite()
{
  std::vector<math::triangle_t> faces = cube_inward();
  subject::mesh_t meshes[6];
  for (int m = 0; m < 6; ++m)
    meshes[m] = subject::mesh_t{2 * m, 2, m % 2};
  subject::material_t materials[2] = {optics_material(0.9f, 0.f, 0.8f, 0.6f), optics_material(0.5f, 0.f, 0.7f, 0.3f)};
  subject::scene_t scene = {12, faces.data(), 6, meshes, 2, materials};
  const float temps[6] = {300, 320, 340, 360, 380, 400};
  const int n_rays = 200000;

  g_case = "B200 radiance (fused): energy";
  float em[6] = {0}, ab[6] = {0};
  {
    radiance_equation::params_t params = {0, n_rays};
    thermal_equation::system_t* eq = b200_radiance_equation::create(&params);
    CHECK(eq->methods->set_scene(eq, &scene) == THERMAL_EQUATION_OK);
    thermal_equation::task_t task = {temps, em, ab};
    CHECK(eq->methods->calculate(eq, &task) == THERMAL_EQUATION_OK);
    float se = 0, sa = 0;
    for (int m = 0; m < 6; ++m) {
      se += em[m];
      sa += ab[m];
    }
    // inward emitters only: every ray lands but for the few float rounding
    // lets through the seams between walls
    CHECK(se > 0 && sa <= se * 1.0001f && sa > se * 0.998f);
    b200_radiance_equation::destroy(eq);
  }

  g_case = "B200 distant source (fused): projected area";
  {
    parallel_rays_cpu::params_t params = {n_rays, 0, 0, &sun_from_above};
    thermal_equation::system_t* eq = b200_distant_source::create(&params);
    CHECK(eq->methods->set_scene(eq, &scene) == THERMAL_EQUATION_OK);
    float a[6] = {0}, e[6] = {0};
    thermal_equation::task_t task = {temps, e, a};
    CHECK(eq->methods->calculate(eq, &task) == THERMAL_EQUATION_OK);
    // straight down: only the top (mesh 1, material 1) is hit, from outside,
    // i.e. on its rear side: 1 m^2 of 1000 W/m^2 at rear absorbance 0.3
    CHECK(within(a[1], 300.f, 0.02f));
    CHECK(a[0] == 0 && a[2] == 0 && a[3] == 0 && a[4] == 0 && a[5] == 0);
    b200_distant_source::destroy(eq);
  }

  g_case = "B200 parallel-rays emitter";
  {
    ray_caster::system_t* r = b200_ray_caster::create();
    emission::system_t* e = b200_parallel_rays_emission::create(r);
    ray_caster::scene_t rs = {12, faces.data()};
    CHECK(e->methods->set_scene(e, &rs) == EMISSION_OK);
    // the reference's task type has no constructor: it lives in malloc'd
    // memory (thermal_equation/parallel_rays_cpu.cpp:27-38)
    alignas(parallel_rays_emission_cpu::task_t) unsigned char storage[sizeof(parallel_rays_emission_cpu::task_t)];
    parallel_rays_emission_cpu::task_t& task = *reinterpret_cast<parallel_rays_emission_cpu::task_t*>(storage);
    task.n_rays = 1000;
    task.rays = 0;
    task.direction = V(0, 0, -1);
    task.center = V(0.5f, 0.5f, 0.5f);
    task.distance = 3.f;
    task.radius = 0.5f;
    CHECK(e->methods->calculate(e, &task) == EMISSION_OK);
    CHECK(task.rays && task.rays->n_tasks == 1000);
    if (task.rays) {
      int hits = 0;
      for (int i = 0; i < 1000; ++i) {
        const math::ray_t ray = task.rays->ray[i];
        CHECK(std::fabs(ray.origin.z - 3.5f) < 1e-5f && std::fabs(ray.direction.z - 3.4f) < 1e-5f);
        hits += task.rays->hit_face[i] == &faces[2] || task.rays->hit_face[i] == &faces[3];
      }
      CHECK(hits == 1000);  // a disc of radius 0.5 about the centre lands on the top
      task_free_all(task.rays);
    }
    b200_parallel_rays_emission::destroy(e);
    b200_ray_caster::destroy(r);
  }

#ifdef FFB_WITH_REFERENCE
  g_case = "B200 radiance vs reference radiance_cpu";
  {
    ray_caster::system_t* rc = ray_caster::system_create(RAY_CASTER_NAIVE_CPU);
    emission::system_t* me = emission::system_create(EMISSION_MALLEY_CPU, rc);
    radiance_equation::params_t rp = {me, n_rays};
    thermal_equation::system_t* ref = radiance_equation::system_create();
    thermal_equation::system_init(ref, &rp);
    CHECK(thermal_equation::system_set_scene(ref, &scene) == THERMAL_EQUATION_OK);
    float rem[6] = {0}, rab[6] = {0};
    thermal_equation::task_t rt = {temps, rem, rab};
    CHECK(thermal_equation::system_calculate(ref, &rt) == THERMAL_EQUATION_OK);
    for (int m = 0; m < 6; ++m) {
      CHECK(em[m] == rem[m]);
      CHECK(within(ab[m], rab[m], 0.03f));
    }
    // the B200 equation has no host absorption path: over the reference's
    // emitter it refuses at init
    radiance_equation::params_t gp = {me, n_rays};
    thermal_equation::system_t* mixed = b200_radiance_equation::system_create();
    CHECK(mixed->methods->init(mixed, &gp) == -THERMAL_EQUATION_ERROR);
    b200_radiance_equation::destroy(mixed);
    thermal_equation::system_free(ref);
    emission::system_free(me);
    ray_caster::system_free(rc);
  }

  g_case = "B200 distant source vs reference parallel_rays_cpu";
  {
    ray_caster::system_t* rc = ray_caster::system_create(RAY_CASTER_NAIVE_CPU);
    emission::system_t* pe = emission::system_create(EMISSION_PARALLEL_RAYS_CPU, rc);
    parallel_rays_cpu::params_t rp = {n_rays, pe, 0, &sun_from_above};
    thermal_equation::system_t* ref = parallel_rays_cpu::system_create();
    thermal_equation::system_init(ref, &rp);
    CHECK(thermal_equation::system_set_scene(ref, &scene) == THERMAL_EQUATION_OK);
    float ra[6] = {0}, re[6] = {0};
    thermal_equation::task_t rt = {temps, re, ra};
    CHECK(thermal_equation::system_calculate(ref, &rt) == THERMAL_EQUATION_OK);
    CHECK(within(ra[1], 300.f, 0.02f));
    // over the reference's emitter the B200 equation refuses at init
    thermal_equation::system_t* mixed = b200_distant_source::system_create();
    CHECK(mixed->methods->init(mixed, &rp) == -THERMAL_EQUATION_ERROR);
    b200_distant_source::destroy(mixed);
    thermal_equation::system_free(ref);
    emission::system_free(pe);
    ray_caster::system_free(rc);
  }
#endif
}

// CSV export (import_export/csv_export.cpp:26-46): the B200 export writes
// the reference's bytes; with the reference built in, the two files are
// compared whole.
static std::string read_file(const char* path)
{
  std::string out;
  FILE* f = std::fopen(path, "rb");
  if (!f)
    return out;
  char buf[4096];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof buf, f)) > 0)
    out.append(buf, k);
  std::fclose(f);
  return out;
}

static void csv_suite()
{
  g_case = "B200 csv export";
  float ff[9] = {0.5f, 0.25f, 0.f, 1.f, 1e-5f, 1.f / 3.f, 123456.7f, -0.f, 2.f};
  form_factors::scene_t scene = {0, 0, 3, 0};
  form_factors::task_t task = {0, ff};
  const char* path = "test_systems_b200.csv";
  CHECK(b200_csv_export::export_csv(path, &scene, &task) == CSV_EXPORT_OK);
  CHECK(read_file(path) == "0.5;0.25;0\n1;1e-05;0.333333\n123457;-0;2\n");
  CHECK(b200_csv_export::export_csv("no_such_dir/x.csv", &scene, &task) == -CSV_EXPORT_FILE_ERROR);
#ifdef FFB_WITH_REFERENCE
  std::vector<float> big(257 * 257);
  for (size_t i = 0; i < big.size(); ++i)
    big[i] = (float)((i * 2654435761u) % 10007u) * (1.f / (float)(1 + i % 977u));
  form_factors::scene_t s2 = {0, 0, 257, 0};
  form_factors::task_t t2 = {0, big.data()};
  CHECK(csv_export::export_csv("test_systems_ref.csv", &s2, &t2) == CSV_EXPORT_OK);
  CHECK(b200_csv_export::export_csv(path, &s2, &t2) == CSV_EXPORT_OK);
  CHECK(read_file(path) == read_file("test_systems_ref.csv"));
  CHECK(csv_export::export_csv("no_such_dir/x.csv", &s2, &t2) == -CSV_EXPORT_FILE_ERROR);
  std::remove("test_systems_ref.csv");
#endif
  std::remove(path);
}

// OBJ import (import_export/obj_import.cpp:167-340)
static void obj_suite()
{
  g_case = "B200 obj import";
  const char* path = "test_systems_scene.obj";
  FILE* f = std::fopen(path, "wb");
  std::fputs("# two objects\no first\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0.5e0\nf 1 2 3\n"
             "g second\nvn 0 0 1\nf 2//1 4//1 3//1\nf 1/1/1 2/2/2 4/4/4\n", f);
  std::fclose(f);
  subject::scene_t* s = 0;
  CHECK(b200_obj_import::scene(path, &s) == OBJ_IMPORT_OK);
  if (s) {
    CHECK(s->n_faces == 3 && s->n_meshes == 2 && s->n_materials == 1);
    CHECK(s->meshes[0].first_idx == 0 && s->meshes[0].n_faces == 1 && s->meshes[1].n_faces == 2);
    CHECK(s->faces[1].points[1].z == 0.5f && std::strcmp(s->materials[0].name, "black_body") == 0);
#ifdef FFB_WITH_REFERENCE
    subject::scene_t* r = 0;
    CHECK(obj_import::scene(path, &r) == OBJ_IMPORT_OK);
    if (r) {
      CHECK(r->n_faces == s->n_faces && r->n_meshes == s->n_meshes && r->n_materials == s->n_materials);
      CHECK(std::memcmp(r->faces, s->faces, sizeof(subject::face_t) * s->n_faces) == 0);
      CHECK(std::memcmp(r->meshes, s->meshes, sizeof(subject::mesh_t) * s->n_meshes) == 0);
      CHECK(std::memcmp(r->materials, s->materials, sizeof(subject::material_t) * s->n_materials) == 0);
      subject::scene_free(r);
    }
#endif
    free(s->faces);
    free(s->meshes);
    free(s->materials);
    free(s);
  }
  CHECK(b200_obj_import::scene("no_such_file.obj", &s) == -OBJ_IMPORT_FILE_ERROR);
  std::remove(path);
}

// The B200 form-factor and thermal types run emission, trace and tallies
// fused on the GPU and have no host path: an emitter of another type is
// refused at init with the type's negative error code.
static int foreign_init(emission::system_t*, ray_caster::system_t*) { return EMISSION_OK; }
static int foreign_shutdown(emission::system_t*) { return EMISSION_OK; }
static int foreign_set_scene(emission::system_t*, ray_caster::scene_t*) { return EMISSION_OK; }
static int foreign_calculate(emission::system_t*, emission::task_t*) { return EMISSION_OK; }

static void refusal_suite()
{
  static const emission::system_methods_t foreign_methods = {&foreign_init, &foreign_shutdown, &foreign_set_scene,
                                                             &foreign_calculate};
  emission::system_t foreign;
  foreign.methods = &foreign_methods;

  g_case = "B200 form factors refuse a foreign emitter";
  {
    form_factors::system_t* f = b200_form_factors::system_create();
    CHECK(f->methods->init(f, &foreign) == -FORM_FACTORS_ERROR);
    b200_form_factors::destroy(f);
  }
  g_case = "B200 radiance refuses a foreign emitter";
  {
    radiance_equation::params_t p = {&foreign, 1000};
    thermal_equation::system_t* eq = b200_radiance_equation::system_create();
    CHECK(eq->methods->init(eq, &p) == -THERMAL_EQUATION_ERROR);
    b200_radiance_equation::destroy(eq);
  }
  g_case = "B200 distant source refuses a foreign emitter";
  {
    parallel_rays_cpu::params_t p = {1000, &foreign, 0, &sun_from_above};
    thermal_equation::system_t* eq = b200_distant_source::system_create();
    CHECK(eq->methods->init(eq, &p) == -THERMAL_EQUATION_ERROR);
    b200_distant_source::destroy(eq);
  }
#ifdef FFB_WITH_REFERENCE
  g_case = "B200 form factors refuse the reference's malley_cpu";
  {
    ray_caster::system_t* r = ray_caster::system_create(RAY_CASTER_NAIVE_CPU);
    emission::system_t* e = emission::system_create(EMISSION_MALLEY_CPU, r);
    form_factors::system_t* f = b200_form_factors::system_create();
    CHECK(f->methods->init(f, e) == -FORM_FACTORS_ERROR);
    b200_form_factors::destroy(f);
    emission::system_free(e);
    ray_caster::system_free(r);
  }
#endif
}

int main()
{
  refusal_suite();
  csv_suite();
  obj_suite();
  thermal_suite();
  for (const Caster& c : casters())
    ray_caster_suite(c);
  emission_suite();
  for (const Calculator& c : calculators())
    form_factor_suite(c);
  std::printf("%d checks, %d failures\n", g_checks, g_failures);
  return g_failures == 0 ? 0 : 1;
}
