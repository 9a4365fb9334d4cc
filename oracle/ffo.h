/*
 * ffo.h -- CPU oracle for the form-factor path (test infrastructure only;
 * see ffo.c).  Plain C, loaded by the Python tests through ctypes.
 */
#ifndef FFO_H
#define FFO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Result codes of the ray/triangle test (math/triangle.h:27-30). */
#define FFO_UNIQUE 0
#define FFO_DISJOINT 1
#define FFO_DEGENERATE 2
#define FFO_SAME_PLANE 3

/* Emission flag: rotate +z towards the raw (unnormalised) cross-product
 * normal exactly as emission/malley_cpu.cpp:125-129 does.  Without it the
 * normal is normalised first, which makes the directions cosine-weighted for
 * any triangle size. */
#define FFO_EMIT_REF_NORMAL 1

/* (pi/4) / 2^21 rounded to float: one step of the 24-bit turn counter
 * inside an octant. */
#define FFO_QUARTER_PI_OVER_2P21 0x1.921fb6p-22f

void ffo_set_threads(int n); /* 0 = all online cores */
int ffo_triangle_intersect(const float* ray6, const float* tri9, float* point3);
void ffo_cast_naive(int n_faces, const float* faces9, long n_rays, const float* rays6,
                    int32_t* hit, float* hit_pt);
int ffo_emitted(int n_rays, float weight, float total_weight);
void ffo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void ffo_sincos_turn24(uint32_t k, float* s, float* c);
void ffo_rotate_towards(const float* subject3, const float* to3, float* m9);
void ffo_face_frame(const float* tri9, int flags, float* frame18);
void ffo_emit_ray(const float* frame18, uint32_t face, uint32_t j, int front,
                  uint64_t seed, uint32_t epoch, float* ray6);
void ffo_emit(int n_faces, const float* faces9, const int32_t* front, const int32_t* rear,
              uint64_t seed, uint32_t epoch, int flags, float* rays6);
void ffo_form_factor_counts(int n_faces, const float* faces9, const int32_t* front,
                            const int32_t* rear, uint64_t seed, uint32_t epoch, int flags,
                            uint32_t* counts);
void ffo_disc_source(const float* direction3, const float* center3, float distance, float radius, float* disc17);
void ffo_emit_disc_ray(const float* disc17, uint64_t j, uint64_t seed, uint32_t epoch, float* ray6);
void ffo_emit_parallel(const float* disc17, long n_rays, uint64_t seed, uint32_t epoch, float* rays6);
void ffo_parallel_rays(int n_faces, const float* faces9, const float* disc17, long n_rays, uint64_t seed,
                       uint32_t epoch, uint32_t* side_counts);
void ffo_radiance_absorption(int n_faces, const float* faces9, const int32_t* front, const int32_t* rear,
                             const float* power_front, const float* power_rear, const int32_t* face_to_mesh,
                             int n_meshes, uint64_t seed, uint32_t epoch, int flags, double* absorption);
double ffo_vf_parallel(double a, double b, double c);
double ffo_vf_perpendicular(double H, double W, double L);

#ifdef __cplusplus
}
#endif
#endif
