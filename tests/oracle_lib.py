"""ctypes bindings to the CPU checkers under oracle/ (test infrastructure only).

* ``Oracle``   -- oracle/_build/libffo.so, the C restatement of the reference
  algorithm (oracle/ffo.c).  Built on demand with make when missing.
* ``Reference`` -- oracle/_ref/libffref.so, the reference's own CPU code compiled
  from its sources (oracle/Makefile, target ``ref``).  Only present where the
  reference sources were available when the repository was built; tests that
  need it skip without it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "libffo.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libffref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    """The C restatement (oracle/ffo.c)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)
        lib = C.CDLL(ORACLE_SO)
        lib.ffo_set_threads.argtypes = [C.c_int]
        lib.ffo_triangle_intersect.argtypes = [_f32p, _f32p, _f32p]
        lib.ffo_triangle_intersect.restype = C.c_int
        lib.ffo_cast_naive.argtypes = [C.c_int, _f32p, C.c_long, _f32p, _i32p, C.c_void_p]
        lib.ffo_emitted.argtypes = [C.c_int, C.c_float, C.c_float]
        lib.ffo_emitted.restype = C.c_int
        lib.ffo_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        lib.ffo_sincos_turn24.argtypes = [C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.ffo_rotate_towards.argtypes = [_f32p, _f32p, _f32p]
        lib.ffo_face_frame.argtypes = [_f32p, C.c_int, _f32p]
        lib.ffo_emit.argtypes = [C.c_int, _f32p, _i32p, _i32p, C.c_uint64, C.c_uint32, C.c_int, _f32p]
        lib.ffo_form_factor_counts.argtypes = [C.c_int, _f32p, _i32p, _i32p, C.c_uint64, C.c_uint32,
                                               C.c_int, _u32p]
        lib.ffo_vf_parallel.argtypes = [C.c_double] * 3
        lib.ffo_vf_parallel.restype = C.c_double
        lib.ffo_vf_perpendicular.argtypes = [C.c_double] * 3
        lib.ffo_vf_perpendicular.restype = C.c_double
        lib.ffo_disc_source.argtypes = [_f32p, _f32p, C.c_float, C.c_float, _f32p]
        lib.ffo_emit_parallel.argtypes = [_f32p, C.c_long, C.c_uint64, C.c_uint32, _f32p]
        lib.ffo_parallel_rays.argtypes = [C.c_int, _f32p, _f32p, C.c_long, C.c_uint64, C.c_uint32, _u32p]
        lib.ffo_radiance_absorption.argtypes = [C.c_int, _f32p, _i32p, _i32p, _f32p, _f32p, _i32p, C.c_int,
                                                C.c_uint64, C.c_uint32, C.c_int, _f64p]
        self.lib = lib

    def disc_source(self, direction, center, distance, radius):
        d = np.zeros(17, np.float32)
        self.lib.ffo_disc_source(_f32(direction), _f32(center), float(distance), float(radius), d)
        return d

    def emit_parallel(self, disc, n_rays, seed, epoch=0):
        rays = np.zeros((int(n_rays), 6), np.float32)
        self.lib.ffo_emit_parallel(_f32(disc), int(n_rays), int(seed), int(epoch), rays)
        return rays

    def parallel_rays(self, faces, disc, n_rays, seed, epoch=0):
        faces = _f32(faces).reshape(-1, 9)
        out = np.zeros((len(faces), 2), np.uint32)
        self.lib.ffo_parallel_rays(len(faces), faces, _f32(disc), int(n_rays), int(seed), int(epoch), out)
        return out

    def radiance_absorption(self, faces, front, rear, power_front, power_rear, face_to_mesh, n_meshes, seed,
                            epoch=0, flags=0):
        faces = _f32(faces).reshape(-1, 9)
        out = np.zeros(int(n_meshes), np.float64)
        self.lib.ffo_radiance_absorption(len(faces), faces, _i32(front), _i32(rear), _f32(power_front),
                                         _f32(power_rear), _i32(face_to_mesh), int(n_meshes), int(seed), int(epoch),
                                         int(flags), out)
        return out

    def set_threads(self, n):
        self.lib.ffo_set_threads(int(n))

    def triangle_intersect(self, ray6, tri9):
        pt = np.zeros(3, np.float32)
        code = self.lib.ffo_triangle_intersect(_f32(ray6), _f32(tri9), pt)
        return code, pt

    def cast_naive(self, faces, rays, want_points=True):
        faces = _f32(faces).reshape(-1, 9)
        rays = _f32(rays).reshape(-1, 6)
        hit = np.empty(len(rays), np.int32)
        pts = np.full((len(rays), 3), np.nan, np.float32) if want_points else None
        self.lib.ffo_cast_naive(len(faces), faces, len(rays), rays, hit,
                                pts.ctypes.data if want_points else None)
        return hit, pts

    def emitted(self, n_rays, weight, total):
        return self.lib.ffo_emitted(int(n_rays), float(weight), float(total))

    def philox(self, ctr, key):
        out = np.zeros(4, np.uint32)
        self.lib.ffo_philox4x32_10(np.ascontiguousarray(ctr, np.uint32),
                                   np.ascontiguousarray(key, np.uint32), out)
        return out

    def sincos_turn24(self, k):
        s, c = C.c_float(), C.c_float()
        self.lib.ffo_sincos_turn24(int(k), C.byref(s), C.byref(c))
        return s.value, c.value

    def rotate_towards(self, subject, to):
        m = np.zeros(9, np.float32)
        self.lib.ffo_rotate_towards(_f32(subject), _f32(to), m)
        return m.reshape(3, 3)

    def face_frame(self, tri9, flags=0):
        out = np.zeros(18, np.float32)
        self.lib.ffo_face_frame(_f32(tri9), int(flags), out)
        return out

    def emit(self, faces, front, rear, seed, epoch=0, flags=0):
        faces = _f32(faces).reshape(-1, 9)
        front, rear = _i32(front), _i32(rear)
        n = int(front.sum() + rear.sum())
        rays = np.zeros((n, 6), np.float32)
        self.lib.ffo_emit(len(faces), faces, front, rear, int(seed), int(epoch), int(flags), rays)
        return rays

    def form_factor_counts(self, faces, front, rear, seed, epoch=0, flags=0):
        faces = _f32(faces).reshape(-1, 9)
        n = len(faces)
        counts = np.zeros((n, n), np.uint32)
        self.lib.ffo_form_factor_counts(n, faces, _i32(front), _i32(rear), int(seed), int(epoch),
                                        int(flags), counts)
        return counts

    def vf_parallel(self, a, b, c):
        return self.lib.ffo_vf_parallel(a, b, c)

    def vf_perpendicular(self, h, w, l):
        return self.lib.ffo_vf_perpendicular(h, w, l)


class Reference:
    """The reference's own CPU path (oracle/_ref/libffref.so)."""

    NAIVE_CPU = 1
    ZGRID_CPU = 3

    @staticmethod
    def available():
        return os.path.exists(REF_SO)

    def __init__(self):
        lib = C.CDLL(REF_SO)
        lib.ffref_triangle_intersect.argtypes = [_f32p, _f32p, _f32p]
        lib.ffref_triangle_intersect.restype = C.c_int
        lib.ffref_rotate_towards.argtypes = [_f32p, _f32p, _f32p]
        lib.ffref_emitted.argtypes = [C.c_int, C.c_float, C.c_float]
        lib.ffref_emitted.restype = C.c_int
        lib.ffref_cast.argtypes = [C.c_int, C.c_int, _f32p, C.c_long, _f32p, _i32p, C.c_void_p,
                                   C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.ffref_cast.restype = C.c_int
        lib.ffref_emit.argtypes = [C.c_int, _f32p, C.c_int, _f32p, C.c_float, C.c_void_p, C.c_long]
        lib.ffref_emit.restype = C.c_long
        lib.ffref_form_factors.argtypes = [C.c_int, _f32p, C.c_int, _i32p, C.c_int, C.c_int, C.c_int,
                                           _f32p]
        lib.ffref_form_factors.restype = C.c_int
        lib.ffref_step_open.argtypes = [C.c_int, C.c_int, _f32p, C.POINTER(C.c_double)]
        lib.ffref_step_open.restype = C.c_void_p
        lib.ffref_step_run.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_float, _u8p, C.c_int,
                                       C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.ffref_step_run.restype = C.c_long
        lib.ffref_step_close.argtypes = [C.c_void_p]
        lib.ffref_export_csv.argtypes = [C.c_char_p, C.c_int, _f32p]
        lib.ffref_export_csv.restype = C.c_int
        lib.ffref_radiance.argtypes = [C.c_int, C.c_int, _f32p, C.c_int, _i32p, C.c_int, _f32p, _f32p, C.c_int,
                                       _f32p, _f32p]
        lib.ffref_radiance.restype = C.c_int
        lib.ffref_parallel_rays.argtypes = [C.c_int, C.c_int, _f32p, C.c_int, _i32p, C.c_int, _f32p, C.c_int,
                                            C.c_float, _f32p, _f32p]
        lib.ffref_parallel_rays.restype = C.c_int
        lib.ffref_bsphere.argtypes = [C.c_int, _f32p, _f32p, C.POINTER(C.c_float)]
        lib.ffref_obj_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), _i32p]
        lib.ffref_obj_load.restype = C.c_int
        lib.ffref_obj_copy.argtypes = [C.c_void_p, _f32p, _i32p, C.c_void_p]
        lib.ffref_obj_free.argtypes = [C.c_void_p]
        self.lib = lib

    def obj_scene(self, filename):
        """obj_import::scene: (status, faces (n, 9), meshes (m, 3), materials
        as raw 184-byte records)."""
        h = C.c_void_p()
        counts = np.zeros(3, np.int32)
        rc = self.lib.ffref_obj_load(os.fsencode(filename), C.byref(h), counts)
        if rc != 0 or not h.value:
            return rc, None, None, None
        faces = np.zeros((counts[0], 9), np.float32)
        meshes = np.zeros((counts[1], 3), np.int32)
        materials = np.zeros(counts[2] * 184, np.uint8)
        self.lib.ffref_obj_copy(h, faces, meshes, materials.ctypes.data)
        self.lib.ffref_obj_free(h)
        return rc, faces, meshes, materials

    def radiance(self, faces, meshes, materials, temperatures, n_rays, caster=3):
        """radiance_equation calculate() with malley_cpu over caster `caster`:
        (status, emission, absorption) per mesh."""
        faces = _f32(faces).reshape(-1, 9)
        m3 = np.ascontiguousarray(np.asarray(meshes, np.int32).reshape(-1, 3))
        opt = _f32(np.asarray(materials, np.float32).reshape(-1, 4))
        em = np.zeros(len(m3), np.float32)
        ab = np.zeros(len(m3), np.float32)
        rc = self.lib.ffref_radiance(int(caster), len(faces), faces, len(m3), m3, len(opt), opt,
                                     _f32(temperatures), int(n_rays), em, ab)
        return rc, em, ab

    def parallel_rays(self, faces, meshes, materials, n_rays, power, direction, caster=3):
        """parallel_rays_cpu calculate() (distant source): (status, absorption)."""
        faces = _f32(faces).reshape(-1, 9)
        m3 = np.ascontiguousarray(np.asarray(meshes, np.int32).reshape(-1, 3))
        opt = _f32(np.asarray(materials, np.float32).reshape(-1, 4))
        ab = np.zeros(len(m3), np.float32)
        rc = self.lib.ffref_parallel_rays(int(caster), len(faces), faces, len(m3), m3, len(opt), opt, int(n_rays),
                                          float(power), _f32(direction), ab)
        return rc, ab

    def bsphere(self, faces):
        faces = _f32(faces).reshape(-1, 9)
        c = np.zeros(3, np.float32)
        r = C.c_float()
        self.lib.ffref_bsphere(len(faces), faces, c, C.byref(r))
        return c, np.float32(r.value)

    def export_csv(self, filename, ff):
        """csv_export::export_csv of an n x n float matrix; returns the
        reference's status (0, or -31 when the file cannot be opened)."""
        ff = np.ascontiguousarray(ff, np.float32)
        return self.lib.ffref_export_csv(os.fsencode(filename), int(ff.shape[0]), ff)

    def csv_text(self, ff, tmpdir):
        path = os.path.join(str(tmpdir), "ref_%d.csv" % os.getpid())
        rc = self.export_csv(path, ff)
        assert rc == 0, rc
        with open(path, "rb") as f:
            return f.read()

    def triangle_intersect(self, ray6, tri9):
        pt = np.zeros(3, np.float32)
        code = self.lib.ffref_triangle_intersect(_f32(ray6), _f32(tri9), pt)
        return code, pt

    def rotate_towards(self, subject, to):
        m = np.zeros(9, np.float32)
        self.lib.ffref_rotate_towards(_f32(subject), _f32(to), m)
        return m.reshape(3, 3)

    def emitted(self, n_rays, weight, total):
        return self.lib.ffref_emitted(int(n_rays), float(weight), float(total))

    def cast(self, caster, faces, rays, threads=1, want_points=True):
        faces = _f32(faces).reshape(-1, 9)
        rays = _f32(rays).reshape(-1, 6)
        hit = np.empty(len(rays), np.int32)
        pts = np.full((len(rays), 3), np.nan, np.float32) if want_points else None
        tp, tc = C.c_double(), C.c_double()
        rc = self.lib.ffref_cast(caster, len(faces), faces, len(rays), rays, hit,
                                 pts.ctypes.data if want_points else None, int(threads),
                                 C.byref(tp), C.byref(tc))
        if rc < 0:
            raise RuntimeError("reference cast failed: %d" % rc)
        return hit, pts, tp.value, tc.value

    def emit(self, faces, n_rays, weights2, total_weight):
        faces = _f32(faces).reshape(-1, 9)
        w = _f32(weights2)
        n = self.lib.ffref_emit(len(faces), faces, int(n_rays), w, float(total_weight), None, 0)
        if n < 0:
            raise RuntimeError("reference emission failed: %d" % n)
        rays = np.zeros((max(n, 1), 6), np.float32)
        self.lib.ffref_emit(len(faces), faces, int(n_rays), w, float(total_weight), rays.ctypes.data, n)
        return rays[:n]

    def form_factors(self, faces, meshes, n_rays, caster=ZGRID_CPU, n_calls=1):
        faces = _f32(faces).reshape(-1, 9)
        meshes = _i32(meshes).reshape(-1, 3)
        m = len(meshes)
        out = np.zeros(m * m, np.float32)
        rc = self.lib.ffref_form_factors(len(faces), faces, m, meshes, int(n_rays), caster,
                                         int(n_calls), out)
        return rc, out.reshape(m, m)
