"""ctypes binding of libffb200.so (the C ABI of include/ffb.h).

Arguments may be numpy arrays (host memory; the library stages them) or
objects exposing ``data_ptr()`` such as CUDA torch tensors (device memory,
used in place).  Loading fails loudly when the library is missing: there is
no CPU fallback for any call.
"""
import ctypes as C
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libffb200.so")
HEADER = os.path.join(ROOT, "include", "ffb.h")

FFB_OK = 0
FFB_EMIT_REF_NORMAL = 1
FFB_ERR_FILE = -309
FFB_ERR_FORMAT = -310
ERRORS = {
    -301: "FFB_ERR_ARG", -302: "FFB_ERR_CUDA", -303: "FFB_ERR_NO_SCENE", -304: "FFB_ERR_NO_GRID",
    -305: "FFB_ERR_NO_MEMORY", -306: "FFB_ERR_TOO_LARGE", -307: "FFB_ERR_NO_DEVICE", -308: "FFB_ERR_TIMEOUT",
    -309: "FFB_ERR_FILE", -310: "FFB_ERR_FORMAT",
}


class FFBError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


class GridParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("cells_per_face", C.c_float),
                ("skip_empty", C.c_int)]


class GridInfo(C.Structure):
    _fields_ = [("lo", C.c_float * 3), ("hi", C.c_float * 3), ("cell", C.c_float * 3), ("nx", C.c_int),
                ("ny", C.c_int), ("nz", C.c_int), ("n_live_faces", C.c_int), ("n_refs", C.c_longlong),
                ("margin", C.c_float), ("skip_empty", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("tests", C.c_ulonglong), ("cells", C.c_ulonglong), ("rays", C.c_ulonglong),
                ("hits", C.c_ulonglong), ("kernel_ms", C.c_float), ("jumps", C.c_ulonglong),
                ("d2h_bytes", C.c_ulonglong)]


class DiscSource(C.Structure):
    """ffb_disc_source: the fields of parallel_rays_emission_cpu::task_t."""
    _fields_ = [("direction", C.c_float * 3), ("center", C.c_float * 3), ("distance", C.c_float),
                ("radius", C.c_float)]

    @classmethod
    def make(cls, direction, center, distance, radius):
        return cls((C.c_float * 3)(*direction), (C.c_float * 3)(*center), float(distance), float(radius))


class ObjInfo(C.Structure):
    _fields_ = [("n_vertices", C.c_int), ("n_faces", C.c_int), ("n_meshes", C.c_int), ("n_materials", C.c_int),
                ("status", C.c_int), ("error_line", C.c_int)]


# subject::material_t / ffb_material: 14 floats (shell, front, rear) and a name
MATERIAL_DTYPE = np.dtype([("props", "<f4", (14,)), ("name", "S128")])


class Mesh(C.Structure):
    _fields_ = [("first_idx", C.c_int), ("n_faces", C.c_int), ("material_idx", C.c_int)]


class Optics(C.Structure):
    _fields_ = [("front_emissivity", C.c_float), ("rear_emissivity", C.c_float), ("front_absorbance", C.c_float),
                ("rear_absorbance", C.c_float)]


def _meshes(meshes):
    """ffb_mesh array as a (n, 3) int32 numpy array (layout-identical)."""
    return np.ascontiguousarray(np.asarray(meshes, np.int32).reshape(-1, 3))


def _optics(materials):
    """ffb_optics array as a (n, 4) float32 numpy array (layout-identical)."""
    return np.ascontiguousarray(np.asarray(materials, np.float32).reshape(-1, 4))


def bounding_sphere(faces):
    """math::triangles_bsphere of a (n, 9) float32 face array: (center, radius)."""
    faces = np.ascontiguousarray(faces, np.float32)
    c = (C.c_float * 3)()
    r = C.c_float()
    _check(load().ffb_bounding_sphere(_ptr(faces), len(faces), c, C.byref(r)))
    return np.array(list(c), np.float32), np.float32(r.value)


class TraceShape(C.Structure):
    _fields_ = [("adv_per_iter", C.c_int), ("test_per_iter", C.c_int), ("refill_min", C.c_int),
                ("blocks_per_sm", C.c_int), ("coherent", C.c_int), ("lanes", C.c_int)]


class TuneResult(C.Structure):
    _fields_ = [("grid", GridParams), ("shape", C.c_int), ("sample_ms", C.c_float), ("from_cache", C.c_int),
                ("timed", C.c_int), ("sample_rays", C.c_longlong)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("error", C.c_int), ("n_faces", C.c_int), ("queue_s", C.c_double),
                ("latency_s", C.c_double), ("gpu_ms", C.c_double), ("trace_start_ns", C.c_ulonglong),
                ("trace_end_ns", C.c_ulonglong), ("slices", C.c_int), ("shape", C.c_int),
                ("cells_per_face", C.c_float)]


class ServerInfo(C.Structure):
    _fields_ = [("queued", C.c_int), ("running", C.c_int), ("peak_running", C.c_int),
                ("reserved_bytes", C.c_ulonglong), ("budget_bytes", C.c_ulonglong), ("peak_tracing", C.c_int)]


_lib = None


def declared_symbols(header=HEADER):
    """Function names declared in a C header (every `ffb_*(` prototype)."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ffb_\w+)\s*\(", text)))


def load(path=LIB_PATH):
    """Loads libffb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("%s is missing: run form_factors_b200.build.build() (or __graft_entry__.build())" % path)
    lib = C.CDLL(path)
    vp, i32, i64, u64, u32 = C.c_void_p, C.c_int, C.c_longlong, C.c_uint64, C.c_uint32
    sig = {
        "ffb_ctx_create": (i32, [i32, C.POINTER(vp)]),
        "ffb_ctx_destroy": (None, [vp]),
        "ffb_ctx_set_stream": (i32, [vp, vp]),
        "ffb_ctx_stream": (vp, [vp]),
        "ffb_ctx_synchronize": (i32, [vp]),
        "ffb_ctx_set_budget": (i32, [vp, C.c_ulonglong]),
        "ffb_ctx_set_stats": (i32, [vp, i32]),
        "ffb_ctx_set_host_threads": (i32, [vp, i32]),
        "ffb_ctx_host_threads": (i32, [vp]),
        "ffb_ctx_bytes": (C.c_ulonglong, [vp]),
        "ffb_last_error": (C.c_char_p, []),
        "ffb_scene_set": (i32, [vp, vp, i32]),
        "ffb_grid_build": (i32, [vp, C.POINTER(GridParams)]),
        "ffb_grid_info_get": (i32, [vp, C.POINTER(GridInfo)]),
        "ffb_grid_export": (i32, [vp, vp, vp]),
        "ffb_cast": (i32, [vp, vp, i64, vp, vp]),
        "ffb_cast_bruteforce": (i32, [vp, vp, i64, vp, vp]),
        "ffb_emit": (i32, [vp, vp, vp, u64, u32, i32, vp]),
        "ffb_form_factor_counts": (i32, [vp, vp, vp, u64, u32, i32, vp, i32, vp]),
        "ffb_normalise": (i32, [vp, vp, vp, i32, vp]),
        "ffb_csv_format": (i32, [vp, vp, i32, vp, C.c_ulonglong, C.POINTER(C.c_ulonglong)]),
        "ffb_csv_format_counts": (i32, [vp, vp, vp, i32, vp, C.c_ulonglong, C.POINTER(C.c_ulonglong)]),
        "ffb_csv_export": (i32, [vp, C.c_char_p, vp, i32]),
        "ffb_csv_export_counts": (i32, [vp, C.c_char_p, vp, vp, i32]),
        "ffb_stats_get": (i32, [vp, C.POINTER(Stats)]),
        "ffb_radiance_absorption": (i32, [vp, vp, vp, vp, vp, vp, i32, u64, u32, i32, vp]),
        "ffb_obj_parse": (i32, [vp, C.c_char_p, C.c_ulonglong, C.c_char_p, C.POINTER(ObjInfo)]),
        "ffb_obj_load": (i32, [vp, C.c_char_p, C.POINTER(ObjInfo)]),
        "ffb_obj_result": (i32, [vp, vp, vp, vp]),
        "ffb_obj_scene_set": (i32, [vp]),
        "ffb_emit_parallel": (i32, [vp, C.POINTER(DiscSource), i64, u64, u32, vp]),
        "ffb_parallel_rays": (i32, [vp, C.POINTER(DiscSource), i64, u64, u32, vp]),
        "ffb_bounding_sphere": (i32, [vp, i32, vp, C.POINTER(C.c_float)]),
        "ffb_radiance_step": (i32, [vp, vp, i32, vp, i32, vp, i32, vp, i32, u64, u32, i32, vp, vp]),
        "ffb_distant_source_step": (i32, [vp, vp, i32, vp, i32, vp, i32, i32, C.c_float, vp, u64, u32, vp]),
        "ffb_cast_bruteforce_static": (i32, [vp, i32, vp, i64, vp, vp, vp]),
        "ffb_form_factors": (i32, [vp, vp, vp, u64, u32, i32, vp, i32, vp, vp]),
        "ffb_form_factor_counts_rows": (i32, [vp, vp, vp, u64, u32, i32, vp, i32, i32, i32, vp]),
        "ffb_autotune_grid": (i32, [vp, vp, vp, u64, vp, i32, i32, C.POINTER(GridParams), C.POINTER(C.c_float)]),
        "ffb_trace_shape_count": (i32, []),
        "ffb_trace_shape_get": (i32, [i32, C.POINTER(TraceShape)]),
        "ffb_ctx_set_trace_shape": (i32, [vp, i32]),
        "ffb_ctx_trace_shape": (i32, [vp]),
        "ffb_autotune": (i32, [vp, vp, vp, u64, vp, i32, i32, i32, vp, C.POINTER(TuneResult)]),
        "ffb_batch_autotune": (i32, [vp, vp, vp, vp]),
        "ffb_batch_set": (i32, [vp, i32, vp, vp, vp]),
        "ffb_batch_grid_info": (i32, [vp, i32, C.POINTER(GridInfo)]),
        "ffb_batch_prepare": (i32, [vp, vp, vp, vp, i32]),
        "ffb_batch_launch": (i32, [vp, vp, vp, C.c_ulonglong, i32]),
        "ffb_server_create": (i32, [i32, C.c_ulonglong, i32, C.POINTER(vp)]),
        "ffb_server_destroy": (None, [vp]),
        "ffb_server_submit": (i32, [vp, vp, i32, i32, u64, i32, C.c_float, C.POINTER(C.c_longlong)]),
        "ffb_server_wait": (i32, [vp, C.c_longlong, C.c_double, C.POINTER(RequestInfo)]),
        "ffb_server_result": (i32, [vp, C.c_longlong, vp]),
        "ffb_server_release": (i32, [vp, C.c_longlong]),
        "ffb_server_stats": (i32, [vp, C.POINTER(ServerInfo)]),
        "ffb_server_set_slicing": (i32, [vp, C.c_longlong, i32]),
        "ffb_server_set_admission": (i32, [vp, i32, C.c_double]),
        "ffb_server_wait_any": (i32, [vp, vp, i32, C.c_double, C.POINTER(C.c_longlong), C.POINTER(RequestInfo)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    """Address of a numpy array or a tensor (data_ptr), or None."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    raise TypeError("unsupported buffer type %r" % type(a))


def _check(code):
    if code < 0:
        raise FFBError(code, load().ffb_last_error().decode(errors="replace"))
    return code


def trace_shapes():
    """The fused kernel's launch shapes (the autotuner's kernel choices)."""
    lib = load()
    out = []
    for v in range(lib.ffb_trace_shape_count()):
        t = TraceShape()
        _check(lib.ffb_trace_shape_get(v, C.byref(t)))
        out.append(dict(adv_per_iter=t.adv_per_iter, test_per_iter=t.test_per_iter, refill_min=t.refill_min,
                        blocks_per_sm=t.blocks_per_sm, coherent=bool(t.coherent), lanes=t.lanes))
    return out


def _tune_dict(r):
    return dict(dims=(r.grid.nx, r.grid.ny, r.grid.nz), cells_per_face=r.grid.cells_per_face,
                skip_empty=bool(r.grid.skip_empty), shape=r.shape, sample_ms=r.sample_ms,
                from_cache=bool(r.from_cache), timed=r.timed, sample_rays=r.sample_rays)


def cast_bruteforce_static(faces, rays, hit, points=None, stream=None):
    """ffb_cast_bruteforce_static on device tensors (no context, no allocation).
    faces: (n, 9) float32, rays: (m, 6) float32, hit: (m,) int32, points: (m, 3)
    float32 or None -- all CUDA tensors.  Enqueued on `stream` (an int
    cudaStream_t or None for the default stream)."""
    lib = load()
    _check(lib.ffb_cast_bruteforce_static(_ptr(faces), int(faces.shape[0]), _ptr(rays), int(rays.shape[0]),
                                          _ptr(hit), _ptr(points), stream or None))


class Context:
    """One device, one stream, a resident scene and grid (see include/ffb.h)."""

    def __init__(self, device=0):
        lib = load()
        h = C.c_void_p()
        _check(lib.ffb_ctx_create(int(device), C.byref(h)))
        self._h = h
        self._lib = lib
        self.n_faces = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ffb_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr):
        """Use a cudaStream_t (an int address); 0/None restores the context's own stream."""
        _check(self._lib.ffb_ctx_set_stream(self._h, stream_ptr or None))

    def synchronize(self):
        """Waits for the context stream (batched launches only enqueue)."""
        _check(self._lib.ffb_ctx_synchronize(self._h))

    def stream_ptr(self):
        return int(self._lib.ffb_ctx_stream(self._h) or 0)

    def set_budget(self, nbytes):
        _check(self._lib.ffb_ctx_set_budget(self._h, int(nbytes)))

    def set_stats(self, on):
        """Counters in the fused kernel on or off (on by default)."""
        _check(self._lib.ffb_ctx_set_stats(self._h, 1 if on else 0))

    def set_host_threads(self, n):
        """Host threads that expand packed host outputs of the count matrix
        (-1: default, 0: dense copies only)."""
        _check(self._lib.ffb_ctx_set_host_threads(self._h, int(n)))

    def host_threads(self):
        return _check(self._lib.ffb_ctx_host_threads(self._h))

    def device_bytes(self):
        return int(self._lib.ffb_ctx_bytes(self._h))

    def scene_set(self, faces):
        n = int(faces.shape[0]) if faces is not None else 0
        if isinstance(faces, np.ndarray):
            faces = np.ascontiguousarray(faces, np.float32).reshape(-1, 9)
            n = len(faces)
        _check(self._lib.ffb_scene_set(self._h, _ptr(faces) if n else None, n))
        self.n_faces = n

    def grid_build(self, dims=None, cells_per_face=None, skip_empty=True):
        """Builds the grid: explicit dims, else about cells_per_face cells per
        face (None: the library default, 32)."""
        p = GridParams(0, 0, 0, float(cells_per_face or 0.0), int(bool(skip_empty)))
        if dims is not None:
            p.nx, p.ny, p.nz = [int(d) for d in dims]
        _check(self._lib.ffb_grid_build(self._h, C.byref(p)))

    def autotune_grid(self, front, rear, seed=1, candidates=None, sample_every=8):
        """Times grid candidates on a sample of the ray budget and keeps the
        fastest built.  candidates: list of dicts with dims / cells_per_face /
        skip_empty; default: cubic 32..128 and 8..64 cells per face."""
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        if candidates is None:
            candidates = [dict(dims=(d, d, d)) for d in (32, 48, 64, 96, 128)] + \
                         [dict(cells_per_face=c) for c in (8, 16, 32, 64)]
        arr = (GridParams * len(candidates))()
        for i, cand in enumerate(candidates):
            arr[i] = GridParams(0, 0, 0, float(cand.get("cells_per_face", 32.0)), int(cand.get("skip_empty", True)))
            if cand.get("dims"):
                arr[i].nx, arr[i].ny, arr[i].nz = cand["dims"]
        best = GridParams()
        ms = C.c_float()
        _check(self._lib.ffb_autotune_grid(self._h, _ptr(front), _ptr(rear), int(seed), C.cast(arr, C.c_void_p),
                                           len(candidates), int(sample_every), C.byref(best), C.byref(ms)))
        return dict(dims=(best.nx, best.ny, best.nz), cells_per_face=best.cells_per_face,
                    skip_empty=bool(best.skip_empty), sample_ms=ms.value)

    def autotune(self, front, rear, seed=1, candidates=None, sample_every=0, force=False, scratch=None):
        """ffb_autotune: chooses the grid (candidates: dicts with dims /
        cells_per_face / skip_empty, None for the library's set) and the
        kernel's launch shape on a sample of the ray budget; builds the grid
        and sets the shape.  Cached per process by scene and budget class."""
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        arr = None
        if candidates is not None:
            arr = (GridParams * len(candidates))()
            for i, cand in enumerate(candidates):
                arr[i] = GridParams(0, 0, 0, float(cand.get("cells_per_face", 32.0)),
                                    int(cand.get("skip_empty", True)))
                if cand.get("dims"):
                    arr[i].nx, arr[i].ny, arr[i].nz = cand["dims"]
        res = TuneResult()
        _check(self._lib.ffb_autotune(self._h, _ptr(front), _ptr(rear), int(seed),
                                      C.cast(arr, C.c_void_p) if arr is not None else None,
                                      len(candidates) if candidates is not None else 0, int(sample_every),
                                      1 if force else 0, _ptr(scratch), C.byref(res)))
        return _tune_dict(res)

    def set_trace_shape(self, shape):
        _check(self._lib.ffb_ctx_set_trace_shape(self._h, int(shape)))

    def trace_shape(self):
        return _check(self._lib.ffb_ctx_trace_shape(self._h))

    def grid_info(self):
        info = GridInfo()
        _check(self._lib.ffb_grid_info_get(self._h, C.byref(info)))
        return info

    def grid_export(self):
        """The current grid: cell records (nz, ny, nx, 2) uint32 and the
        references (face index per reference, each cell's in ascending
        order), as ffb_grid_export lays them out."""
        info = self.grid_info()
        rec = np.empty((info.nz, info.ny, info.nx, 2), np.uint32)
        refs = np.empty(max(int(info.n_refs), 1), np.int32)
        _check(self._lib.ffb_grid_export(self._h, _ptr(rec), _ptr(refs)))
        return rec, refs[:int(info.n_refs)]

    def cast(self, rays, hit=None, points=None, want_points=True, brute=False):
        """rays: (n, 6) float32 host array or device tensor.  Returns (hit, points)."""
        n = int(rays.shape[0]) if not isinstance(rays, np.ndarray) else len(rays.reshape(-1, 6))
        if isinstance(rays, np.ndarray):
            rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        if hit is None:
            hit = np.empty(n, np.int32)
        if points is None and want_points:
            points = np.empty((n, 3), np.float32)
        fn = self._lib.ffb_cast_bruteforce if brute else self._lib.ffb_cast
        _check(fn(self._h, _ptr(rays), n, _ptr(hit), _ptr(points)))
        return hit, points

    def emit(self, front, rear, seed, epoch=0, flags=0, out=None):
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        total = int(front.sum(dtype=np.int64) + rear.sum(dtype=np.int64))
        if out is None:
            out = np.empty((total, 6), np.float32)
        _check(self._lib.ffb_emit(self._h, _ptr(front), _ptr(rear), int(seed), int(epoch), int(flags), _ptr(out)))
        return out

    def form_factor_counts(self, front, rear, seed, epoch=0, flags=0, face_to_row=None, n_rows=None, out=None):
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        if face_to_row is not None:
            face_to_row = np.ascontiguousarray(face_to_row, np.int32)
        if n_rows is None:
            n_rows = self.n_faces if face_to_row is None else int(face_to_row.max()) + 1
        if out is None:
            out = np.empty((n_rows, n_rows), np.uint32)
        _check(self._lib.ffb_form_factor_counts(self._h, _ptr(front), _ptr(rear), int(seed), int(epoch), int(flags),
                                                _ptr(face_to_row), int(n_rows), _ptr(out)))
        return out

    def form_factor_counts_rows(self, front, rear, seed, row_begin, row_end, epoch=0, flags=0, face_to_row=None,
                                n_rows=None, out=None):
        """Rows [row_begin, row_end) of the count matrix (one shard)."""
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        if face_to_row is not None:
            face_to_row = np.ascontiguousarray(face_to_row, np.int32)
        if n_rows is None:
            n_rows = self.n_faces if face_to_row is None else int(face_to_row.max()) + 1
        if out is None:
            out = np.empty((row_end - row_begin, n_rows), np.uint32)
        _check(self._lib.ffb_form_factor_counts_rows(self._h, _ptr(front), _ptr(rear), int(seed), int(epoch),
                                                     int(flags), _ptr(face_to_row), int(n_rows), int(row_begin),
                                                     int(row_end), _ptr(out)))
        return out

    def normalise(self, counts, outgoing, out=None):
        outgoing = np.ascontiguousarray(outgoing, np.int32)
        n = len(outgoing)
        if isinstance(counts, np.ndarray):
            counts = np.ascontiguousarray(counts, np.uint32)
        if out is None:
            out = np.empty((n, n), np.float32)
        _check(self._lib.ffb_normalise(self._h, _ptr(counts), _ptr(outgoing), n, _ptr(out)))
        return out

    @staticmethod
    def _csv_args(ff, counts, outgoing):
        if ff is not None:
            if isinstance(ff, np.ndarray):
                ff = np.ascontiguousarray(ff, np.float32)
            n = int(ff.shape[0]) if ff.ndim == 2 else int(round(ff.shape[0] ** 0.5))
            return ff, None, None, n
        outgoing = np.ascontiguousarray(outgoing, np.int32) if isinstance(outgoing, (np.ndarray, list)) else outgoing
        if isinstance(counts, np.ndarray):
            counts = np.ascontiguousarray(counts, np.uint32)
        return None, counts, outgoing, int(len(outgoing))

    def csv_length(self, ff=None, counts=None, outgoing=None):
        """Length in bytes of the CSV text of the matrix (ff, or counts
        normalised by outgoing)."""
        ff, counts, outgoing, n = self._csv_args(ff, counts, outgoing)
        ln = C.c_ulonglong()
        if ff is not None:
            _check(self._lib.ffb_csv_format(self._h, _ptr(ff), n, None, 0, C.byref(ln)))
        else:
            _check(self._lib.ffb_csv_format_counts(self._h, _ptr(counts), _ptr(outgoing), n, None, 0, C.byref(ln)))
        return ln.value

    def csv_format(self, ff=None, counts=None, outgoing=None, out=None):
        """CSV text of the matrix as the reference's csv_export writes it.
        Returns bytes, or, with `out` (a host or device byte buffer), the
        number of bytes written into it."""
        ff, counts, outgoing, n = self._csv_args(ff, counts, outgoing)
        ret_bytes = out is None
        if out is None:
            out = np.empty(max(self.csv_length(ff=ff, counts=counts, outgoing=outgoing), 1), np.uint8)
        cap = out.nbytes if isinstance(out, np.ndarray) else out.numel() * out.element_size()
        ln = C.c_ulonglong()
        if ff is not None:
            _check(self._lib.ffb_csv_format(self._h, _ptr(ff), n, _ptr(out), cap, C.byref(ln)))
        else:
            _check(self._lib.ffb_csv_format_counts(self._h, _ptr(counts), _ptr(outgoing), n, _ptr(out), cap,
                                                   C.byref(ln)))
        return out[:ln.value].tobytes() if ret_bytes else ln.value

    def csv_export(self, filename, ff=None, counts=None, outgoing=None):
        """Writes the CSV file (ffb_csv_export / ffb_csv_export_counts)."""
        ff, counts, outgoing, n = self._csv_args(ff, counts, outgoing)
        name = os.fsencode(filename)
        if ff is not None:
            _check(self._lib.ffb_csv_export(self._h, name, _ptr(ff), n))
        else:
            _check(self._lib.ffb_csv_export_counts(self._h, name, _ptr(counts), _ptr(outgoing), n))

    def _obj_info(self, rc, info):
        d = {k: getattr(info, k) for k, _ in ObjInfo._fields_}
        if rc < 0 and rc not in (FFB_ERR_FORMAT, FFB_ERR_FILE):
            _check(rc)
        return d

    def obj_parse(self, text, filename=None):
        """obj_import::scene on OBJ text (bytes) with the geometry parsed on
        the GPU; `filename` locates mtllib files.  Returns the info dict
        (status: the reference's return code, error_line)."""
        info = ObjInfo()
        rc = self._lib.ffb_obj_parse(self._h, text, len(text), os.fsencode(filename) if filename else None,
                                     C.byref(info))
        return self._obj_info(rc, info)

    def obj_load(self, filename):
        info = ObjInfo()
        rc = self._lib.ffb_obj_load(self._h, os.fsencode(filename), C.byref(info))
        return self._obj_info(rc, info)

    def obj_result(self, info):
        """(faces (n, 9) float32, meshes (m, 3) int32, materials) of the last parse."""
        faces = np.empty((info["n_faces"], 9), np.float32)
        meshes = np.empty((info["n_meshes"], 3), np.int32)
        materials = np.zeros(info["n_materials"], MATERIAL_DTYPE)
        _check(self._lib.ffb_obj_result(self._h, _ptr(faces), _ptr(meshes), materials.ctypes.data))
        return faces, meshes, materials

    def obj_scene_set(self, n_faces):
        """The parsed faces become this context's scene (device to device)."""
        _check(self._lib.ffb_obj_scene_set(self._h))
        self.n_faces = int(n_faces)

    def radiance_absorption(self, front, rear, power_front, power_rear, face_to_mesh, n_meshes, seed, epoch=0,
                            flags=0):
        """ffb_radiance_absorption: absorbed power per mesh (float64)."""
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        pf = np.ascontiguousarray(power_front, np.float32)
        pr = np.ascontiguousarray(power_rear, np.float32)
        f2m = np.ascontiguousarray(face_to_mesh, np.int32)
        out = np.zeros(int(n_meshes), np.float64)
        _check(self._lib.ffb_radiance_absorption(self._h, _ptr(front), _ptr(rear), _ptr(pf), _ptr(pr), _ptr(f2m),
                                                 int(n_meshes), int(seed), int(epoch), int(flags), _ptr(out)))
        return out

    def emit_parallel(self, source, n_rays, seed, epoch=0, out=None):
        """Rays of a disc source (ffb_emit_parallel), (n_rays, 6) float32."""
        if out is None:
            out = np.empty((int(n_rays), 6), np.float32)
        _check(self._lib.ffb_emit_parallel(self._h, C.byref(source), int(n_rays), int(seed), int(epoch), _ptr(out)))
        return out

    def parallel_rays(self, source, n_rays, seed, epoch=0, out=None):
        """Hits of a disc source per (face, side) (ffb_parallel_rays), (n_faces, 2) uint32."""
        if out is None:
            out = np.empty((self.n_faces, 2), np.uint32)
        _check(self._lib.ffb_parallel_rays(self._h, C.byref(source), int(n_rays), int(seed), int(epoch), _ptr(out)))
        return out

    def radiance_step(self, faces, meshes, materials, temperatures, n_rays, seed, epoch=0, flags=0,
                      emission=None, absorption=None):
        """One radiance-equation calculate(): (emission, absorption) per mesh,
        added to the given float32 arrays (zeros by default).  meshes: (first,
        count, material) triples; materials: (front emissivity, rear
        emissivity, front absorbance, rear absorbance)."""
        faces = np.ascontiguousarray(faces, np.float32)
        t = np.ascontiguousarray(temperatures, np.float32)
        n_m = len(meshes)
        emission = np.zeros(n_m, np.float32) if emission is None else emission
        absorption = np.zeros(n_m, np.float32) if absorption is None else absorption
        m3, opt = _meshes(meshes), _optics(materials)
        _check(self._lib.ffb_radiance_step(self._h, _ptr(faces), len(faces), _ptr(m3), n_m,
                                           _ptr(opt), len(opt), _ptr(t), int(n_rays), int(seed),
                                           int(epoch), int(flags), _ptr(emission), _ptr(absorption)))
        return emission, absorption

    def distant_source_step(self, faces, meshes, materials, n_rays, power, direction, seed, epoch=0,
                            absorption=None):
        """One distant-source calculate(): absorbed power per mesh added to
        `absorption` (zeros by default)."""
        faces = np.ascontiguousarray(faces, np.float32)
        d = np.ascontiguousarray(direction, np.float32)
        n_m = len(meshes)
        absorption = np.zeros(n_m, np.float32) if absorption is None else absorption
        m3, opt = _meshes(meshes), _optics(materials)
        _check(self._lib.ffb_distant_source_step(self._h, _ptr(faces), len(faces), _ptr(m3), n_m,
                                                 _ptr(opt), len(opt), int(n_rays), float(power),
                                                 _ptr(d), int(seed), int(epoch), _ptr(absorption)))
        return absorption

    def form_factors(self, front, rear, seed, epoch=0, flags=0, face_to_row=None, n_rows=None, outgoing=None,
                     out=None):
        """Counts and row normalisation in one call (ffb_form_factors)."""
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        if face_to_row is not None:
            face_to_row = np.ascontiguousarray(face_to_row, np.int32)
        if n_rows is None:
            n_rows = self.n_faces if face_to_row is None else int(face_to_row.max()) + 1
        if outgoing is None:
            rows = np.arange(self.n_faces) if face_to_row is None else face_to_row
            outgoing = np.zeros(n_rows, np.int64)
            np.add.at(outgoing, rows, front.astype(np.int64) + rear)
        outgoing = np.ascontiguousarray(outgoing, np.int32)
        if out is None:
            out = np.empty((n_rows, n_rows), np.float32)
        _check(self._lib.ffb_form_factors(self._h, _ptr(front), _ptr(rear), int(seed), int(epoch), int(flags),
                                          _ptr(face_to_row), int(n_rows), _ptr(outgoing), _ptr(out)))
        return out

    # ---- batched scenes -------------------------------------------------
    def batch_set(self, scenes_faces, cells_per_face=32.0, skip_empty=True, dims=None):
        """Uploads a list of (n_i, 9) float32 scenes and builds their grids."""
        sizes = [len(f) for f in scenes_faces]
        offsets = np.zeros(len(sizes) + 1, np.int64)
        offsets[1:] = np.cumsum(sizes)
        faces = np.ascontiguousarray(np.concatenate(scenes_faces), np.float32)
        params = (GridParams * len(sizes))()
        for i in range(len(sizes)):
            params[i] = GridParams(0, 0, 0, float(cells_per_face), int(bool(skip_empty)))
            if dims is not None:
                params[i].nx, params[i].ny, params[i].nz = dims[i]
        _check(self._lib.ffb_batch_set(self._h, len(sizes), _ptr(offsets), _ptr(faces), C.cast(params, C.c_void_p)))
        self.batch_sizes = sizes
        self.batch_offsets = offsets
        return offsets

    def batch_grid_info(self, scene):
        info = GridInfo()
        _check(self._lib.ffb_batch_grid_info(self._h, int(scene), C.byref(info)))
        return info

    def batch_prepare(self, front, rear, seeds=None, flags=0):
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        if seeds is not None:
            seeds = np.ascontiguousarray(seeds, np.uint64)
        _check(self._lib.ffb_batch_prepare(self._h, _ptr(front), _ptr(rear), _ptr(seeds), int(flags)))

    def batch_autotune(self, front, rear):
        """ffb_batch_autotune: each scene's grid and launch shape from the
        tuning cache, tuning the scenes it has no choice for."""
        front = np.ascontiguousarray(front, np.int32)
        rear = np.ascontiguousarray(rear, np.int32)
        shapes = np.zeros(len(self.batch_sizes), np.int32)
        _check(self._lib.ffb_batch_autotune(self._h, _ptr(front), _ptr(rear), _ptr(shapes)))
        return shapes

    def batch_counts_layout(self):
        """(offsets, words): where each scene's N x N matrix starts in one buffer."""
        sq = np.array([n * n for n in self.batch_sizes], np.uint64)
        offs = np.zeros(len(sq), np.uint64)
        offs[1:] = np.cumsum(sq)[:-1]
        return np.ascontiguousarray(offs), int(sq.sum())

    def batch_launch(self, counts, counts_offsets, advance_epoch=True):
        counts_offsets = np.ascontiguousarray(counts_offsets, np.uint64)
        words = int(counts.numel()) if hasattr(counts, "numel") else int(counts.size)
        _check(self._lib.ffb_batch_launch(self._h, _ptr(counts), _ptr(counts_offsets), words, int(bool(advance_epoch))))

    def stats(self):
        s = Stats()
        _check(self._lib.ffb_stats_get(self._h, C.byref(s)))
        return s


class Server:
    """Request loop over the C ABI's ffb_server_* (admission by memory budget,
    concurrent slots, resident results)."""

    def __init__(self, device=0, budget_bytes=0, slots=4):
        lib = load()
        h = C.c_void_p()
        _check(lib.ffb_server_create(int(device), int(budget_bytes), int(slots), C.byref(h)))
        self._h, self._lib = h, lib

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ffb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, faces, rays_per_face, seed, flags=0, cells_per_face=32.0):
        faces = np.ascontiguousarray(faces, np.float32).reshape(-1, 9)
        rid = C.c_longlong()
        _check(self._lib.ffb_server_submit(self._h, _ptr(faces), len(faces), int(rays_per_face), int(seed),
                                           int(flags), float(cells_per_face), C.byref(rid)))
        return rid.value

    def wait(self, rid, timeout_s=-1.0):
        info = RequestInfo()
        _check(self._lib.ffb_server_wait(self._h, int(rid), float(timeout_s), C.byref(info)))
        return info

    def wait_any(self, rids, timeout_s=-1.0):
        """(request id, RequestInfo) of the first of `rids` to finish."""
        arr = np.ascontiguousarray(rids, np.int64)
        done = C.c_longlong()
        info = RequestInfo()
        _check(self._lib.ffb_server_wait_any(self._h, _ptr(arr), len(arr), float(timeout_s), C.byref(done),
                                             C.byref(info)))
        return done.value, info

    def result(self, rid, n_faces, out=None):
        if out is None:
            out = np.empty((n_faces, n_faces), np.uint32)
        _check(self._lib.ffb_server_result(self._h, int(rid), _ptr(out)))
        return out

    def set_slicing(self, slice_rays, window=2):
        """Rays per trace slice and slices in flight (ffb_server_set_slicing)."""
        _check(self._lib.ffb_server_set_slicing(self._h, int(slice_rays), int(window)))

    def set_admission(self, shortest_first=False, max_wait_s=0.0):
        """Admission order (ffb_server_set_admission): arrival order, or the
        least work first with the oldest request first once it has waited
        max_wait_s."""
        _check(self._lib.ffb_server_set_admission(self._h, 1 if shortest_first else 0, float(max_wait_s)))

    def release(self, rid):
        _check(self._lib.ffb_server_release(self._h, int(rid)))

    def stats(self):
        info = ServerInfo()
        _check(self._lib.ffb_server_stats(self._h, C.byref(info)))
        return info
