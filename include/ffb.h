/*
 * ffb.h -- C ABI of libffb200.so, the B200 (sm_100a) form-factor path.
 *
 * Plain pointers and sizes only.  Every function returns FFB_OK (0) or a
 * negative FFB_ERR_* code and never exits or resets the device; the message
 * of the last failure on the calling thread is in ffb_last_error().
 *
 * Pointer arguments marked "host or device" are classified with
 * cudaPointerGetAttributes: device (or managed) memory is used in place;
 * host memory is staged through the context's buffers.  A call whose outputs
 * are all in device memory only enqueues work on the context stream and
 * returns (CUDA-graph capturable); a call with a host output synchronises the
 * stream before it returns.
 *
 * Geometry layouts are the reference's (math/types.h:36-76):
 *   face  = 9 floats, three vertices            (math::triangle_t, 36 B)
 *   ray   = 6 floats, origin then END POINT     (math::ray_t, 24 B; the
 *           direction is end - origin, ray_caster/naive_cpu.cpp, math/triangle.cpp:41)
 *
 * The C++ system_t types of ffb_systems.h wrap these calls behind the
 * reference's own ray_caster / emission / form_factors interfaces.
 */
#ifndef FFB_H
#define FFB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFB_OK 0
#define FFB_ERR_ARG (-301)       /* invalid argument */
#define FFB_ERR_CUDA (-302)      /* CUDA runtime failure (see ffb_last_error) */
#define FFB_ERR_NO_SCENE (-303)  /* no scene, or a scene with no faces */
#define FFB_ERR_NO_GRID (-304)   /* cast before ffb_grid_build */
#define FFB_ERR_NO_MEMORY (-305) /* device allocation failed or over the context budget */
#define FFB_ERR_TOO_LARGE (-306) /* a size beyond a documented limit */
#define FFB_ERR_NO_DEVICE (-307) /* no CUDA device / not an sm_100 device */
#define FFB_ERR_TIMEOUT (-308)   /* a wait ended before the work finished */
#define FFB_ERR_FILE (-309)      /* a file could not be opened or written */
#define FFB_ERR_FORMAT (-310)    /* malformed input file (see the call's status) */

/* Emission flag: rotate +z towards the raw cross-product normal, as the
 * reference's emission/malley_cpu.cpp:125-129 does.  Without it the normal is
 * normalised first (cosine-weighted directions for any triangle size). */
#define FFB_EMIT_REF_NORMAL 1

typedef struct ffb_ctx ffb_ctx;

typedef struct {
  int nx, ny, nz;          /* cells per axis, each <= 256; 0 = choose from cells_per_face */
  float cells_per_face;    /* automatic sizing target (cells ~ this * faces); <= 0 means 32 */
  int skip_empty;          /* 1 = jump through empty space (distance map), 0 = plain DDA */
} ffb_grid_params;

typedef struct {
  float lo[3], hi[3];      /* grid box */
  float cell[3];           /* cell size */
  int nx, ny, nz;
  int n_live_faces;        /* faces that can be hit (finite, non-degenerate) */
  long long n_refs;        /* triangle references in all cells */
  float margin;            /* binning margin, world units */
  int skip_empty;
} ffb_grid_info;

typedef struct {
  unsigned long long tests; /* ray/triangle tests executed */
  unsigned long long cells; /* grid cells visited */
  unsigned long long rays;  /* rays traced */
  unsigned long long hits;  /* rays that hit a face */
  float kernel_ms;          /* device time of the trace kernel (CUDA events) */
  unsigned long long jumps; /* empty-space jumps among the cells visited */
  unsigned long long d2h_bytes; /* device-to-host bytes of the last counts call with a host output (0 for a
                                   device output) */
} ffb_stats;

/* Context: one device, one stream, resident scene and grid.
 * Replaces the state of ray_caster::system_create (ray_caster/system.cpp:65-90).
 * Device buffers come from the device's default stream-ordered memory pool,
 * which ffb_ctx_create sets to keep freed blocks for reuse (this process
 * only); ffb_ctx_destroy trims the blocks no one uses back to the driver. */
int ffb_ctx_create(int device, ffb_ctx** out);
void ffb_ctx_destroy(ffb_ctx* ctx);
/* Use `stream` (a cudaStream_t) instead of the context's own; NULL restores it. */
int ffb_ctx_set_stream(ffb_ctx* ctx, void* stream);
void* ffb_ctx_stream(ffb_ctx* ctx);
/* Waits for all work enqueued on the context's stream (the batched launch
 * and calls with device outputs return without waiting).  No reference
 * counterpart: the reference's calls are synchronous. */
int ffb_ctx_synchronize(ffb_ctx* ctx);
/* Device-memory budget of the context in bytes (0 = unlimited). */
int ffb_ctx_set_budget(ffb_ctx* ctx, unsigned long long bytes);
unsigned long long ffb_ctx_bytes(ffb_ctx* ctx);
/* Test / cell / ray / hit counters of the fused kernel (on by default).  Off,
 * the kernel variant without counters runs and ffb_stats_get reports zero
 * counts (kernel_ms stays).  No reference counterpart: the reference keeps no
 * such counters. */
int ffb_ctx_set_stats(ffb_ctx* ctx, int on);
/* Host threads of the context (-1: the default, min(12, hardware threads);
 * 0 to 256).  A count matrix written to a host buffer in row blocks (64 MB
 * or more, ffb_form_factor_counts(_rows)) crosses PCIe as the (column, count)
 * pairs of each block's nonzero entries, packed on the device, and these
 * threads expand them into the caller's rows with streaming stores while the
 * next block traces; a block denser than a quarter of its entries is copied
 * dense.  0: every block is copied dense.  The result is the same either
 * way.  No reference counterpart (the reference's matrix is on the host). */
int ffb_ctx_set_host_threads(ffb_ctx* ctx, int n);
int ffb_ctx_host_threads(ffb_ctx* ctx);
const char* ffb_last_error(void);

/* Scene upload and per-face precompute (host or device faces9).
 * ray_caster::system_set_scene, ray_caster/system.h:95.  n_faces == 0 is
 * accepted (the reference accepts an empty scene); ffb_grid_build then
 * fails with FFB_ERR_NO_SCENE as ray_caster prepare does (zgrid_cpu.cpp:59). */
int ffb_scene_set(ffb_ctx* ctx, const float* faces9, int n_faces);

/* Device grid build (counting sort of triangle references into cells).
 * ray_caster::system_prepare, ray_caster/system.h:98; zgrid_cpu.cpp:57-68.
 * params may be NULL (automatic). */
int ffb_grid_build(ffb_ctx* ctx, const ffb_grid_params* params);
int ffb_grid_info_get(ffb_ctx* ctx, ffb_grid_info* out);

/* Copies the grid of the current scene to host or device buffers (either
 * may be NULL):
 *  cell_rec: 2 uint32 per cell, x fastest.  An occupied cell holds {first
 *    reference, end}.  An empty one holds {octant distances 0-3,
 *    0x80000000 | octant distances 4-7}, one byte per octant (octant o in
 *    byte o & 3).  Octant o points down axis a when bit a of o is set; its
 *    distance is the side of the largest cube of empty cells that extends
 *    from the cell in those directions (capped at 127; 1 for every octant
 *    when the grid skips no empty space).
 *  ref_tri: n_refs face indices, each cell's references in ascending order.
 * No reference counterpart (zgrid_cpu keeps its 2-D cells internal,
 * math/grid.h:36-49): an inspection hook for tests and tools. */
int ffb_grid_export(ffb_ctx* ctx, uint32_t* cell_rec, int32_t* ref_tri);

/* Nearest hit per ray through the grid.  rays6: host or device; hit_face:
 * host or device, face index or -1; hit_point: host, device or NULL, the
 * reference's hit point for hits and NaN for misses.  Equal bit for bit to
 * ray_caster/naive_cpu.cpp:65-97.  ray_caster::system_cast, ray_caster/system.h:102. */
int ffb_cast(ffb_ctx* ctx, const float* rays6, long long n_rays, int32_t* hit_face, float* hit_point);

/* Same result by brute force (every ray against every face), the naive
 * definition without the grid; needs only ffb_scene_set. */
int ffb_cast_bruteforce(ffb_ctx* ctx, const float* rays6, long long n_rays, int32_t* hit_face, float* hit_point);

/* Malley emission rays, packed face by face, front then rear
 * (emission/malley_cpu.cpp:142-189), ray j of face f drawn from
 * Philox4x32-10 keyed by (seed, epoch, f, j).  front/rear: host int32[n_faces]
 * ray counts; rays6: host or device, 6 * sum(front + rear) floats. */
int ffb_emit(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch, int flags,
             float* rays6);

/* Fused emission + grid trace + count: counts[row(f) * n_rows + row(h)] +=
 * number of rays of face f whose nearest hit is face h, where row() is
 * face_to_row (host int32[n_faces], values in [0, n_rows)) or the identity
 * when face_to_row is NULL (then n_rows must equal n_faces).  counts: host or
 * device uint32[n_rows * n_rows], overwritten.  The per-face (row) form of
 * cpuFactorsCalculator/cpu_system.cpp:162-190. */
int ffb_form_factor_counts(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch,
                           int flags, const int32_t* face_to_row, int n_rows, uint32_t* counts);

/* The rows [row_begin, row_end) of the same matrix: only the faces of those
 * rows emit, and counts ((row_end - row_begin) x n_rows, host or device)
 * receives row r at (r - row_begin) * n_rows.  Row blocks are independent,
 * which is how the matrix is sharded across GPUs (no collective while
 * tracing; the blocks are gathered afterwards if a rank needs them all). */
int ffb_form_factor_counts_rows(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, uint64_t seed,
                                uint32_t epoch, int flags, const int32_t* face_to_row, int n_rows, int row_begin,
                                int row_end, uint32_t* counts);

/* ff[m * n_rows + j] = (float)counts[m * n_rows + j] * (1.f / (float)outgoing[m]),
 * the row normalisation of cpuFactorsCalculator/cpu_system.cpp:193-195.
 * counts and ff: host or device; outgoing: host int32[n_rows]. */
int ffb_normalise(ffb_ctx* ctx, const uint32_t* counts, const int32_t* outgoing, int n_rows, float* ff);

/* Form factors in one call: the counts of ffb_form_factor_counts in device
 * scratch, then ff[m * n_rows + j] = (float)count * (1.f / (float)outgoing[m])
 * as cpuFactorsCalculator/cpu_system.cpp:162-196 computes them.  outgoing:
 * host int32[n_rows], the rays leaving each row (mesh); ff: host or device
 * float[n_rows * n_rows].  form_factors::system_calculate, form_factors/system.h:115. */
int ffb_form_factors(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch,
                     int flags, const int32_t* face_to_row, int n_rows, const int32_t* outgoing, float* ff);

/* Batched scenes: up to 4096 independent scenes, each with its own resident
 * grid and count matrix (the batched workload: many scenes of uneven size).  Scene s is faces [face_offsets[s], face_offsets[s+1]) of
 * faces9 (host or device); params: one ffb_grid_params per scene, or NULL
 * (automatic).  The batch is separate from the scene of the single-scene
 * calls above, which keep working. */
int ffb_batch_set(ffb_ctx* ctx, int n_scenes, const long long* face_offsets, const float* faces9,
                  const ffb_grid_params* params);
int ffb_batch_grid_info(ffb_ctx* ctx, int scene, ffb_grid_info* out);
/* Work list of the next batched launches: front/rear ray counts for every
 * face of every scene (host, concatenated like the faces), one Philox seed
 * per scene (host, or NULL for 1), emission flags.  Resets the device epoch
 * to 0 and synchronises. */
int ffb_batch_prepare(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, const uint64_t* seeds, int flags);
/* Traces every prepared scene: zeroes `counts` (device, counts_words
 * uint32) and adds scene s's per-face counts into the N_s x N_s matrix at
 * counts + counts_offsets[s] (host offsets).  One fused launch per scene,
 * largest first, dealt over four side streams forked from and joined back
 * to the context stream, so that one scene's launch tail overlaps the next
 * scenes.  With advance_epoch the device epoch is incremented first, so that
 * successive calls -- or the replays of a CUDA graph that captured this
 * call -- draw fresh rays.  Only enqueues work (capturable as one graph). */
int ffb_batch_launch(ffb_ctx* ctx, uint32_t* counts, const unsigned long long* counts_offsets,
                     unsigned long long counts_words, int advance_epoch);

/* Serving: form-factor solves submitted as requests of different sizes,
 * admitted in arrival order into `n_slots` slots while the device-memory
 * budget allows (0 = no budget); a finished result keeps its reservation
 * until released.  Each slot is a context (own stream, resident scene) whose
 * worker thread prepares its request -- scene upload, grid build, zeroed
 * count matrix, chunk table -- while other requests trace.  One scheduler
 * thread then traces the prepared requests in slices (64 Mi rays by default,
 * ffb_server_set_slicing), round-robin over them, two in flight on the requests' own
 * streams: a request admitted while others are on the GPU joins at the next
 * slice boundary, its kernels overlap theirs on the device, and a small
 * request finishes within its first turn instead of queueing behind a large
 * one (processor sharing).  A request is a scene (host faces9, copied at
 * submit), rays_per_face front-side rays per face, a Philox seed, emission
 * flags and a grid target cells_per_face (0: grid and launch shape chosen by
 * ffb_autotune, through its process-wide cache; the budget then reserves
 * room for its largest grid); its per-face N x N uint32 counts stay resident
 * on the device until
 * ffb_server_release.  The result of a request does not depend on the other
 * requests in flight or on the slicing: it equals ffb_form_factor_counts on
 * the same scene with epoch 0. */
#define FFB_REQ_QUEUED 0
#define FFB_REQ_RUNNING 1
#define FFB_REQ_DONE 2
#define FFB_REQ_FAILED 3

typedef struct ffb_server ffb_server;

typedef struct {
  int state;         /* FFB_REQ_* */
  int error;         /* FFB_ERR_* of a failed request */
  int n_faces;
  double queue_s;    /* submit -> admission */
  double latency_s;  /* submit -> result resident */
  double gpu_ms;     /* trace_end_ns - trace_start_ns, in ms */
  unsigned long long trace_start_ns; /* %globaltimer at the first block start of the request's first trace slice */
  unsigned long long trace_end_ns;   /* %globaltimer at the last warp end of its last trace slice */
  int slices;        /* trace launches the request took */
  int shape;         /* launch shape of its trace */
  float cells_per_face; /* grid target of its trace (the autotuner's choice when submitted with 0) */
} ffb_request_info;

typedef struct {
  int queued, running, peak_running;
  unsigned long long reserved_bytes, budget_bytes;
  int peak_tracing;  /* most requests in the trace rotation at once */
} ffb_server_info;

int ffb_server_create(int device, unsigned long long budget_bytes, int n_slots, ffb_server** out);
void ffb_server_destroy(ffb_server* server);
int ffb_server_submit(ffb_server* server, const float* faces9, int n_faces, int rays_per_face, uint64_t seed,
                      int flags, float cells_per_face, long long* request_id);
/* Waits for a request (timeout_s < 0: no limit); FFB_ERR_TIMEOUT if it is
 * still queued or running when the time is up. */
int ffb_server_wait(ffb_server* server, long long request_id, double timeout_s, ffb_request_info* info);
/* Waits until one of the n requests `ids` has finished (timeout_s < 0: no
 * limit) and reports it in *done_id and *info, as ffb_server_wait does.  A
 * client that consumes results in completion order -- and releases each --
 * keeps the budget free for the requests still queued: a finished result
 * keeps its reservation until released, so a client that holds finished
 * results while it waits for a request that has not been admitted can leave
 * that request no room. */
int ffb_server_wait_any(ffb_server* server, const long long* ids, int n, double timeout_s, long long* done_id,
                        ffb_request_info* info);
/* Copies a finished request's counts (host or device, N*N uint32). */
int ffb_server_result(ffb_server* server, long long request_id, uint32_t* counts);
/* Frees a finished request's resident matrix and its budget reservation. */
int ffb_server_release(ffb_server* server, long long request_id);
int ffb_server_stats(ffb_server* server, ffb_server_info* out);
/* Trace slicing of the server: at most slice_rays rays per slice (default
 * 64 Mi, rounded down to whole 256-ray chunks) and `window` slices in flight
 * (default 2, at most 8).  Applies to the slices launched after the call. */
int ffb_server_set_slicing(ffb_server* server, long long slice_rays, int window);
/* Admission order.  FFB_ADMIT_FIFO (default): arrival order, no overtaking.
 * FFB_ADMIT_SHORTEST: the queued request with the least work (faces x rays
 * per face) first, unless the oldest queued request has waited longer than
 * max_wait_s, which then goes first (starvation bounded by the age limit). */
#define FFB_ADMIT_FIFO 0
#define FFB_ADMIT_SHORTEST 1
int ffb_server_set_admission(ffb_server* server, int policy, double max_wait_s);

/* One step of the radiance equation (thermal_equation/radiance_cpu.cpp:96-190)
 * on the resident scene and grid: every face emits front[f] + rear[f] Malley
 * rays (seed, epoch, flags as ffb_form_factor_counts); a ray of face f that
 * hits face h adds power_front[f] (front rays) or power_rear[f] (rear rays)
 * to absorption[face_to_mesh[h]] (host arrays, n_faces and n_meshes long).
 * The sums are exact integer sums of the powers rounded to a fixed point of
 * 2^k units per watt, k the largest that keeps the total of every ray's power
 * below 2^62; absorption[] is set (not added to).  The caller computes the
 * ray counts and per-ray powers as the reference does (calculate_weights,
 * emitted_front/rear, front_emission / face_rays_front). */
int ffb_radiance_absorption(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, const float* power_front,
                            const float* power_rear, const int32_t* face_to_mesh, int n_meshes, uint64_t seed,
                            uint32_t epoch, int flags, double* absorption);

/* A disc of parallel rays (a distant source; the fields of
 * parallel_rays_emission_cpu::task_t, emission/parallel_rays_cpu.h:27-33). */
typedef struct {
  float direction[3]; /* ray direction (the reference does not normalise it) */
  float center[3];    /* the point the disc's axis passes through */
  float distance;     /* the disc lies at -distance along direction from center */
  float radius;       /* disc radius */
} ffb_disc_source;

/* Rays [0, n_rays) of the disc (emission/parallel_rays_cpu.cpp:88-106):
 * origin uniform on the disc, end point origin + 0.1 * direction, Philox
 * draws keyed by (seed, epoch, ray index).  rays6 host or device. */
int ffb_emit_parallel(ffb_ctx* ctx, const ffb_disc_source* src, long long n_rays, uint64_t seed, uint32_t epoch,
                      float* rays6);
/* The same rays cast through the resident grid, tallied per hit face and
 * side (the loop of thermal_equation/parallel_rays_cpu.cpp:110-122, fused):
 * side_counts[2h] counts rays meeting face h from its front
 * (dot(triangle_normal(h), direction) < 0), side_counts[2h + 1] the others.
 * side_counts is host or device, 2 * n_faces entries. */
int ffb_parallel_rays(ffb_ctx* ctx, const ffb_disc_source* src, long long n_rays, uint64_t seed, uint32_t epoch,
                      uint32_t* side_counts);

/* A mesh (subject::mesh_t, subject/system.h:64-69) and the optical
 * properties the ray-traced thermal equations read from its material
 * (subject::material_t front / rear, subject/system.h:41-59). */
typedef struct {
  int first_idx;
  int n_faces;
  int material_idx;
} ffb_mesh;
typedef struct {
  float front_emissivity, rear_emissivity;
  float front_absorbance, rear_absorbance;
} ffb_optics;

/* math::triangles_bsphere (math/triangle.cpp:361-384), host arithmetic op for
 * op (including the radius loop starting at the second triangle). */
int ffb_bounding_sphere(const float* faces9, int n_faces, float* center3, float* radius);

/* One calculate() of the radiance equation (thermal_equation/radiance_cpu.cpp
 * :96-190) on the resident scene and grid (faces9 / n_faces: the same scene
 * on the host, for areas).  Weights, ray budgets (n_rays), emission and
 * per-ray powers follow the reference in float; the rays run through
 * ffb_radiance_absorption.  emission[m] and absorption[m] are ADDED to, as the
 * reference's thermal_equation::task_t asks.  Meshes must cover every face
 * exactly once; FFB_ERR_ARG otherwise. */
int ffb_radiance_step(ffb_ctx* ctx, const float* faces9, int n_faces, const ffb_mesh* meshes, int n_meshes,
                      const ffb_optics* materials, int n_materials, const float* temperatures, int n_rays,
                      uint64_t seed, uint32_t epoch, int flags, float* emission, float* absorption);
/* One calculate() of the distant-source equation (thermal_equation/
 * parallel_rays_cpu.cpp:92-131): a disc of n_rays parallel rays of radius
 * 1.1 * bounding radius, 1.1 + radius in front of the bounding sphere's
 * centre along `direction`; each hit adds absorbance(side) * ray_power to its
 * mesh, ray_power = power * pi * radius^2 / n_rays.  absorption[m] is ADDED to. */
int ffb_distant_source_step(ffb_ctx* ctx, const float* faces9, int n_faces, const ffb_mesh* meshes, int n_meshes,
                            const ffb_optics* materials, int n_materials, int n_rays, float power,
                            const float* direction3, uint64_t seed, uint32_t epoch, float* absorption);

/* subject::material_t (subject/system.h:31-59), layout-identical. */
typedef struct {
  float shell_density, shell_heat_capacity, shell_thermal_conductivity, shell_thickness;
  float front_specular_reflectance, front_diffuse_reflectance, front_absorbance, front_transmittance, front_emissivity;
  float rear_specular_reflectance, rear_diffuse_reflectance, rear_absorbance, rear_transmittance, rear_emissivity;
  char name[128];
} ffb_material;

typedef struct {
  int n_vertices, n_faces, n_meshes, n_materials;
  int status;     /* what obj_import::scene returns: 0 or -OBJ_IMPORT_* (-21 file, -22 format, -23..-25 material) */
  int error_line; /* 1-based line of the first error, 0 when none */
} ffb_obj_info;

/* obj_import::scene (import_export/obj_import.cpp:167-340) with the geometry
 * parsed on the GPU: the text goes to the device once; lines, vertex ("v x y
 * z", sscanf "%f" = correctly rounded strtof) and face lines ("f" in the
 * reference's three formats) are split, converted and gathered into
 * triangles by kernels; the few object, usemtl and mtllib lines (and the
 * material library itself) are handled on the host in file order.  The
 * result is the reference's: faces, meshes (o/g), materials (or the black
 * body).  ffb_obj_parse takes the text in memory (filename: where mtllib
 * paths are resolved from, may be NULL); ffb_obj_load reads the file.
 * FFB_ERR_FORMAT / FFB_ERR_FILE on failure with info->status the reference's
 * code and info->error_line the line where the reference would stop.  A face
 * index outside the vertex list (undefined in the reference) and usemtl
 * before any object are format errors here. */
int ffb_obj_parse(ffb_ctx* ctx, const char* text, unsigned long long n_bytes, const char* filename,
                  ffb_obj_info* info);
int ffb_obj_load(ffb_ctx* ctx, const char* filename, ffb_obj_info* info);
/* The parsed scene: faces9 (host or device, 9 * n_faces floats), meshes
 * (n_meshes), materials (n_materials); any may be NULL. */
int ffb_obj_result(ffb_ctx* ctx, float* faces9, ffb_mesh* meshes, ffb_material* materials);
/* Makes the parsed faces the context's scene without a copy through the host
 * (then ffb_grid_build). */
int ffb_obj_scene_set(ffb_ctx* ctx);

/* CSV text of an n x n form-factor matrix, byte for byte the file of
 * csv_export::export_csv (import_export/csv_export.cpp:26-46): row i is the n
 * entries of matrix row i as `std::ostream << float` prints them ("%g",
 * 6 significant digits), separated by ';', each row ended by '\n'.
 *
 * ffb_csv_format: ff is host or device (n*n floats); text is a host or device
 * buffer of text_cap bytes, or NULL to get only the length in *text_len.
 * ffb_csv_format_counts: the same for counts normalised on the fly by their
 * row's outgoing rays, as ffb_normalise computes them (no float matrix is
 * formed).  FFB_ERR_ARG if the text does not fit text_cap (*text_len then
 * holds the length needed; a device buffer may hold part of the text).
 * ffb_csv_export / ffb_csv_export_counts: write the text to `filename`
 * (created or truncated); FFB_ERR_FILE when it cannot be opened or written,
 * where the reference returns -CSV_EXPORT_FILE_ERROR.  n == 0 writes an empty
 * file, as the reference does for a scene without meshes. */
int ffb_csv_format(ffb_ctx* ctx, const float* ff, int n, char* text, unsigned long long text_cap,
                   unsigned long long* text_len);
int ffb_csv_format_counts(ffb_ctx* ctx, const uint32_t* counts, const int32_t* outgoing, int n, char* text,
                          unsigned long long text_cap, unsigned long long* text_len);
int ffb_csv_export(ffb_ctx* ctx, const char* filename, const float* ff, int n);
int ffb_csv_export_counts(ffb_ctx* ctx, const char* filename, const uint32_t* counts, const int32_t* outgoing, int n);

/* Grid autotuner: builds the grid with each candidate (resolution,
 * cells_per_face, empty-space jumps), times the fused kernel on a sample of
 * the given ray budget (every sample_every-th face emits its rays), keeps the
 * fastest built and returns it in *best (and its sample time in *best_ms).
 * The scene must be set; nothing about the results depends on the choice. */
int ffb_autotune_grid(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, uint64_t seed,
                      const ffb_grid_params* candidates, int n_candidates, int sample_every, ffb_grid_params* best,
                      float* best_ms);

/* Launch shapes of the fused kernel: the kernel-side choices of the
 * autotuner.  A shape changes only the order in which a warp's lanes do their
 * work, never a ray's result or the counts. */
typedef struct {
  int adv_per_iter;   /* cell advances a lane may make per loop iteration */
  int test_per_iter;  /* triangle tests a lane may make per loop iteration */
  int refill_min;     /* idle lanes a warp waits for before it refills them */
  int blocks_per_sm;  /* resident 128-thread blocks per SM the kernel is built for */
  int coherent;       /* 1: a chunk's rays are handed out in direction order */
  int lanes;          /* 0: one ray per lane in registers; K: K rays per lane in shared memory, one
                         body (advances or tests) per iteration chosen by a vote of the lanes */
} ffb_trace_shape;

int ffb_trace_shape_count(void);
int ffb_trace_shape_get(int shape, ffb_trace_shape* out);
/* Launch shape of the context's form-factor traces (default 0). */
int ffb_ctx_set_trace_shape(ffb_ctx* ctx, int shape);
int ffb_ctx_trace_shape(ffb_ctx* ctx);

typedef struct {
  ffb_grid_params grid;  /* the chosen grid */
  int shape;             /* the chosen launch shape */
  float sample_ms;       /* its kernel time on the sample (0 when cached) */
  int from_cache;        /* 1: taken from the process-wide cache, not timed */
  int timed;             /* candidate runs timed */
  long long sample_rays; /* rays of the timing sample */
} ffb_tune_result;

#define FFB_TUNE_FORCE 1 /* time the candidates even when the cache holds a choice */

/* Autotuner of the fused form-factor trace for the context's scene and ray
 * budget (the reference's only tuning is the grid side of
 * math/grid.cpp:376-386 with a fixed 128-thread block,
 * cuda_ray_caster/system.cu:61).  Times the fused kernel on a sample of the
 * source faces (every sample_every-th face emits its rays; 0: a sample of
 * about 4 Mi rays): each grid candidate (`candidates`, or NULL for targets of
 * 32, 64, 128, 192 and 256 cells per face with empty-space jumps) with shape
 * 0, then every launch shape on the fastest grid.  Builds the chosen grid and
 * sets the context's shape.  The choice is cached per process under a key of
 * face count (half-octave steps), scene-box aspect and rays per emitting face
 * (octave steps); a cached choice is applied without timing unless flags has
 * FFB_TUNE_FORCE.  scratch: a device buffer of n_faces^2 uint32 the sample
 * traces may use (NULL: context memory).  Results never depend on the
 * choice. */
int ffb_autotune(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, uint64_t seed,
                 const ffb_grid_params* candidates, int n_candidates, int sample_every, int flags,
                 uint32_t* scratch, ffb_tune_result* out);

/* The autotuner over the scenes of a batch (after ffb_batch_set, before
 * ffb_batch_prepare): per scene, the cached choice for its key, or a tuning
 * run on that scene (through the context's main scene, which it replaces)
 * when the cache has none; each scene's grid is rebuilt with its choice and
 * its launch uses its shape.  front/rear as ffb_batch_prepare.  shapes (may
 * be NULL) gets each scene's shape. */
int ffb_batch_autotune(ffb_ctx* ctx, const int32_t* front, const int32_t* rear, int* shapes);

/* Counters and kernel time of the last ffb_cast / ffb_form_factor_counts
 * (synchronises the stream). */
int ffb_stats_get(ffb_ctx* ctx, ffb_stats* out);

/* Brute-force nearest hit for callers that cannot allocate device memory.
 * No counterpart in the reference: it exists for callers that may not call
 * cudaMalloc (code running under an allocator that owns all device memory,
 * or in a plugin host that forbids device allocations after start-up).
 * Same results as ffb_cast_bruteforce, without
 * a context: faces9, rays6, hit_face and hit_point (may be NULL) must all be
 * device memory of the current device (or managed memory), else FFB_ERR_ARG;
 * n_rays is at most (2^31 - 1) * 128, else FFB_ERR_TOO_LARGE.  The work is
 * enqueued on `stream` (a cudaStream_t, NULL for
 * the default stream) and the call returns without waiting.  The only
 * scratch, the per-face triangle records, lives in a static device array of
 * 16384 faces (1 MiB, held by every GPU that loads the library until exit);
 * larger scenes return FFB_ERR_TOO_LARGE.  All calls share that array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * The first call on a device resolves the array's address with that device
 * current; make it before any stream capture. */
int ffb_cast_bruteforce_static(const float* faces9, int n_faces, const float* rays6, long long n_rays,
                               int32_t* hit_face, float* hit_point, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FFB_H */
