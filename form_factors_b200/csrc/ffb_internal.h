// ffb_internal.h -- library-internal entry points shared by the translation
// units of libffb200.so (not part of the public C ABI in include/ffb.h).
#pragma once

#include <cstdint>

#include "ffb.h"

// Records an error for ffb_last_error and returns `code`.
int ffb_set_error(int code, const char* msg);

// Sliced traces, for the serving loop.  ffb_trace_prepare readies one fused
// form-factor trace of the context's scene (grid built) with per-face
// (front, rear) ray counts, Philox (seed, epoch) and emission flags: it
// builds the chunk table (256 consecutive rays of one face per chunk), zeroes
// the device matrix `counts` (n_faces^2 uint32) and returns the number of
// chunks.  ffb_trace_slice enqueues the launch over chunks
// [first, first + count) on `stream` (NULL: the context stream; the
// prepare's work must be complete or ordered before it, and all slices of
// one prepared trace must go to one stream: they share its chunk cursor);
// the slices of a prepared
// trace may come in any split, and once every chunk has been traced exactly
// once `counts` equals what ffb_form_factor_counts gives for the same
// arguments (integer sums do not depend on the order).  ffb_trace_span
// returns the earliest block start and latest warp end of all slices since
// the prepare, in %globaltimer nanoseconds (synchronises the stream).
int ffb_trace_prepare(ffb_ctx* c, const int32_t* front, const int32_t* rear, uint64_t seed, uint32_t epoch, int flags,
                      uint32_t* counts, long long* n_chunks);
int ffb_trace_slice(ffb_ctx* c, long long first, long long count, void* stream);
int ffb_trace_span(ffb_ctx* c, unsigned long long* start_ns, unsigned long long* end_ns);

// Host threads that write count-matrix rows into a host buffer from the
// (column, count) pairs of their nonzero entries (ffb_host_rows.cpp).
// ffb_host_expand_start hands rows [0, rows) to the pool and returns: row r
// of the n_cols-wide uint32 matrix at dst gets the count[r] pairs from pair
// first[r] on (columns ascending and below n_cols) and zeros elsewhere;
// every entry of the rows is written.  A pair is two words (column, count),
// or with `narrow` one word column | count << 16.  ffb_host_expand_join
// waits until the rows are written (and their streaming stores are
// visible).  One job at a time per pool; the buffers must stay valid until
// the join.
struct ffb_host_pool;
ffb_host_pool* ffb_host_pool_create(int threads);  // null when threads or memory run out
void ffb_host_pool_destroy(ffb_host_pool* p);
int ffb_host_pool_threads(const ffb_host_pool* p);
void ffb_host_expand_start(ffb_host_pool* p, uint32_t* dst, int rows, int n_cols, const uint32_t* first,
                           const uint32_t* count, const uint32_t* pairs, int narrow);
// The same rows as floats (float)count * inv[r] -- zeros as 0.f * inv[r] --
// for a normalised form-factor matrix (inv[r] = 1.f / (float)outgoing[r]).
void ffb_host_expand_norm_start(ffb_host_pool* p, float* dst, int rows, int n_cols, const uint32_t* first,
                                const uint32_t* count, const uint32_t* pairs, int narrow, const float* inv);
void ffb_host_expand_join(ffb_host_pool* p);
