// ffb_pack.cuh -- compaction of a finished row block of the count matrix to
// (column, count) pairs, the form in which a host output crosses PCIe.
#pragma once

#include <cstdint>

namespace ffb {

// Header of a packed row block of `rows` rows, in uint32 words:
//   [0] pairs reserved by the rows (their cursor; may exceed the cap)
//   [1] unused
//   [2 + r] first pair of row r          [2 + rows + r] pairs of row r
__host__ __device__ constexpr size_t pack_header_words(int rows) { return 2 + 2 * (size_t)rows; }

constexpr int kPackThreads = 256;

// A pair is two words (column, count), or with kNarrow one word
// column | count << 16, when columns and counts are below 2^16.
template <bool kNarrow>
__device__ __forceinline__ void pack_pair_store(void* pairs, uint32_t k, uint32_t col, uint32_t v)
{
  if (kNarrow)
    static_cast<uint32_t*>(pairs)[k] = col | (v << 16);
  else
    static_cast<uint2*>(pairs)[k] = make_uint2(col, v);
}

// One CTA per row (grid-stride over rows).  Pass 1 counts the row's nonzero
// entries (16-byte loads when the row is 16-byte aligned), one atomic on
// hdr[0] reserves that many pairs, and (first, count) goes to the header.
// Pass 2 walks the row in tiles of 4 entries per thread (the row is in L2
// from pass 1): a CTA-wide exclusive scan of the threads' nonzero counts
// gives each nonzero its slot, so the pairs (column, count) of a row are in
// column order.  A row whose pairs would pass `cap` writes none: the host
// sees hdr[0] > cap and copies the block dense.  hdr[0] is zero before the
// launch.
template <bool kNarrow>
__global__ void __launch_bounds__(kPackThreads) k_rows_pack(const uint32_t* __restrict__ counts, int rows,
                                                            int n_cols, uint32_t* __restrict__ hdr, uint32_t cap,
                                                            void* __restrict__ pairs)
{
  constexpr int kWarps = kPackThreads / 32;
  constexpr uint32_t kSkip = 0xFFFFFFFFu;
  __shared__ uint32_t s_warp[kWarps];
  __shared__ uint32_t s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const uint32_t* row = counts + (size_t)r * (size_t)n_cols;
    uint32_t nz = 0;
    if ((n_cols & 3) == 0 && ((uintptr_t)row & 15u) == 0) {
      const uint4* v = reinterpret_cast<const uint4*>(row);
      for (int i = tid; i < (n_cols >> 2); i += kPackThreads) {
        const uint4 q = __ldg(v + i);
        nz += (q.x != 0u) + (q.y != 0u) + (q.z != 0u) + (q.w != 0u);
      }
    } else {
      for (int i = tid; i < n_cols; i += kPackThreads)
        nz += __ldg(row + i) != 0u;
    }
    nz = __reduce_add_sync(0xFFFFFFFFu, nz);
    if (lane == 0)
      s_warp[warp] = nz;
    __syncthreads();
    if (tid == 0) {
      uint32_t total = 0;
      for (int w = 0; w < kWarps; ++w)
        total += s_warp[w];
      const uint32_t base = total ? atomicAdd(hdr, total) : 0u;
      hdr[2 + r] = base;
      hdr[2 + (size_t)rows + r] = total;
      s_base = (total == 0u || base > cap || total > cap - base) ? kSkip : base;
    }
    __syncthreads();
    uint32_t pos = s_base;
    if (pos != kSkip) {  // uniform over the CTA
      for (int t0 = 0; t0 < n_cols; t0 += 4 * kPackThreads) {
        const int i0 = t0 + 4 * tid;
        uint32_t v[4];
        uint32_t c = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          v[j] = i0 + j < n_cols ? row[i0 + j] : 0u;
          c += v[j] != 0u;
        }
        // inclusive scan of c over the warp, then over the warps
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
          if (lane >= d)
            incl += y;
        }
        __syncthreads();  // the previous tile's reads of s_warp are done
        if (lane == 31)
          s_warp[warp] = incl;
        __syncthreads();
        uint32_t before = 0, tile = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
          const uint32_t x = s_warp[w];
          before += w < warp ? x : 0u;
          tile += x;
        }
        uint32_t q = pos + before + incl - c;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (v[j] != 0u)
            pack_pair_store<kNarrow>(pairs, q++, (uint32_t)(i0 + j), v[j]);
        pos += tile;
      }
    }
    __syncthreads();  // s_warp and s_base are rewritten for the next row
  }
}

}  // namespace ffb
