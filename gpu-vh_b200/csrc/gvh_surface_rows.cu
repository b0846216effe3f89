// gvh_surface_rows.cu -- the surface.dat rows of a slab's crossed hypercubes on the device.
//
// One thread per crossed hypercube runs the code of gvh_surface_rows.hpp (cornelius, the
// reference's interpolation to the element's centroid, the row) -- the code the host pool
// runs -- and writes its rows to a fixed slot; a scan over the per-cube counts and a
// compaction then give the rows in the reference's order (hypercubes in loop order, a
// cube's elements in cornelius' order), written straight into mapped pinned host memory, so
// nothing waits between the kernels and the copy. This file is compiled without FMA contraction
// (-fmad=false, like the host side's -ffp-contract=off), so device and host rows agree to
// the last bit; the host then only formats them (gvh_surface.cu).
#include <cuda_runtime.h>

#include "gvh_format.hpp"
#include "gvh_surface_device.h"
#include "gvh_surface_rows.hpp"

namespace gvh {
namespace surface {
namespace {

constexpr int kRowThreads = 128;
constexpr int kSlotRows = iso::kMaxElements;  // rows a hypercube can have

__global__ void point_index_kernel(long long npoints, const int *__restrict__ point_cell, int *__restrict__ c2p) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < npoints) c2p[point_cell[p]] = (int)p;
}

__global__ void __launch_bounds__(kRowThreads) cube_rows_kernel(RowGeometry g, long long ncubes,
                                                                const int *__restrict__ cube_key,
                                                                const int *__restrict__ c2p,
                                                                const double *__restrict__ point_vals,
                                                                double *__restrict__ slot_rows,
                                                                int *__restrict__ slot_n,
                                                                unsigned long long *__restrict__ errors) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= ncubes) return;
  RowWork w;
  const int key = cube_key[c];
  gather_corners(g, key, c2p, point_vals, w);
  const int n = cube_rows(g, key, w, slot_rows + c * (long long)(kSlotRows * kRowColumns));
  if (n < 0) {
    slot_n[c] = 0;
    atomicAdd(errors, 1ull);
  } else {
    slot_n[c] = n;
  }
}

// Exclusive offsets of slot_n (one block); totals[0] = the number of rows.
__global__ void rows_scan_kernel(long long n, const int *__restrict__ slot_n, int *__restrict__ offsets,
                                 long long *__restrict__ totals) {
  __shared__ long long part[1024];
  const long long per = (n + blockDim.x - 1) / blockDim.x;
  const long long lo = min(n, (long long)threadIdx.x * per), hi = min(n, lo + per);
  long long sum = 0;
  for (long long i = lo; i < hi; ++i) sum += slot_n[i];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {
    const long long v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - sum;
  for (long long i = lo; i < hi; ++i) {
    offsets[i] = (int)run;
    run += slot_n[i];
  }
  if (threadIdx.x == blockDim.x - 1) totals[0] = part[threadIdx.x];
}

// The text of slot (c, i) (hypercube c, its i-th element), row offsets[c] + i: the fast path
// of %g for each number, a space between them, a newline after the last; -1 as the length
// when the fast path leaves a number to the exact one.
__global__ void rows_text_kernel(long long ncubes, const double *__restrict__ slot_rows,
                                 const int *__restrict__ slot_n, const int *__restrict__ offsets,
                                 char *__restrict__ text_slots, int *__restrict__ row_len) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long c = t / kSlotRows;
  if (c >= ncubes) return;
  const int i = (int)(t - c * kSlotRows);
  if (i >= slot_n[c]) return;
  const long long r = (long long)offsets[c] + i;
  const double *row = slot_rows + t * kRowColumns;
  char *out = text_slots + r * kTextSlot;
  char *p = out;
  for (int k = 0; k < kRowColumns; ++k) {
    char *q = fmt::g6_fast(p, row[k]);
    if (!q) {
      row_len[r] = -1;
      return;
    }
    p = q;
    *p++ = k + 1 < kRowColumns ? ' ' : '\n';
  }
  row_len[r] = (int)(p - out);
}

// Exclusive offsets of the rows' text (one block; a row of length -1 counts 0), into
// text_off and the host's copy; totals[2] = the text's bytes, totals[3] = whether they fit,
// totals[4] = the rows the host formats.
__global__ void text_scan_kernel(const int *__restrict__ row_len, long long text_cap,
                                 long long *__restrict__ totals, long long *__restrict__ text_off,
                                 long long *__restrict__ host_text_off) {
  __shared__ long long part[1024];
  const long long n = totals[0];
  const long long per = (n + blockDim.x - 1) / blockDim.x;
  const long long lo = min(n, (long long)threadIdx.x * per), hi = min(n, lo + per);
  long long sum = 0;
  unsigned long long host_rows = 0;
  for (long long i = lo; i < hi; ++i) {
    sum += max(row_len[i], 0);
    host_rows += row_len[i] < 0;
  }
  if (host_rows) atomicAdd(reinterpret_cast<unsigned long long *>(totals + 4), host_rows);
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {
    const long long v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - sum;
  for (long long i = lo; i < hi; ++i) {
    text_off[i] = run;
    host_text_off[i] = run;
    run += max(row_len[i], 0);
  }
  if (threadIdx.x == blockDim.x - 1) {
    const long long bytes = part[threadIdx.x];
    text_off[n] = bytes;
    host_text_off[n] = bytes;
    totals[2] = bytes;
    totals[3] = bytes <= text_cap ? 1 : 0;
  }
}

// One thread per value of a slot (hypercube c, row i, column k): consecutive threads write
// consecutive values of a row, so each row crosses the host link as one contiguous write.
// With row_len (text made) a row is written only when the host formats it, the text did not
// fit, or copy_all.
__global__ void rows_compact_kernel(long long ncubes, const double *__restrict__ slot_rows,
                                    const int *__restrict__ slot_n, const int *__restrict__ offsets,
                                    const int *__restrict__ row_len, const long long *__restrict__ totals,
                                    bool copy_all, double *__restrict__ rows) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per_cube = (long long)kSlotRows * kRowColumns;
  const long long c = t / per_cube;
  if (c >= ncubes) return;
  const int v = (int)(t - c * per_cube);
  if (v >= slot_n[c] * kRowColumns) return;
  const long long at = (long long)offsets[c] * kRowColumns + v;
  if (row_len && !copy_all && totals[3] && row_len[at / kRowColumns] >= 0) return;
  rows[at] = slot_rows[c * per_cube + v];
}

// One warp per row (grid-stride): the row's text to its place in the concatenated text, in
// mapped host memory, 32 consecutive bytes per warp store.
__global__ void text_compact_kernel(const long long *__restrict__ totals, const int *__restrict__ row_len,
                                    const long long *__restrict__ text_off, const char *__restrict__ text_slots,
                                    char *__restrict__ text) {
  if (!totals[3]) return;
  const long long n = totals[0];
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const int len = row_len[r];
    const char *src = text_slots + r * kTextSlot;
    char *dst = text + text_off[r];
    for (int b = lane; b < len; b += 32) dst[b] = src[b];
  }
}

__global__ void host_totals_kernel(const long long *__restrict__ totals, long long *__restrict__ host_totals) {
  for (int i = 0; i < 5; ++i) host_totals[i] = totals[i];
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

size_t device_rows_slot_bytes(long long ncubes) {
  const size_t slots = (size_t)ncubes * kSlotRows;
  return align256(slots * kRowColumns * sizeof(double)) + 2 * align256((size_t)ncubes * sizeof(int)) +
         align256(slots * sizeof(int)) + align256((slots + 1) * sizeof(long long)) + align256(slots * kTextSlot);
}

void device_rows_carve(DeviceRows &d, char *base, long long cap) {
  const size_t slots = (size_t)cap * kSlotRows;
  char *p = base;
  d.totals = reinterpret_cast<long long *>(p); p += 1024;
  d.slot_rows = reinterpret_cast<double *>(p); p += align256(slots * kRowColumns * sizeof(double));
  d.slot_n = reinterpret_cast<int *>(p); p += align256((size_t)cap * sizeof(int));
  d.offsets = reinterpret_cast<int *>(p); p += align256((size_t)cap * sizeof(int));
  d.row_len = reinterpret_cast<int *>(p); p += align256(slots * sizeof(int));
  d.text_off = reinterpret_cast<long long *>(p); p += align256((slots + 1) * sizeof(long long));
  d.text_slots = p;
}

cudaError_t launch_device_rows(const DeviceRows &d, cudaStream_t st) {
  if (d.ncubes <= 0) return cudaSuccess;  // the caller sets the totals to zero
  cudaError_t e = cudaMemsetAsync(d.totals, 0, 5 * sizeof(long long), st);
  if (e != cudaSuccess) return e;
  point_index_kernel<<<(unsigned)((d.npoints + 255) / 256), 256, 0, st>>>(d.npoints, d.point_cell, d.c2p);
  const unsigned blocks = (unsigned)((d.ncubes + kRowThreads - 1) / kRowThreads);
  cube_rows_kernel<<<blocks, kRowThreads, 0, st>>>(d.g, d.ncubes, d.cube_key, d.c2p, d.point_vals, d.slot_rows,
                                                   d.slot_n, reinterpret_cast<unsigned long long *>(d.totals + 1));
  rows_scan_kernel<<<1, 1024, 0, st>>>(d.ncubes, d.slot_n, d.offsets, d.totals);
  const long long slots = d.ncubes * (long long)kSlotRows;
  if (d.text) {
    rows_text_kernel<<<(unsigned)((slots + 255) / 256), 256, 0, st>>>(d.ncubes, d.slot_rows, d.slot_n, d.offsets,
                                                                     d.text_slots, d.row_len);
    text_scan_kernel<<<1, 1024, 0, st>>>(d.row_len, d.text_cap, d.totals, d.text_off, d.host_text_off);
  }
  const long long values = slots * kRowColumns;
  rows_compact_kernel<<<(unsigned)((values + 255) / 256), 256, 0, st>>>(
      d.ncubes, d.slot_rows, d.slot_n, d.offsets, d.text ? d.row_len : nullptr, d.totals, d.keep_rows, d.rows);
  if (d.text) text_compact_kernel<<<148 * 8, 256, 0, st>>>(d.totals, d.row_len, d.text_off, d.text_slots, d.text);
  host_totals_kernel<<<1, 1, 0, st>>>(d.totals, d.host_totals);
  return cudaGetLastError();
}

}  // namespace surface
}  // namespace gvh
