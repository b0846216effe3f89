// gvh_surface_rows.cu -- the surface.dat rows of a slab's crossed hypercubes on the device,
// and their text.
//
// One thread per crossed hypercube runs the code of gvh_surface_rows.hpp (cornelius, the
// reference's interpolation to the element's centroid, the row) -- the code the host pool
// runs -- and writes its rows to fixed slots (kMaxElements per hypercube); the rows are the
// filled slots in slot order, which is the reference's order (hypercubes in loop order, a
// cube's elements in cornelius' order). One thread per hypercube then writes its rows' text with
// the fast path of %g (gvh_format.hpp); a scan over the slots' text lengths places each row's
// text in the slab's text, compacted in device memory for one copy to the host by the copy
// engine. Rows with a number the fast path leaves to the exact one go to the host as values
// (HostRow), which formats them and splices them in. This file is compiled without FMA
// contraction (-fmad=false, like the host side's -ffp-contract=off), so device and host rows
// agree to the last bit.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include "gvh_format.hpp"
#include "gvh_surface_device.h"
#include "gvh_surface_rows.hpp"

namespace gvh {
namespace surface {
namespace {

// One thread per crossed hypercube: a slab's ~47 k hypercubes make one partial wave, so
// small blocks spread them evenly over the SMs (32 threads: 491.5 us a slab against 521.6 us
// with 128 on the 131x131x61 event).
constexpr int kRowThreads = 32;
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

// The text of hypercube c's rows, one thread per hypercube: for each of its filled slots the
// fast path of %g for each number, a space between them, a newline after the last. An empty
// slot, or a row with a number the fast path leaves to the exact one (a host row), gets
// length 0; thread 0 also writes the scan's closing 0 (slot_len[ncubes kSlotRows]).
__global__ void slot_text_kernel(long long ncubes, const double *__restrict__ slot_rows,
                                 const int *__restrict__ slot_n, char *__restrict__ text_slots,
                                 long long *__restrict__ slot_len, unsigned char *__restrict__ slot_host) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c == 0) slot_len[ncubes * kSlotRows] = 0;
  if (c >= ncubes) return;
  const int n = slot_n[c];
  for (int i = 0; i < kSlotRows; ++i) {
    const long long t = c * kSlotRows + i;
    long long len = 0;
    if (i < n) {
      const double *row = slot_rows + t * kRowColumns;
      char *out = text_slots + t * kTextSlot;
      char *p = out;
      unsigned char host = 0;
      for (int k = 0; k < kRowColumns; ++k) {
        char *q = fmt::g6_fast(p, row[k]);
        if (!q) {
          host = 1;
          break;
        }
        p = q;
        *p++ = k + 1 < kRowColumns ? ' ' : '\n';
      }
      slot_host[t] = host;
      len = host ? 0 : p - out;
    }
    slot_len[t] = len;
  }
}

// One warp per hypercube (grid-stride): each of its rows' text to its place in the slab's
// text (32 consecutive bytes per warp store), a host row's values and places to host_rows.
__global__ void text_compact_kernel(long long ncubes, const int *__restrict__ slot_n,
                                    const int *__restrict__ offsets, const double *__restrict__ slot_rows,
                                    const long long *__restrict__ slot_len, const long long *__restrict__ text_off,
                                    const unsigned char *__restrict__ slot_host, const char *__restrict__ text_slots,
                                    char *__restrict__ text, HostRow *__restrict__ host_rows, long long host_rows_cap,
                                    long long *__restrict__ totals) {
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long c = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; c < ncubes; c += warps) {
    const int n = slot_n[c];
    for (int i = 0; i < n; ++i) {
      const long long s = c * kSlotRows + i;
      if (slot_host[s]) {
        long long j = 0;
        if (lane == 0) j = (long long)atomicAdd(reinterpret_cast<unsigned long long *>(totals + 3), 1ull);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j < host_rows_cap) {
          HostRow &h = host_rows[j];
          if (lane < kRowColumns) h.v[lane] = slot_rows[s * kRowColumns + lane];
          if (lane == kRowColumns) h.text_off = text_off[s];
          if (lane == kRowColumns + 1) h.row = (long long)offsets[c] + i;
        }
      } else {
        const int len = (int)slot_len[s];
        const char *src = text_slots + s * kTextSlot;
        char *dst = text + text_off[s];
        for (int b = lane; b < len; b += 32) dst[b] = src[b];
      }
    }
  }
}

// Every row in order to rows (grid-stride over the slots' values, one thread per value) when
// all rows are wanted: always (copy_all), or when the host rows overflowed their buffer.
__global__ void rows_compact_kernel(long long ncubes, const double *__restrict__ slot_rows,
                                    const int *__restrict__ slot_n, const int *__restrict__ offsets,
                                    const long long *__restrict__ totals, bool copy_all, long long host_rows_cap,
                                    double *__restrict__ rows) {
  if (!copy_all && totals[3] <= host_rows_cap) return;
  const long long per_cube = (long long)kSlotRows * kRowColumns;
  const long long values = ncubes * per_cube;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < values; t += stride) {
    const long long c = t / per_cube;
    const int v = (int)(t - c * per_cube);
    if (v < slot_n[c] * kRowColumns) rows[(long long)offsets[c] * kRowColumns + v] = slot_rows[t];
  }
}

// totals[0] (rows) and [2] (text bytes) from the scans' closing entries, then all of them to
// the host.
__global__ void totals_kernel(long long ncubes, const int *__restrict__ offsets, long long n_slots,
                              const long long *__restrict__ text_off, bool text, long long *__restrict__ totals,
                              long long *__restrict__ host_totals) {
  totals[0] = offsets[ncubes];
  totals[2] = text ? text_off[n_slots] : 0;
  for (int i = 0; i < 4; ++i) host_totals[i] = totals[i];
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

size_t scan_temp_bytes(long long cap) {
  size_t a = 0, b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, a, (const int *)nullptr, (int *)nullptr, (int)(cap + 1));
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const long long *)nullptr, (long long *)nullptr,
                                (int)(cap * kSlotRows + 1));
  return align256(a > b ? a : b);
}

}  // namespace

size_t device_rows_scratch_bytes(long long cap) {
  const size_t slots = (size_t)cap * kSlotRows;
  return 1024 + 2 * align256(slots * kRowColumns * sizeof(double)) + 2 * align256((size_t)(cap + 1) * sizeof(int)) +
         2 * align256((slots + 1) * sizeof(long long)) + align256(slots) + 2 * align256(slots * kTextSlot) +
         scan_temp_bytes(cap);
}

void device_rows_carve(DeviceRows &d, char *base, long long cap) {
  const size_t slots = (size_t)cap * kSlotRows;
  char *p = base;
  d.totals = reinterpret_cast<long long *>(p); p += 1024;
  d.slot_rows = reinterpret_cast<double *>(p); p += align256(slots * kRowColumns * sizeof(double));
  d.rows = reinterpret_cast<double *>(p); p += align256(slots * kRowColumns * sizeof(double));
  d.slot_n = reinterpret_cast<int *>(p); p += align256((size_t)(cap + 1) * sizeof(int));
  d.offsets = reinterpret_cast<int *>(p); p += align256((size_t)(cap + 1) * sizeof(int));
  d.slot_len = reinterpret_cast<long long *>(p); p += align256((slots + 1) * sizeof(long long));
  d.text_off = reinterpret_cast<long long *>(p); p += align256((slots + 1) * sizeof(long long));
  d.slot_host = reinterpret_cast<unsigned char *>(p); p += align256(slots);
  d.text_slots = p; p += align256(slots * kTextSlot);
  d.text = p; p += align256(slots * kTextSlot);
  d.scan_temp = p;
  d.scan_temp_bytes = scan_temp_bytes(cap);
}

cudaError_t launch_device_rows(const DeviceRows &d, cudaStream_t st) {
  if (d.ncubes <= 0) return cudaSuccess;  // the caller sets the totals to zero
  cudaError_t e = cudaMemsetAsync(d.totals, 0, 4 * sizeof(long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d.slot_n + d.ncubes, 0, sizeof(int), st);  // the scan's closing 0
  if (e != cudaSuccess) return e;
  point_index_kernel<<<(unsigned)((d.npoints + 255) / 256), 256, 0, st>>>(d.npoints, d.point_cell, d.c2p);
  const unsigned blocks = (unsigned)((d.ncubes + kRowThreads - 1) / kRowThreads);
  cube_rows_kernel<<<blocks, kRowThreads, 0, st>>>(d.g, d.ncubes, d.cube_key, d.c2p, d.point_vals, d.slot_rows,
                                                   d.slot_n, reinterpret_cast<unsigned long long *>(d.totals + 1));
  size_t temp = d.scan_temp_bytes;
  if ((e = cub::DeviceScan::ExclusiveSum(d.scan_temp, temp, d.slot_n, d.offsets, (int)(d.ncubes + 1), st)))
    return e;
  const long long n_slots = d.ncubes * kSlotRows;
  const bool text = d.text != nullptr;
  if (text) {
    slot_text_kernel<<<(unsigned)((d.ncubes + kRowThreads - 1) / kRowThreads), kRowThreads, 0, st>>>(
        d.ncubes, d.slot_rows, d.slot_n, d.text_slots, d.slot_len, d.slot_host);
    temp = d.scan_temp_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(d.scan_temp, temp, d.slot_len, d.text_off, (int)(n_slots + 1), st)))
      return e;
    text_compact_kernel<<<148 * 8, 256, 0, st>>>(d.ncubes, d.slot_n, d.offsets, d.slot_rows, d.slot_len, d.text_off,
                                                 d.slot_host, d.text_slots, d.text, d.host_rows, d.host_rows_cap,
                                                 d.totals);
  }
  rows_compact_kernel<<<148 * 8, 256, 0, st>>>(d.ncubes, d.slot_rows, d.slot_n, d.offsets, d.totals,
                                               d.keep_rows || !text, d.host_rows_cap, d.rows);
  totals_kernel<<<1, 1, 0, st>>>(d.ncubes, d.offsets, n_slots, d.text_off, text, d.totals, d.host_totals);
  return cudaGetLastError();
}

}  // namespace surface
}  // namespace gvh
