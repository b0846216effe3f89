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

#include "gvh_surface_rows.hpp"
#include "gvh_surface_device.h"

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
                                 long long *__restrict__ totals, long long *__restrict__ host_totals) {
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
  if (threadIdx.x == blockDim.x - 1) {
    totals[0] = part[threadIdx.x];
    host_totals[0] = part[threadIdx.x];
    host_totals[1] = totals[1];  // the row kernel's error count (it ran before this kernel)
  }
}

// One thread per value of a slot (hypercube c, row i, column k): consecutive threads write
// consecutive values of a row, so each row crosses the host link as one contiguous write.
__global__ void rows_compact_kernel(long long ncubes, const double *__restrict__ slot_rows,
                                    const int *__restrict__ slot_n, const int *__restrict__ offsets,
                                    double *__restrict__ rows) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per_cube = (long long)kSlotRows * kRowColumns;
  const long long c = t / per_cube;
  if (c >= ncubes) return;
  const int v = (int)(t - c * per_cube);
  if (v >= slot_n[c] * kRowColumns) return;
  rows[(long long)offsets[c] * kRowColumns + v] = slot_rows[c * per_cube + v];
}

}  // namespace

size_t device_rows_slot_bytes(long long ncubes) {
  return (size_t)ncubes * (kSlotRows * kRowColumns * sizeof(double) + 2 * sizeof(int));
}

cudaError_t launch_device_rows(const DeviceRows &d, cudaStream_t st) {
  if (d.ncubes <= 0) return cudaSuccess;  // the caller sets the totals to zero
  cudaError_t e = cudaMemsetAsync(d.totals, 0, 2 * sizeof(long long), st);
  if (e != cudaSuccess) return e;
  point_index_kernel<<<(unsigned)((d.npoints + 255) / 256), 256, 0, st>>>(d.npoints, d.point_cell, d.c2p);
  const unsigned blocks = (unsigned)((d.ncubes + kRowThreads - 1) / kRowThreads);
  cube_rows_kernel<<<blocks, kRowThreads, 0, st>>>(d.g, d.ncubes, d.cube_key, d.c2p, d.point_vals, d.slot_rows,
                                                   d.slot_n, reinterpret_cast<unsigned long long *>(d.totals + 1));
  rows_scan_kernel<<<1, 1024, 0, st>>>(d.ncubes, d.slot_n, d.offsets, d.totals, d.host_totals);
  const long long values = d.ncubes * (long long)(kSlotRows * kRowColumns);
  rows_compact_kernel<<<(unsigned)((values + 255) / 256), 256, 0, st>>>(d.ncubes, d.slot_rows, d.slot_n, d.offsets,
                                                                        d.rows);
  return cudaGetLastError();
}

}  // namespace surface
}  // namespace gvh
