// leco_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "../../include/leco.h"

namespace leco {

struct EncodeLaunch {
  const void *values;
  uint64_t n;
  uint32_t bs;
  uint64_t nb;
  uint8_t *payload;
  uint64_t payload_cap;
  uint64_t *offsets;
  leco_dir_entry *dir;
  double *seq_models;  // non-null: run the sequential reference fit first
  double polyX[10];    // X sums (full block, tail block) for the degree-2 fit
  uint64_t *status;
  uint32_t *ticket;
  uint32_t *error;
};

struct DecodeLaunch {
  const uint8_t *payload;
  const uint64_t *offsets;
  uint64_t n;
  uint32_t bs;
  uint64_t first, count;
  void *out;
  uint32_t *error;
};

struct GatherLaunch {
  const uint8_t *payload;
  const uint64_t *offsets;
  const leco_dir_entry *dir;
  uint64_t n;
  uint32_t bs;
  const uint64_t *idx;
  uint64_t m;
  void *out;
  uint32_t *error;
};

// Predicate pushdown over a column (leco_filter.cu).
struct FilterLaunch {
  const uint8_t *payload;
  const uint64_t *offsets;
  uint64_t n;
  uint32_t bs;
  uint64_t nb;
  uint64_t f1, f2;       // range: f1 = the filter; close range: the window (LeCo) or residue (FOR) bounds
  uint64_t base;         // close range: window step (LeCo) / modulus (FOR), 1..INT32_MAX
  const uint64_t *zone;  // range: per-block maxima (nullable); close-range LeCo: per-block minima (nullable)
  const uint64_t *zone_lo;  // range: per-block minima (nullable)
  uint32_t *out;
  uint64_t cap;
  uint64_t *count;
  uint64_t *counts;      // [nb] matches per block (workspace)
  uint64_t *group_tot;   // [ceil(nb/32)] matches per group of 32 blocks, then their exclusive prefix (workspace)
  uint32_t *error;
  uint32_t max_windows;  // close-range LeCo: windows per block before kErrLimit (a multiple of 32)
  int vec_out;           // out is 16-byte aligned: runs of indices are written with 16-byte stores
};

int launch_encode(int codec, int s, const EncodeLaunch &L, cudaStream_t st);
// 0: launched; 1: no kernel for the codec and type; < 0: -(cudaError_t) of a failed launch
int launch_filter(int codec, int s, const FilterLaunch &L, int close, cudaStream_t st);
int launch_zonemap(int codec, int s, const DecodeLaunch &L, uint64_t *zmin, uint64_t *zmax, cudaStream_t st);
int launch_decode(int codec, int s, const DecodeLaunch &L, cudaStream_t st);
int launch_gather(int codec, int s, const GatherLaunch &L, cudaStream_t st);
int launch_sum(int codec, int s, const DecodeLaunch &L, uint64_t *d_sum, cudaStream_t st);
int launch_build_dir(int codec, int s, const uint8_t *payload, const uint64_t *offsets, uint64_t n, uint32_t bs,
                     leco_dir_entry *dir, uint32_t *error, cudaStream_t st);

// Reference X sums of polynomial_regression_iter: X[k] = sum_{j<N} j^k as a
// sequential FP64 loop (polynomial_regression_internals.hpp:111-116), x^k built
// by repeated multiplication (:80-99).  Host code, compiled with
// -ffp-contract=off.
void poly2_x_sums(uint32_t N, double X[5]);

// Device address of the library's error word on the current device.
int device_error_word(uint32_t **p);

// Records `msg` as this thread's leco_last_error() message and returns `code`.
int record_error(int code, const std::string &msg);

}  // namespace leco
