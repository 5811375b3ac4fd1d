// Validation of caller-supplied index arrays before kernels index other arrays with them.
//
// The public entry points take node ids, element / face tables and CSR patterns
// as device arrays.  Each one runs these checks once, at set-up, before the first
// kernel that uses the ids as addresses, and turns a bad id into DGP_ERR_MESH
// instead of an out-of-bounds access.
#include <algorithm>
#include <string>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr int CHECK_NT = 256;
constexpr int64_t CHECK_MAX_BLOCKS = 148 * 16;

unsigned check_grid(int64_t count) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(count, CHECK_NT), CHECK_MAX_BLOCKS));
}

// *err |= 1 when any of ids[0..count) lies outside [0, limit)
__global__ void k_ids_in_range(const int32_t *__restrict__ ids, int64_t count, int64_t limit, int *err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    if (ids[i] < 0 || ids[i] >= limit) atomicOr(err, 1);
}

// *err |= 2 unless rowptr[0] == 0 and rowptr is non-decreasing over [0, nrows];
// *err |= 4 when a row holds more than max_row entries (max_row > 0)
__global__ void k_rowptr_ok(const int32_t *__restrict__ rowptr, int64_t nrows, int64_t max_row, int *err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t len = (int64_t)rowptr[i + 1] - rowptr[i];
    if (len < 0 || (i == 0 && rowptr[0] != 0)) atomicOr(err, 2);
    if (max_row > 0 && len > max_row) atomicOr(err, 4);
  }
}

int read_flag(const DevBuf &err, cudaStream_t st, int *h) {
  DGP_CUDA(cudaMemcpyAsync(h, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

}  // namespace

int ids_in_range(const int32_t *d_ids, int64_t count, int64_t limit, const char *who, cudaStream_t st) {
  if (count <= 0) return DGP_OK;
  DGP_REQUIRE(d_ids, std::string(who) + ": null index array");
  DevBuf err;
  DGP_TRY(err.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  k_ids_in_range<<<check_grid(count), CHECK_NT, 0, st>>>(d_ids, count, limit, err.as<int>());
  DGP_CHECK_LAUNCH();
  int h = 0;
  DGP_TRY(read_flag(err, st, &h));
  if (h) return fail(DGP_ERR_MESH, std::string(who) + ": node index out of range");
  return DGP_OK;
}

int csr_in_range(const int32_t *d_rowptr, const int32_t *d_col, int64_t nrows, int64_t ncols, int64_t nnz,
                 int64_t max_row, const char *who, cudaStream_t st) {
  DGP_REQUIRE(d_rowptr && nrows > 0, std::string(who) + ": empty or null CSR row pointer");
  DevBuf err;
  DGP_TRY(err.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  k_rowptr_ok<<<check_grid(nrows), CHECK_NT, 0, st>>>(d_rowptr, nrows, max_row, err.as<int>());
  DGP_CHECK_LAUNCH();
  int h = 0;
  DGP_TRY(read_flag(err, st, &h));
  if (h & 2) return fail(DGP_ERR_MESH, std::string(who) + ": CSR row pointer must start at 0 and not decrease");
  if (h & 4)
    return fail(DGP_ERR_MESH, std::string(who) + ": a CSR row holds more than " + std::to_string(max_row) + " entries");
  int32_t last = 0;
  DGP_CUDA(cudaMemcpyAsync(&last, d_rowptr + nrows, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (nnz >= 0 && last != nnz)
    return fail(DGP_ERR_MESH, std::string(who) + ": CSR row pointer ends at " + std::to_string(last) +
                                  ", not at nnz = " + std::to_string(nnz));
  if (last == 0) return DGP_OK;
  DGP_REQUIRE(d_col, std::string(who) + ": null CSR column array");
  DGP_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  k_ids_in_range<<<check_grid(last), CHECK_NT, 0, st>>>(d_col, last, ncols, err.as<int>());
  DGP_CHECK_LAUNCH();
  DGP_TRY(read_flag(err, st, &h));
  if (h) return fail(DGP_ERR_MESH, std::string(who) + ": CSR column index out of range");
  return DGP_OK;
}

}  // namespace dgp
