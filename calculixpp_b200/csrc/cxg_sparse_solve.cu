// The compute backend's sparse solve on the device (ComputeBackend::solve_sparse,
// include/calculixpp/compute/backend.hpp:40-57; the CPU backend converts COO to CSR and
// calls a sparse Cholesky / LU or an IC0-preconditioned CG, src/compute/cpu_backend.cpp:
// 24-72). COO triplets come in with duplicates, as the reference's LinearSystem may hold
// them after other scatters; they are sorted by (row, column) on the device (stable, so
// duplicates are summed in input order) and reduced to CSR. The direct kind is a sparse
// Cholesky factorisation on the device (cuSOLVER, symmetric reverse Cuthill-McKee
// reordering); the iterative kind is this library's Jacobi-preconditioned CG.
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <cusolverSp.h>
#include <cusparse.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/cxg.h"
#include "cxg_plan.hpp"

using namespace cxg;
using namespace cxg::api;

namespace {

unsigned gsz(int64_t n) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32))); }

__global__ void coo_keys_kernel(const int32_t* rows, const int32_t* cols, int64_t nnz, int64_t n, uint64_t* key,
                                int* bad) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nnz;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t r = rows[i], c = cols[i];
    if (r < 0 || r >= n || c < 0 || c >= n) {
      atomicExch(bad, 1);
      key[i] = 0;
    } else {
      key[i] = static_cast<uint64_t>(r) * static_cast<uint64_t>(n) + static_cast<uint64_t>(c);
    }
  }
}

__global__ void csr_from_keys_kernel(const uint64_t* ukey, int64_t nu, int64_t n, int64_t* row_ptr64, int32_t* row_ptr32,
                                     int32_t* col) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r <= n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t lo = static_cast<uint64_t>(r) * static_cast<uint64_t>(n);
    int64_t a = 0, b = nu;
    while (a < b) {
      const int64_t m = (a + b) / 2;
      if (ukey[m] < lo) a = m + 1; else b = m;
    }
    row_ptr64[r] = a;
    row_ptr32[r] = static_cast<int32_t>(a);
  }
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nu;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    col[i] = static_cast<int32_t>(ukey[i] % static_cast<uint64_t>(n));
}

// RAII list of device allocations of one call
struct Scratch {
  std::vector<void*> p;
  cudaError_t alloc(void** q, size_t bytes) {
    const cudaError_t e = cudaMalloc(q, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) p.push_back(*q);
    return e;
  }
  ~Scratch() {
    for (void* q : p) cudaFree(q);
  }
};

}  // namespace

extern "C" int cxg_solve_sparse(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols, const double* vals,
                                const double* rhs, double* x, int32_t solver, double rtol, int32_t max_iter,
                                int32_t* iterations, double* rel_residual) {
  if (n < 0 || nnz < 0 || !x || (n > 0 && !rhs) || (nnz > 0 && (!rows || !cols || !vals)) ||
      (solver != CXG_SOLVER_DIRECT && solver != CXG_SOLVER_CG))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  if (nnz > INT32_MAX) return set_err(CXG_ERR_UNSUPPORTED, "more than 2^31-1 triplets");
  if (iterations) *iterations = 0;
  if (rel_residual) *rel_residual = 0.0;
  if (n == 0) return CXG_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(CXG_ERR_NO_GPU, "no CUDA device");
  }
  cudaStream_t s = nullptr;
  CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  Scratch sc;
  int32_t *d_rows, *d_cols, *row_ptr32, *col;
  double *d_vals, *d_rhs, *d_x, *vsum, *vs2;
  uint64_t *key, *key2, *ukey;
  int64_t *row_ptr64, *n_u_d;
  int* bad;
  cudaError_t e = sc.alloc(reinterpret_cast<void**>(&d_rows), 4 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&d_cols), 4 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&d_vals), 8 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&d_rhs), 8 * static_cast<size_t>(n));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&d_x), 8 * static_cast<size_t>(n));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&key), 8 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&key2), 8 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&ukey), 8 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&vs2), 8 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&vsum), 8 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&row_ptr64), 8 * (static_cast<size_t>(n) + 1));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&row_ptr32), 4 * (static_cast<size_t>(n) + 1));
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&col), 4 * nnz);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&n_u_d), 8);
  if (e == cudaSuccess) e = sc.alloc(reinterpret_cast<void**>(&bad), sizeof(int));
  if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_rows, rows, 4 * nnz, cudaMemcpyDefault, s);
  if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_cols, cols, 4 * nnz, cudaMemcpyDefault, s);
  if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_vals, vals, 8 * nnz, cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_rhs, rhs, 8 * static_cast<size_t>(n), cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_x, 0, 8 * static_cast<size_t>(n), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), s);
  if (e == cudaSuccess && nnz) {
    coo_keys_kernel<<<gsz(nnz), 256, 0, s>>>(d_rows, d_cols, nnz, n, key, bad);
    e = cudaGetLastError();
  }
  int end_bit = 1;
  while (end_bit < 64 && ((static_cast<uint64_t>(n) * static_cast<uint64_t>(n)) >> end_bit) != 0) ++end_bit;
  size_t tb = 0, tb2 = 0;
  void* temp = nullptr;
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, d_vals, vs2, nnz, 0, end_bit, s);
  if (e == cudaSuccess)
    e = cub::DeviceReduce::ReduceByKey(nullptr, tb2, key2, ukey, vs2, vsum, n_u_d, cub::Sum(), nnz, s);
  if (e == cudaSuccess) e = sc.alloc(&temp, std::max(tb, tb2));
  tb = tb2 = std::max(tb, tb2);
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, tb, key, key2, d_vals, vs2, nnz, 0, end_bit, s);
  if (e == cudaSuccess)
    e = cub::DeviceReduce::ReduceByKey(temp, tb2, key2, ukey, vs2, vsum, n_u_d, cub::Sum(), nnz, s);
  int64_t nu = 0;
  int hbad = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nu, n_u_d, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && hbad) {
    cudaStreamDestroy(s);
    return set_err(CXG_ERR_INVALID_ARGUMENT, "COO index outside [0, n)");
  }
  if (e == cudaSuccess) {
    csr_from_keys_kernel<<<gsz(static_cast<int64_t>(n) + 1), 256, 0, s>>>(ukey, nu, n, row_ptr64, row_ptr32, col);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaStreamDestroy(s);
    return cuda_err(e, "COO to CSR");
  }
  int it = 0;
  double rel = 0.0;
  if (solver == CXG_SOLVER_DIRECT) {
    cusolverSpHandle_t h = nullptr;
    cusparseMatDescr_t d = nullptr;
    int singular = -1;
    cusolverStatus_t st = cusolverSpCreate(&h);
    if (st == CUSOLVER_STATUS_SUCCESS) st = cusolverSpSetStream(h, s);
    if (st == CUSOLVER_STATUS_SUCCESS && cusparseCreateMatDescr(&d) != CUSPARSE_STATUS_SUCCESS)
      st = CUSOLVER_STATUS_ALLOC_FAILED;
    if (d) {
      cusparseSetMatType(d, CUSPARSE_MATRIX_TYPE_GENERAL);
      cusparseSetMatIndexBase(d, CUSPARSE_INDEX_BASE_ZERO);
    }
    if (st == CUSOLVER_STATUS_SUCCESS)
      st = cusolverSpDcsrlsvchol(h, n, static_cast<int>(nu), d, vsum, row_ptr32, col, d_rhs, 0.0, 1, d_x, &singular);
    if (d) cusparseDestroyMatDescr(d);
    if (h) cusolverSpDestroy(h);
    if (st != CUSOLVER_STATUS_SUCCESS) {
      cudaStreamDestroy(s);
      return set_err(CXG_ERR_CUDA, "sparse Cholesky failed (status " + std::to_string(static_cast<int>(st)) + ")");
    }
    if (singular >= 0) {
      cudaStreamDestroy(s);
      return set_err(CXG_ERR_NOT_CONVERGED, "matrix is not positive definite (pivot " + std::to_string(singular) + ")");
    }
  } else {
    double* work = nullptr;
    e = sc.alloc(reinterpret_cast<void**>(&work), sizeof(double) * (5 * static_cast<size_t>(n) + 2056));
    if (e == cudaSuccess) e = cg_solve(n, row_ptr64, col, vsum, d_rhs, d_x, rtol, max_iter, work, &it, &rel, s);
    if (e != cudaSuccess) {
      cudaStreamDestroy(s);
      return cuda_err(e, "cg");
    }
  }
  e = cudaMemcpyAsync(x, d_x, 8 * static_cast<size_t>(n), cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  CHECK_CUDA(e, "solution copy");
  if (iterations) *iterations = it;
  if (rel_residual) *rel_residual = rel;
  if (solver == CXG_SOLVER_CG && !(rel <= rtol)) {
    char buf[160];
    snprintf(buf, sizeof buf, "CG did not converge (relative residual %.3e after %d iterations)", rel, it);
    return set_err(CXG_ERR_NOT_CONVERGED, buf);
  }
  return CXG_OK;
}
