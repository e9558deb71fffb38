// The compute backend's sparse solve on the device (ComputeBackend::solve_sparse,
// include/calculixpp/compute/backend.hpp:40-57; the CPU backend converts COO to CSR and
// calls a sparse Cholesky / LU or an IC0-preconditioned CG, src/compute/cpu_backend.cpp:
// 24-72). COO triplets come in with duplicates, as the reference's LinearSystem may hold
// them after other scatters; they are sorted by (row, column) on the device (stable, so
// duplicates are summed in input order) and reduced to CSR. The direct kind is a sparse
// Cholesky factorisation on the device (cuSOLVER, symmetric reverse Cuthill-McKee
// reordering); the iterative kinds are CG preconditioned with IC0 (the reference's CG
// kind) or with the diagonal (Jacobi).
// csric02 (zero-fill incomplete Cholesky) is marked deprecated in this toolkit and has no
// generic-API replacement; its deprecation warning is silenced here.
#define DISABLE_CUSPARSE_DEPRECATED
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

// L[k] = A[k], plus alpha * A[k] on the diagonal (one thread per row)
__global__ void shift_copy_kernel(int32_t n, const int32_t* rp, const int32_t* ci, const double* A, double alpha,
                                  double* L) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    for (int32_t k = rp[r]; k < rp[r + 1]; ++k) L[k] = ci[k] == r ? A[k] * (1.0 + alpha) : A[k];
}

// bad = 1 when a row of L has no positive, finite diagonal entry
__global__ void check_diag_kernel(int32_t n, const int32_t* rp, const int32_t* ci, const double* L, int* bad) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int32_t lo = rp[r], hi = rp[r + 1];
    while (lo < hi) {  // columns are sorted
      const int32_t mid = (lo + hi) >> 1;
      if (ci[mid] < r) lo = mid + 1; else hi = mid;
    }
    const double d = lo < rp[r + 1] && ci[lo] == r ? L[lo] : 0.0;
    if (!(d > 0.0) || !(d < INFINITY)) atomicExch(bad, 1);
  }
}

// IC0 preconditioner, the one the reference's CG kind uses (SciPP cg_report with
// Preconditioner::IC0, src/compute/cpu_backend.cpp:52-63): A ~ L L^T with L on the lower
// triangle of A's pattern, no fill (cuSPARSE csric02), applied as two triangular solves
// (cusparseSpSV with L, then L^T). The incomplete factor of an SPD matrix can meet a
// non-positive pivot; the factorisation is then retried on A + alpha diag(A) for
// alpha = 1e-4, 1e-3, 1e-2, 1e-1 (a diagonal shift), and fails past that.
struct Ic0 {
  cusparseHandle_t h = nullptr;
  cusparseMatDescr_t descr = nullptr;
  csric02Info_t info = nullptr;
  cusparseSpMatDescr_t mat = nullptr;
  cusparseDnVecDescr_t vr = nullptr, vy = nullptr, vz = nullptr;
  cusparseSpSVDescr_t sl = nullptr, slt = nullptr;
  double* L = nullptr;
  double* y = nullptr;
  void* buf = nullptr;
  void* bl = nullptr;
  void* blt = nullptr;
  int* bad = nullptr;
  double alpha = 0.0;
  cudaStream_t s = nullptr;
  ~Ic0() {
    if (sl) cusparseSpSV_destroyDescr(sl);
    if (slt) cusparseSpSV_destroyDescr(slt);
    if (vr) cusparseDestroyDnVec(vr);
    if (vy) cusparseDestroyDnVec(vy);
    if (vz) cusparseDestroyDnVec(vz);
    if (mat) cusparseDestroySpMat(mat);
    if (info) cusparseDestroyCsric02Info(info);
    if (descr) cusparseDestroyMatDescr(descr);
    if (h) cusparseDestroy(h);
    for (void* q : {static_cast<void*>(L), static_cast<void*>(y), buf, bl, blt, static_cast<void*>(bad)}) cudaFree(q);
  }
};

#define IC0_SP(call, what)                                                                              \
  do {                                                                                                  \
    const cusparseStatus_t st_ = (call);                                                                \
    if (st_ != CUSPARSE_STATUS_SUCCESS)                                                                 \
      return set_err(CXG_ERR_CUDA, std::string("IC0 ") + (what) + ": " + cusparseGetErrorString(st_)); \
  } while (0)

// Factor (with the shift retries) and set up the two triangular solves; r and z are the
// CG loop's residual and preconditioned-residual vectors.
int ic0_build(Ic0& P, int32_t n, int32_t nnz, const int32_t* rp, const int32_t* ci, const double* A, double* r,
              double* z, cudaStream_t s) {
  P.s = s;
  CHECK_CUDA(cudaMalloc(&P.L, sizeof(double) * std::max<int32_t>(nnz, 1)), "IC0 factor");
  CHECK_CUDA(cudaMalloc(&P.y, sizeof(double) * std::max<int32_t>(n, 1)), "IC0 vector");
  CHECK_CUDA(cudaMalloc(&P.bad, sizeof(int)), "IC0 flag");
  IC0_SP(cusparseCreate(&P.h), "handle");
  IC0_SP(cusparseSetStream(P.h, s), "stream");
  IC0_SP(cusparseCreateMatDescr(&P.descr), "descriptor");
  cusparseSetMatType(P.descr, CUSPARSE_MATRIX_TYPE_GENERAL);
  cusparseSetMatIndexBase(P.descr, CUSPARSE_INDEX_BASE_ZERO);
  IC0_SP(cusparseCreateCsric02Info(&P.info), "info");
  int bytes = 0;
  IC0_SP(cusparseDcsric02_bufferSize(P.h, n, nnz, P.descr, P.L, rp, ci, P.info, &bytes), "buffer size");
  CHECK_CUDA(cudaMalloc(&P.buf, std::max(bytes, 16)), "IC0 buffer");
  IC0_SP(cusparseDcsric02_analysis(P.h, n, nnz, P.descr, P.L, rp, ci, P.info, CUSPARSE_SOLVE_POLICY_USE_LEVEL, P.buf),
         "analysis");
  int pos = -1;
  if (cusparseXcsric02_zeroPivot(P.h, P.info, &pos) == CUSPARSE_STATUS_ZERO_PIVOT)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "IC0: row " + std::to_string(pos) + " has no diagonal entry");
  const double shifts[] = {0.0, 1e-4, 1e-3, 1e-2, 1e-1};
  bool ok = false;
  for (double alpha : shifts) {
    shift_copy_kernel<<<gsz(n), 256, 0, s>>>(n, rp, ci, A, alpha, P.L);
    CHECK_CUDA(cudaGetLastError(), "IC0 copy");
    IC0_SP(cusparseDcsric02(P.h, n, nnz, P.descr, P.L, rp, ci, P.info, CUSPARSE_SOLVE_POLICY_USE_LEVEL, P.buf),
           "factorisation");
    const bool zero = cusparseXcsric02_zeroPivot(P.h, P.info, &pos) == CUSPARSE_STATUS_ZERO_PIVOT;
    int hbad = 0;
    CHECK_CUDA(cudaMemsetAsync(P.bad, 0, sizeof(int), s), "IC0 flag");
    check_diag_kernel<<<gsz(n), 256, 0, s>>>(n, rp, ci, P.L, P.bad);
    CHECK_CUDA(cudaMemcpyAsync(&hbad, P.bad, sizeof(int), cudaMemcpyDeviceToHost, s), "IC0 flag");
    CHECK_CUDA(cudaStreamSynchronize(s), "IC0 factorisation");
    if (!zero && !hbad) {
      P.alpha = alpha;
      ok = true;
      break;
    }
  }
  if (!ok) return set_err(CXG_ERR_NOT_CONVERGED, "IC0 factorisation broke down up to a diagonal shift of 0.1");
  IC0_SP(cusparseCreateCsr(&P.mat, n, n, nnz, const_cast<int32_t*>(rp), const_cast<int32_t*>(ci), P.L,
                           CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F),
         "matrix");
  cusparseFillMode_t fill = CUSPARSE_FILL_MODE_LOWER;
  cusparseDiagType_t diag = CUSPARSE_DIAG_TYPE_NON_UNIT;
  IC0_SP(cusparseSpMatSetAttribute(P.mat, CUSPARSE_SPMAT_FILL_MODE, &fill, sizeof(fill)), "fill mode");
  IC0_SP(cusparseSpMatSetAttribute(P.mat, CUSPARSE_SPMAT_DIAG_TYPE, &diag, sizeof(diag)), "diagonal type");
  IC0_SP(cusparseCreateDnVec(&P.vr, n, r, CUDA_R_64F), "vector");
  IC0_SP(cusparseCreateDnVec(&P.vy, n, P.y, CUDA_R_64F), "vector");
  IC0_SP(cusparseCreateDnVec(&P.vz, n, z, CUDA_R_64F), "vector");
  IC0_SP(cusparseSpSV_createDescr(&P.sl), "solve descriptor");
  IC0_SP(cusparseSpSV_createDescr(&P.slt), "solve descriptor");
  const double one = 1.0;
  size_t b1 = 0, b2 = 0;
  IC0_SP(cusparseSpSV_bufferSize(P.h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, P.mat, P.vr, P.vy, CUDA_R_64F,
                                 CUSPARSE_SPSV_ALG_DEFAULT, P.sl, &b1),
         "solve buffer");
  IC0_SP(cusparseSpSV_bufferSize(P.h, CUSPARSE_OPERATION_TRANSPOSE, &one, P.mat, P.vy, P.vz, CUDA_R_64F,
                                 CUSPARSE_SPSV_ALG_DEFAULT, P.slt, &b2),
         "solve buffer");
  CHECK_CUDA(cudaMalloc(&P.bl, std::max<size_t>(b1, 16)), "IC0 solve buffer");
  CHECK_CUDA(cudaMalloc(&P.blt, std::max<size_t>(b2, 16)), "IC0 solve buffer");
  IC0_SP(cusparseSpSV_analysis(P.h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, P.mat, P.vr, P.vy, CUDA_R_64F,
                               CUSPARSE_SPSV_ALG_DEFAULT, P.sl, P.bl),
         "solve analysis");
  IC0_SP(cusparseSpSV_analysis(P.h, CUSPARSE_OPERATION_TRANSPOSE, &one, P.mat, P.vy, P.vz, CUDA_R_64F,
                               CUSPARSE_SPSV_ALG_DEFAULT, P.slt, P.blt),
         "solve analysis");
  return CXG_OK;
}

// z = (L L^T)^-1 r
cudaError_t ic0_apply(Ic0& P, const double* r, double* z) {
  const double one = 1.0;
  if (cusparseDnVecSetValues(P.vr, const_cast<double*>(r)) != CUSPARSE_STATUS_SUCCESS ||
      cusparseDnVecSetValues(P.vz, z) != CUSPARSE_STATUS_SUCCESS ||
      cusparseSpSV_solve(P.h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, P.mat, P.vr, P.vy, CUDA_R_64F,
                         CUSPARSE_SPSV_ALG_DEFAULT, P.sl) != CUSPARSE_STATUS_SUCCESS ||
      cusparseSpSV_solve(P.h, CUSPARSE_OPERATION_TRANSPOSE, &one, P.mat, P.vy, P.vz, CUDA_R_64F,
                         CUSPARSE_SPSV_ALG_DEFAULT, P.slt) != CUSPARSE_STATUS_SUCCESS)
    return cudaErrorUnknown;
  return cudaGetLastError();
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
      (solver != CXG_SOLVER_DIRECT && solver != CXG_SOLVER_CG && solver != CXG_SOLVER_IC0_CG))
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
  } else if (solver == CXG_SOLVER_IC0_CG) {
    double* work = nullptr;
    e = sc.alloc(reinterpret_cast<void**>(&work), sizeof(double) * (5 * static_cast<size_t>(n) + 2056));
    if (e != cudaSuccess) {
      cudaStreamDestroy(s);
      return cuda_err(e, "cg work");
    }
    int rc = CXG_OK;
    {
      Ic0 P;
      rc = ic0_build(P, n, static_cast<int32_t>(nu), row_ptr32, col, vsum, work, work + n, s);
      if (rc == CXG_OK) {
        const Preconditioner ic0 = [&](const double* r, double* z) { return ic0_apply(P, r, z); };
        e = pcg_solve(n, row_ptr64, col, vsum, d_rhs, d_x, rtol, max_iter, work, &it, &rel, s, ic0);
        if (e != cudaSuccess) rc = cuda_err(e, "IC0-preconditioned cg");
      }
    }
    if (rc != CXG_OK) {
      cudaStreamDestroy(s);
      return rc;
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
  if (solver != CXG_SOLVER_DIRECT && !(rel <= rtol)) {
    char buf[160];
    snprintf(buf, sizeof buf, "CG did not converge (relative residual %.3e after %d iterations)", rel, it);
    return set_err(CXG_ERR_NOT_CONVERGED, buf);
  }
  return CXG_OK;
}
