// Compliance adjoint and the device solve of the reduced system.
//
// Adjoint. For K(theta) u = f with a load independent of the design and zero
// prescribed values, the compliance c = f^T u has dc/dtheta = -u^T (dK/dtheta) u, and
// u^T K_e u = sum_q s_q sigma_q : eps_q (s = w det J). Per Gauss point, with
// H = sum_k u_k (x) g_k, eps = sym(H), sigma = lam tr(eps) I + 2 mu eps, W = sigma : eps:
//   d/dE_e : u^T K_e u is linear in E (lam, mu proportional to E), so
//            dc/dE_e = -(1/E_e) sum_q s_q W_q;
//   d/dx_m : dg_k/dx_m = -g_m g_k^T (from J^-1 derivative), d(det J)/dx_m = det J g_m,
//            so d(s W)/dx_m = s (W I - 2 H^T sigma) g_m and dc/dx_m = -sum of that.
// The reference obtains the coordinate part by central differences of the assembled
// reduced operator (src/numerics/sensitivity.cpp:77-108); this is its closed form.
//
// Solve. Jacobi-preconditioned conjugate gradients on the CSR K_ff with a warp-per-row
// SpMV and two-stage reductions; the reference's solve_sparse (SciPP spsolve / IC0-CG,
// src/compute/cpu_backend.cpp:24-72) is the CPU counterpart.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "cxg_internal.cuh"

namespace cxg {
namespace {

template <int ET>
__global__ void adjoint_kernel(ElemArgs A, double* dc_dE, double* dc_dX) {
  constexpr int n = nodes_of(ET), nq = gauss_of(ET);
  __shared__ double sdN[n * 3 * nq];
  __shared__ double sw[nq];
  __shared__ double xs[4][3 * n];
  __shared__ double us[4][3 * n];
  for (int i = threadIdx.x; i < n * 3 * nq; i += blockDim.x) sdN[i] = c_dN[dn_offset(ET) + i];
  for (int i = threadIdx.x; i < nq; i += blockDim.x) sw[i] = c_w[ET][i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; e < A.n_elems; e += nwarps) {
    for (int t = lane; t < n; t += 32) {
      const int64_t node = A.conn[e * n + t];
      for (int d = 0; d < 3; ++d) {
        xs[warp][3 * t + d] = A.coords[3 * node + d];
        us[warp][3 * t + d] = A.u[3 * node + d];
      }
    }
    __syncwarp();
    const double E = A.young[e], nu = A.poisson[e];
    const double um2 = E / (1.0 + nu), lam = nu * um2 / (1.0 - 2.0 * nu), mu = um2 / 2.0;
    double sW = 0.0;
    double g[n][3];
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // s (W I - 2 H^T sigma)
    if (lane < nq) {
      const int q = lane;
      double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[i][j] += xs[warp][3 * k + i] * sdN[(3 * k + j) * nq + q];
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      if (!(det > 0.0)) {
        atomicCAS(&A.status->code, 0, 4);
        atomicMin(&A.status->bad_elem, static_cast<unsigned long long>(e));
      }
      const double inv = 1.0 / det;
      const double it[3][3] = {
          {c00 * inv, c01 * inv, c02 * inv},
          {(J[0][2] * J[2][1] - J[0][1] * J[2][2]) * inv, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv,
           (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * inv},
          {(J[0][1] * J[1][2] - J[0][2] * J[1][1]) * inv, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * inv,
           (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv}};
      double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k) {
        for (int i = 0; i < 3; ++i)
          g[k][i] = it[i][0] * sdN[(3 * k) * nq + q] + it[i][1] * sdN[(3 * k + 1) * nq + q] +
                    it[i][2] * sdN[(3 * k + 2) * nq + q];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) H[i][j] += us[warp][3 * k + i] * g[k][j];
      }
      double eps[3][3], sig[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) eps[i][j] = 0.5 * (H[i][j] + H[j][i]);
      const double tr = eps[0][0] + eps[1][1] + eps[2][2];
      double W = 0.0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          sig[i][j] = 2.0 * mu * eps[i][j] + (i == j ? lam * tr : 0.0);
          W += sig[i][j] * eps[i][j];
        }
      const double s = det * sw[q];
      sW = s * W;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double hs = 0.0;  // (H^T sigma)_{ab}
          for (int i = 0; i < 3; ++i) hs += H[i][a] * sig[i][b];
          M[a][b] = s * ((a == b ? W : 0.0) - 2.0 * hs);
        }
    } else {
      for (int k = 0; k < n; ++k) g[k][0] = g[k][1] = g[k][2] = 0.0;
    }
    // element sums over the Gauss points (lanes)
    double tot = sW;
    for (int off = 16; off > 0; off >>= 1) tot += __shfl_down_sync(0xffffffffu, tot, off);
    if (lane == 0 && dc_dE) dc_dE[e] = -tot / E;
    if (dc_dX) {
      for (int k = 0; k < n; ++k) {
        for (int a = 0; a < 3; ++a) {
          double v = M[a][0] * g[k][0] + M[a][1] * g[k][1] + M[a][2] * g[k][2];
          for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
          if (lane == 0) atomicAdd(dc_dX + 3 * static_cast<int64_t>(A.conn[e * n + k]) + a, -v);
        }
      }
    }
    __syncwarp();
  }
}

// y = A x (CSR, one warp per row), optionally also r = b - A x.
__global__ void spmv_kernel(int32_t nrows, const int64_t* rp, const int32_t* ci, const double* v, const double* x,
                            double* y) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < nrows; r += nw) {
    double s = 0.0;
    for (int64_t k = rp[r] + lane; k < rp[r + 1]; k += 32) s += v[k] * x[ci[k]];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) y[r] = s;
  }
}

__global__ void diag_inv_kernel(int32_t nrows, const int64_t* rp, const int32_t* ci, const double* v, double* dinv) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < nrows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double d = 0.0;
    int64_t lo = rp[r], hi = rp[r + 1];
    while (lo < hi) {  // columns are sorted
      const int64_t mid = (lo + hi) >> 1;
      if (ci[mid] < r)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < rp[r + 1] && ci[lo] == r) d = v[lo];
    dinv[r] = d != 0.0 ? 1.0 / d : 1.0;
  }
}

// partial dot products: out[block] = sum a*b over the block's stride
__global__ void dot_kernel(int32_t n, const double* a, const double* b, double* partial) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s += a[i] * b[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

__global__ void finish_dot_kernel(const double* partial, int nparts, double* out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += 32) s += partial[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (threadIdx.x == 0) *out = s;
}

// CG vector updates driven by device scalars (no host round trip per update)
__global__ void cg_update_xr(int32_t n, const double* rz, const double* pAp, double* x, double* r, const double* p,
                             const double* Ap) {
  const double alpha = *pAp != 0.0 ? *rz / *pAp : 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    x[i] += alpha * p[i];
    r[i] -= alpha * Ap[i];
  }
}

__global__ void cg_precond(int32_t n, const double* dinv, const double* r, double* z) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    z[i] = dinv[i] * r[i];
}

__global__ void cg_update_p(int32_t n, const double* rz_new, const double* rz_old, const double* z, double* p) {
  const double beta = *rz_old != 0.0 ? *rz_new / *rz_old : 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

__global__ void residual_kernel(int32_t n, const double* b, const double* Ax, double* r) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    r[i] = b[i] - Ax[i];
}

unsigned g1(int64_t n) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 2048))); }

}  // namespace

cudaError_t launch_adjoint(int t, const ElemArgs& a, double* dc_dE, double* dc_dX, cudaStream_t s) {
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((a.n_elems + 3) / 4, 148 * 16)));
  switch (t) {
    case C3D4: adjoint_kernel<C3D4><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    case C3D10: adjoint_kernel<C3D10><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    case C3D8: adjoint_kernel<C3D8><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    case C3D20: adjoint_kernel<C3D20><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    case C3D20R: adjoint_kernel<C3D20R><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    case C3D6: adjoint_kernel<C3D6><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    case C3D15: adjoint_kernel<C3D15><<<grid, 128, 0, s>>>(a, dc_dE, dc_dX); break;
    default: return cudaErrorNotSupported;
  }
  return cudaGetLastError();
}

cudaError_t launch_spmv(int32_t nrows, const int64_t* rp, const int32_t* ci, const double* v, const double* x, double* y,
                        cudaStream_t s) {
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((nrows + 7) / 8, 148 * 32)));
  spmv_kernel<<<grid, 256, 0, s>>>(nrows, rp, ci, v, x, y);
  return cudaGetLastError();
}

// Jacobi-PCG. work: 5*n + 2048 + 8 doubles. Host reads the residual every 20
// iterations; returns iterations and the final relative residual.
cudaError_t cg_solve(int32_t n, const int64_t* rp, const int32_t* ci, const double* v, const double* b, double* x,
                     double rtol, int max_iter, double* work, int* iters_out, double* rel_out, cudaStream_t s) {
  double* dinv = work + 4 * static_cast<int64_t>(n);
  diag_inv_kernel<<<g1(n), 256, 0, s>>>(n, rp, ci, v, dinv);
  const Preconditioner jacobi = [&](const double* r, double* z) {
    cg_precond<<<g1(n), 256, 0, s>>>(n, dinv, r, z);
    return cudaGetLastError();
  };
  return pcg_solve(n, rp, ci, v, b, x, rtol, max_iter, work, iters_out, rel_out, s, jacobi);
}

// Preconditioned CG with z = M^-1 r from `precond`. work: 5*n + 2048 + 8 doubles (the
// fifth n-vector is left to the preconditioner's owner).
cudaError_t pcg_solve(int32_t n, const int64_t* rp, const int32_t* ci, const double* v, const double* b, double* x,
                      double rtol, int max_iter, double* work, int* iters_out, double* rel_out, cudaStream_t s,
                      const Preconditioner& precond) {
  double* r = work;
  double* z = r + n;
  double* p = z + n;
  double* Ap = p + n;
  double* partial = Ap + 2 * static_cast<int64_t>(n);
  double* sc = partial + 2048;  // rz, rz_new, pAp, bb, rr
  const unsigned gd = g1(n);
  cudaError_t e;
  if ((e = launch_spmv(n, rp, ci, v, x, Ap, s)) != cudaSuccess) return e;
  residual_kernel<<<gd, 256, 0, s>>>(n, b, Ap, r);
  if ((e = precond(r, z)) != cudaSuccess) return e;
  cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
  auto dot = [&](const double* a, const double* c, double* out) {
    dot_kernel<<<gd, 256, 0, s>>>(n, a, c, partial);
    finish_dot_kernel<<<1, 32, 0, s>>>(partial, static_cast<int>(gd), out);
  };
  dot(b, b, sc + 3);
  dot(r, z, sc + 0);
  double hb = 0.0;
  cudaMemcpyAsync(&hb, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  const double bnorm = std::sqrt(hb) > 0.0 ? std::sqrt(hb) : 1.0;
  int it = 0;
  double rel = 1.0;
  for (; it < max_iter; ++it) {
    if ((e = launch_spmv(n, rp, ci, v, p, Ap, s)) != cudaSuccess) return e;
    dot(p, Ap, sc + 2);
    cg_update_xr<<<gd, 256, 0, s>>>(n, sc + 0, sc + 2, x, r, p, Ap);
    if ((e = precond(r, z)) != cudaSuccess) return e;
    dot(r, z, sc + 1);
    cg_update_p<<<gd, 256, 0, s>>>(n, sc + 1, sc + 0, z, p);
    cudaMemcpyAsync(sc + 0, sc + 1, sizeof(double), cudaMemcpyDeviceToDevice, s);
    if ((it + 1) % 20 == 0 || it + 1 == max_iter) {
      dot(r, r, sc + 4);
      double hr = 0.0;
      cudaMemcpyAsync(&hr, sc + 4, sizeof(double), cudaMemcpyDeviceToHost, s);
      if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
      rel = std::sqrt(hr) / bnorm;
      if (rel <= rtol) {
        ++it;
        break;
      }
    }
  }
  if (iters_out) *iters_out = it;
  if (rel_out) *rel_out = rel;
  return cudaGetLastError();
}

}  // namespace cxg
