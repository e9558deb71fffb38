// The reference's own sparsity pattern for the linear-static operator.
//
// The reference scatters K_e into its hash map one DOF pair at a time and skips every
// value that is exactly 0.0 (src/fem/assembly.cpp:86-90), so an entry of K_ff exists in its
// LinearSystem only when at least one element contributes a nonzero value to it in the
// reference's own FP64 arithmetic. Exact zeros come from geometry (straight, axis-aligned
// elements give exactly vanishing gradient components and exactly cancelling sums), so
// deciding them needs K_e evaluated in the reference's operation order:
//   * Gauss points and weights           src/fem/element.cpp:10-77
//   * shape-function derivatives         element.cpp:160-359 (the same formulas)
//   * J, det J, J^-T and gradients       element.cpp:80-102, 361-380 (same loop order)
//   * isotropic D                        element.cpp:410-422
//   * DB per column, then Ke[a][b] += scale * (B^T DB) for b >= a, Gauss point by Gauss
//     point                              element.cpp:440-462
//   * C3D8R hourglass, added after the Gauss loop   element.cpp:529-610
// This file is compiled with -fmad=false: no multiply-add contraction, and CUDA's default
// FP64 division is correctly rounded, so every operation here rounds exactly as the
// reference's x86 build does and the zero / nonzero decision is the reference's.
//
// refmask_kernel writes, in the FP64 element-buffer layout of the row gather (upper 3x3
// blocks padded to 10 doubles), 1.0 where the reference's K_e value is nonzero and 0.0
// where it is exactly zero. The ordinary FP64 row gather then sums these flags per CSR
// entry: an entry is kept when the count is positive.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "cxg_internal.cuh"

namespace cxg {
namespace {

constexpr int kRefWarps = 4;

__device__ __forceinline__ double sgn(int s) { return s < 0 ? -1.0 : 1.0; }

__constant__ int c_hex_sign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                     {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
__constant__ int c_mid_hex[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                     {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
__constant__ int c_edge_axis[12] = {0, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2};
__constant__ double c_hg_gamma[4][8] = {{1, 1, -1, -1, -1, -1, 1, 1},
                                        {1, -1, -1, 1, -1, 1, 1, -1},
                                        {1, -1, 1, -1, 1, -1, 1, -1},
                                        {-1, 1, -1, 1, 1, -1, 1, -1}};

// Gauss point q of the family (xi, et, ze, w), as the reference's rule tables hold them.
template <int ET>
__device__ void ref_gauss(int q, double* p) {
  constexpr double kG2 = 0.577350269189625764, kG3 = 0.774596669241483377;
  if constexpr (ET == C3D8 || ET == C3D20R) {
    p[0] = (q & 1) ? kG2 : -kG2;
    p[1] = (q & 2) ? kG2 : -kG2;
    p[2] = (q & 4) ? kG2 : -kG2;
    p[3] = 1.0;
  } else if constexpr (ET == C3D8R) {
    p[0] = p[1] = p[2] = 0.0;
    p[3] = 8.0;
  } else if constexpr (ET == C3D20) {
    const double nodes[3] = {-kG3, 0.0, kG3};
    const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    const int a = q % 3, b = (q / 3) % 3, c = q / 9;
    p[0] = nodes[a];
    p[1] = nodes[b];
    p[2] = nodes[c];
    p[3] = wts[a] * wts[b] * wts[c];
  } else if constexpr (ET == C3D6) {
    p[0] = p[1] = 1.0 / 3.0;
    p[2] = q ? kG2 : -kG2;
    p[3] = 0.5;
  } else if constexpr (ET == C3D15) {
    const double kT = 1.0 / 6.0, kU = 2.0 / 3.0;
    const int t = q % 3;
    p[0] = t == 1 ? kU : kT;
    p[1] = t == 2 ? kU : kT;
    p[2] = q < 3 ? -kG2 : kG2;
    p[3] = kT;
  } else if constexpr (ET == C3D4) {
    p[0] = p[1] = p[2] = 0.25;
    p[3] = 1.0 / 6.0;
  } else {  // C3D10
    constexpr double kA = 0.138196601125010515, kB = 0.585410196624968454;
    p[0] = q == 1 ? kB : kA;
    p[1] = q == 2 ? kB : kA;
    p[2] = q == 3 ? kB : kA;
    p[3] = 1.0 / 24.0;
  }
}

// Natural derivatives dN[3k + d] of the family at (xi, et, ze), by the reference's formulas.
template <int ET>
__device__ void ref_dshape(double xi, double et, double ze, double* dN) {
  if constexpr (ET == C3D8 || ET == C3D8R) {
    for (int k = 0; k < 8; ++k) {
      const double sg = sgn(c_hex_sign[k][0]), sh = sgn(c_hex_sign[k][1]), sr = sgn(c_hex_sign[k][2]);
      const double g = 1.0 + sg * xi, h = 1.0 + sh * et, r = 1.0 + sr * ze;
      dN[3 * k + 0] = sg * h * r / 8.0;
      dN[3 * k + 1] = sh * g * r / 8.0;
      dN[3 * k + 2] = sr * g * h / 8.0;
    }
  } else if constexpr (ET == C3D20 || ET == C3D20R) {
    const double p[3] = {xi, et, ze};
    for (int k = 0; k < 8; ++k) {
      const double s[3] = {sgn(c_hex_sign[k][0]), sgn(c_hex_sign[k][1]), sgn(c_hex_sign[k][2])};
      const double g = 1.0 + s[0] * xi, h = 1.0 + s[1] * et, r = 1.0 + s[2] * ze;
      const double q = s[0] * xi + s[1] * et + s[2] * ze - 2.0;
      const double fac[3] = {g, h, r};
      for (int d = 0; d < 3; ++d) {
        double others = 1.0;
        for (int m = 0; m < 3; ++m)
          if (m != d) others *= fac[m];
        dN[3 * k + d] = (s[d] * others * q + g * h * r * s[d]) / 8.0;
      }
    }
    for (int j = 0; j < 12; ++j) {
      const int node = 8 + j, a = c_edge_axis[j], c0 = c_mid_hex[j][0];
      const double s[3] = {sgn(c_hex_sign[c0][0]), sgn(c_hex_sign[c0][1]), sgn(c_hex_sign[c0][2])};
      const double pa = p[a];
      double plane = 1.0;
      for (int m = 0; m < 3; ++m)
        if (m != a) plane *= 1.0 + s[m] * p[m];
      for (int d = 0; d < 3; ++d) {
        if (d == a) {
          dN[3 * node + d] = (-2.0 * pa) * plane / 4.0;
        } else {
          double other = 1.0;
          for (int m = 0; m < 3; ++m)
            if (m != a && m != d) other *= 1.0 + s[m] * p[m];
          dN[3 * node + d] = (1.0 - pa * pa) * s[d] * other / 4.0;
        }
      }
    }
  } else if constexpr (ET == C3D6) {
    const double a = 1.0 - xi - et;
    const double m = 0.5 * (1.0 - ze), p = 0.5 * (1.0 + ze);
    const double d6[18] = {-m, -m, -0.5 * a, m, 0.0, -0.5 * xi, 0.0, m, -0.5 * et,
                           -p, -p, 0.5 * a,  p, 0.0, 0.5 * xi,  0.0, p, 0.5 * et};
    for (int i = 0; i < 18; ++i) dN[i] = d6[i];
  } else if constexpr (ET == C3D15) {
    const double a = 1.0 - xi - et;
    const double omz = 1.0 - ze, opz = 1.0 + ze, omz2 = 1.0 - ze * ze;
    const double dxi[15] = {0.5 * omz * (4 * xi + 4 * et + ze - 2), 0.5 * omz * (4 * xi - ze - 2), 0.0,
                            0.5 * opz * (4 * xi + 4 * et - ze - 2), 0.5 * opz * (4 * xi + ze - 2), 0.0,
                            2 * omz * (1 - 2 * xi - et),            2 * et * omz,                  -2 * et * omz,
                            2 * opz * (1 - 2 * xi - et),            2 * et * opz,                  -2 * et * opz,
                            -omz2,                                  omz2,                          0.0};
    const double det[15] = {0.5 * omz * (4 * xi + 4 * et + ze - 2), 0.0, 0.5 * omz * (4 * et - ze - 2),
                            0.5 * opz * (4 * xi + 4 * et - ze - 2), 0.0, 0.5 * opz * (4 * et + ze - 2),
                            -2 * xi * omz,                          2 * xi * omz, 2 * omz * (1 - xi - 2 * et),
                            -2 * xi * opz,                          2 * xi * opz, 2 * opz * (1 - xi - 2 * et),
                            -omz2,                                  0.0,          omz2};
    const double dz[15] = {-0.5 * a * (-1.0 * (2 * xi + 2 * et + ze) + omz * 1.0),
                           0.5 * xi * (-1.0 * (2 * xi - 2 - ze) + omz * (-1.0)),
                           0.5 * et * (-1.0 * (2 * et - 2 - ze) + omz * (-1.0)),
                           -0.5 * a * (1.0 * (2 * xi + 2 * et - ze) + opz * (-1.0)),
                           0.5 * xi * (1.0 * (2 * xi - 2 + ze) + opz * (1.0)),
                           0.5 * et * (1.0 * (2 * et - 2 + ze) + opz * (1.0)),
                           -2 * xi * a,
                           -2 * xi * et,
                           -2 * et * a,
                           2 * xi * a,
                           2 * xi * et,
                           2 * et * a,
                           a * (-2 * ze),
                           xi * (-2 * ze),
                           et * (-2 * ze)};
    for (int k = 0; k < 15; ++k) {
      dN[3 * k] = dxi[k];
      dN[3 * k + 1] = det[k];
      dN[3 * k + 2] = dz[k];
    }
  } else if constexpr (ET == C3D4) {
    const double d[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int i = 0; i < 12; ++i) dN[i] = d[i];
  } else {  // C3D10
    const double a = 1.0 - xi - et - ze;
    const double d[30] = {1 - 4 * a, 1 - 4 * a, 1 - 4 * a, 4 * xi - 1, 0, 0, 0, 4 * et - 1, 0, 0, 0, 4 * ze - 1,
                          4 * (a - xi), -4 * xi, -4 * xi, 4 * et, 4 * xi, 0, -4 * et, 4 * (a - et), -4 * et,
                          -4 * ze, -4 * ze, 4 * (a - ze), 4 * ze, 0, 4 * xi, 0, 4 * ze, 4 * et};
    for (int i = 0; i < 30; ++i) dN[i] = d[i];
  }
}

// Physical gradients g[3k + i] and det J, in the reference's loop order.
__device__ double ref_gradients(int n, const double* dN, const double* x, double* g) {
  double J[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < n; ++k) v += x[3 * k + i] * dN[3 * k + j];
      J[i][j] = v;
    }
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double inv = 1.0 / det;
  const double Jinv[3][3] = {
      {c00 * inv, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * inv, (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * inv},
      {c01 * inv, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * inv},
      {c02 * inv, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * inv, (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv}};
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < 3; ++i) {
      double v = 0.0;
      for (int j = 0; j < 3; ++j) v += Jinv[j][i] * dN[3 * k + j];
      g[3 * k + i] = v;
    }
  return det;
}

__device__ __forceinline__ double b_entry(int row, const double* gk, int dir) {
  const double gx = gk[0], gy = gk[1], gz = gk[2];
  switch (row) {
    case 0: return dir == 0 ? gx : 0.0;
    case 1: return dir == 1 ? gy : 0.0;
    case 2: return dir == 2 ? gz : 0.0;
    case 3: return dir == 0 ? gy : (dir == 1 ? gx : 0.0);
    case 4: return dir == 0 ? gz : (dir == 2 ? gx : 0.0);
    default: return dir == 1 ? gz : (dir == 2 ? gy : 0.0);
  }
}

template <int ET>
struct RefWarp {
  static constexpr int n = nodes_of(ET), nq = gauss_of(ET);
  double x[3 * n];
  double g[nq][3 * n];
  double scale[nq];
  double gamma[4][8];
  double kappa;
};

template <int ET>
__global__ void __launch_bounds__(kRefWarps * 32) refmask_kernel(ElemArgs A, double* out) {
  constexpr int n = nodes_of(ET), nq = gauss_of(ET), NB = n * (n + 1) / 2, BS = 10;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RefWarp<ET>& W = reinterpret_cast<RefWarp<ET>*>(smem)[warp];
  const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kRefWarps + warp;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kRefWarps;
  for (int64_t e = gwarp; e < A.n_elems; e += nwarps) {
    for (int t = lane; t < 3 * n; t += 32) W.x[t] = A.coords[3 * static_cast<int64_t>(A.conn[e * n + t / 3]) + t % 3];
    __syncwarp();
    if (lane < nq) {
      double p[4], dN[3 * n];
      ref_gauss<ET>(lane, p);
      ref_dshape<ET>(p[0], p[1], p[2], dN);
      const double det = ref_gradients(n, dN, W.x, W.g[lane]);
      W.scale[lane] = det * p[3];
    }
    // elastic_D (element.cpp:410-422)
    const double E = A.young[e], nu = A.poisson[e];
    const double um2 = E / (1.0 + nu);
    const double lam = nu * um2 / (1.0 - 2.0 * nu);
    const double mu = um2 / 2.0;
    const double lam2mu = lam + um2;
    if constexpr (ET == C3D8R) {
      // build_hourglass (element.cpp:545-579)
      if (lane == 0) {
        double dN[24], b[24];
        ref_dshape<C3D8>(0.0, 0.0, 0.0, dN);
        const double det = ref_gradients(8, dN, W.x, b);
        const double vol = 8.0 * det;
        for (int al = 0; al < 4; ++al) {
          double gx[3] = {0, 0, 0};
          for (int j = 0; j < 8; ++j)
            for (int d = 0; d < 3; ++d) gx[d] += c_hg_gamma[al][j] * W.x[3 * j + d];
          for (int j = 0; j < 8; ++j) {
            double corr = 0.0;
            for (int d = 0; d < 3; ++d) corr += gx[d] * b[3 * j + d];
            W.gamma[al][j] = c_hg_gamma[al][j] - corr;
          }
        }
        double b2 = 0.0;
        for (int j = 0; j < 8; ++j)
          for (int d = 0; d < 3; ++d) b2 += b[3 * j + d] * b[3 * j + d];
        const double mu_hg = E / (2.0 * (1.0 + nu));
        W.kappa = 0.05 * mu_hg * vol * b2;
      }
    }
    __syncwarp();
    double* dst = out + e * (NB * BS);
    for (int t = lane; t < NB * 9; t += 32) {
      const int blk = t / 9, q9 = t % 9;
      int ka = 0, r = blk;
      while (r >= n - ka) {
        r -= n - ka;
        ++ka;
      }
      const int kb = ka + r;
      int A0 = 3 * ka + q9 / 3, B0 = 3 * kb + q9 % 3;
      if (A0 > B0) {  // lower half of a diagonal block: the mirrored upper value
        const int tmp = A0;
        A0 = B0;
        B0 = tmp;
      }
      const int na = A0 / 3, da = A0 % 3, nb = B0 / 3, db = B0 % 3;
      double K = 0.0;
      for (int q = 0; q < nq; ++q) {
        const double* ga = W.g[q] + 3 * na;
        const double* gb = W.g[q] + 3 * nb;
        double DBa[6];
        for (int row = 0; row < 6; ++row) {
          double v = 0.0;
          for (int c = 0; c < 6; ++c) {
            const double Drc = row < 3 ? (c < 3 ? (c == row ? lam2mu : lam) : 0.0) : (c == row ? mu : 0.0);
            v += Drc * b_entry(c, ga, da);
          }
          DBa[row] = v;
        }
        double v = 0.0;
        for (int row = 0; row < 6; ++row) v += b_entry(row, gb, db) * DBa[row];
        K += W.scale[q] * v;
      }
      if constexpr (ET == C3D8R) {  // accumulate_hourglass (element.cpp:581-592)
        if (da == db)
          for (int al = 0; al < 4; ++al) K += W.kappa * W.gamma[al][na] * W.gamma[al][nb];
      }
      dst[blk * BS + q9] = K != 0.0 ? 1.0 : 0.0;
    }
    __syncwarp();
  }
}

template <int ET>
cudaError_t launch_refmask_t(const ElemArgs& a, double* out, cudaStream_t s) {
  if (a.n_elems == 0) return cudaSuccess;
  auto kern = refmask_kernel<ET>;
  const size_t smem = sizeof(RefWarp<ET>) * kRefWarps;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  const int64_t grid = std::min<int64_t>((a.n_elems + kRefWarps - 1) / kRefWarps, 148 * 16);
  kern<<<static_cast<unsigned>(grid), kRefWarps * 32, smem, s>>>(a, out);
  return cudaGetLastError();
}

// keep[i] = 1 when at least one element contributes a nonzero value to CSR entry i
__global__ void keep_kernel(const double* counts, uint8_t* keep, int64_t nnz) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nnz;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    keep[i] = counts[i] != 0.0 ? 1 : 0;
}

__global__ void row_len_kernel(const int64_t* row_ptr, const uint8_t* keep, int32_t n_rows, int64_t* row_len) {
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n_rows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t c = 0;
    for (int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) c += keep[k];
    row_len[r] = c;
  }
}

__global__ void gather_cols_kernel(const int64_t* src, const int32_t* col_idx, int64_t nnz, int32_t* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nnz;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = col_idx[src[i]];
}

__global__ void gather_vals_kernel(const int64_t* src, const double* topo, int64_t nnz, double* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nnz;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = topo[src[i]];
}

unsigned grid_of(int64_t n) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32))); }

}  // namespace

cudaError_t launch_refmask(int t, const ElemArgs& a, double* out, cudaStream_t s) {
  switch (t) {
    case C3D4: return launch_refmask_t<C3D4>(a, out, s);
    case C3D10: return launch_refmask_t<C3D10>(a, out, s);
    case C3D8: return launch_refmask_t<C3D8>(a, out, s);
    case C3D8R: return launch_refmask_t<C3D8R>(a, out, s);
    case C3D20: return launch_refmask_t<C3D20>(a, out, s);
    case C3D20R: return launch_refmask_t<C3D20R>(a, out, s);
    case C3D6: return launch_refmask_t<C3D6>(a, out, s);
    case C3D15: return launch_refmask_t<C3D15>(a, out, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t compact_pattern(const int64_t* row_ptr, const int32_t* col_idx, int32_t n_rows, int64_t nnz,
                            const double* counts, int64_t** row_ptr_c, int32_t** col_idx_c, int64_t** src,
                            int64_t* nnz_c, cudaStream_t s) {
  uint8_t* keep = nullptr;
  int64_t *row_len = nullptr, *d_count = nullptr;
  void* temp = nullptr;
  size_t temp_bytes = 0, t2 = 0;
  cudaError_t e = cudaMalloc(&keep, std::max<int64_t>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&row_len, sizeof(int64_t) * (static_cast<size_t>(n_rows) + 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_count, sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(row_ptr_c, sizeof(int64_t) * (static_cast<size_t>(n_rows) + 1));
  if (e == cudaSuccess) {
    keep_kernel<<<grid_of(nnz), 256, 0, s>>>(counts, keep, nnz);
    row_len_kernel<<<grid_of(n_rows), 256, 0, s>>>(row_ptr, keep, n_rows, row_len);
    e = cudaMemsetAsync(row_len + n_rows, 0, sizeof(int64_t), s);
  }
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, row_len, *row_ptr_c, n_rows + 1, s);
  cub::CountingInputIterator<int64_t> idx(0);
  if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, t2, idx, keep, static_cast<int64_t*>(nullptr), d_count, nnz, s);
  temp_bytes = std::max(temp_bytes, t2);
  if (e == cudaSuccess) e = cudaMalloc(&temp, std::max<size_t>(temp_bytes, 16));
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(temp, temp_bytes, row_len, *row_ptr_c, n_rows + 1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(nnz_c, *row_ptr_c + n_rows, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMalloc(src, sizeof(int64_t) * static_cast<size_t>(std::max<int64_t>(*nnz_c, 1)));
  if (e == cudaSuccess) e = cudaMalloc(col_idx_c, sizeof(int32_t) * static_cast<size_t>(std::max<int64_t>(*nnz_c, 1)));
  if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(temp, temp_bytes, idx, keep, *src, d_count, nnz, s);
  if (e == cudaSuccess) {
    gather_cols_kernel<<<grid_of(*nnz_c), 256, 0, s>>>(*src, col_idx, *nnz_c, *col_idx_c);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(keep);
  cudaFree(row_len);
  cudaFree(d_count);
  cudaFree(temp);
  return e;
}

cudaError_t gather_values(const int64_t* src, const double* topo, int64_t nnz_c, double* out, cudaStream_t s) {
  if (nnz_c == 0) return cudaSuccess;
  gather_vals_kernel<<<grid_of(nnz_c), 256, 0, s>>>(src, topo, nnz_c, out);
  return cudaGetLastError();
}

}  // namespace cxg
