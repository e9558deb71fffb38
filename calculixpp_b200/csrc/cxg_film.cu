// *FILM faces of the conduction assembly (assemble_conduction, src/fem/thermal.cpp:
// 113-126; face_surface_integrals, src/fem/loads.cpp:361-389).
//
// Film pass: one thread per element that carries films, its films in film order. For
// each film face it evaluates M_ij = int N_i N_j dA and L_i = int N_i dA with the face
// rule (3-point triangle, 2x2 quad; dA = |t_xi x t_eta| w), adds h M_ij to the element's
// FP64 block of nodes (fn_i, fn_j) that the conduction element pass wrote (so the row
// gather scatters the film matrix with the element's, prescribed columns included), and
// writes h T_sink L_i per face node. Load pass: one thread per node that lies on a film
// face sums those loads in film order into component 0 of the load vector the gather
// adds to the rhs. No atomics: results do not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "cxg_faces.hpp"
#include "cxg_internal.cuh"

namespace cxg {

namespace {

__host__ __device__ constexpr int upper_block(int n, int a, int b) { return a * n - a * (a - 1) / 2 + (b - a); }

__global__ void film_elem_kernel(ElemArgs A, int type, FilmArgs F, double* edata) {
  const int n = nodes_of(type), NB = n * (n + 1) / 2;
  constexpr double kTri[3][3] = {{1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
                                 {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                                 {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
  constexpr double qg = 0.577350269189625764;  // 1 / sqrt(3)
  constexpr double kQuad[4][3] = {{-qg, -qg, 1.0}, {qg, -qg, 1.0}, {qg, qg, 1.0}, {-qg, qg, 1.0}};
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < F.n_felem;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t e = F.felem[g];
    double* blocks = edata + e * (static_cast<int64_t>(NB) * 10);
    for (int32_t k = F.fptr[g]; k < F.fptr[g + 1]; ++k) {
      const int32_t f = F.flist[k];
      int fn[8], nf = 0;
      bool quad = false;
      face_nodes_of(type, F.face[f], fn, &nf, &quad);  // validated when the films were set
      double x[8][3];
      for (int i = 0; i < nf; ++i) {
        const int64_t node = A.conn[e * n + fn[i]];
        for (int d = 0; d < 3; ++d) x[i][d] = A.coords[3 * node + d];
      }
      double M[8][8], L[8];
      for (int i = 0; i < 8; ++i) {
        L[i] = 0.0;
        for (int j = 0; j < 8; ++j) M[i][j] = 0.0;
      }
      const int ng = quad ? 4 : 3;
      for (int q = 0; q < ng; ++q) {
        const double* gp = quad ? kQuad[q] : kTri[q];
        double N[8], dxi[8], deta[8], txi[3] = {0, 0, 0}, teta[3] = {0, 0, 0};
        face_shape(quad, nf, gp[0], gp[1], N, dxi, deta);
        for (int i = 0; i < nf; ++i)
          for (int d = 0; d < 3; ++d) {
            txi[d] += dxi[i] * x[i][d];
            teta[d] += deta[i] * x[i][d];
          }
        const double c0 = txi[1] * teta[2] - txi[2] * teta[1], c1 = txi[2] * teta[0] - txi[0] * teta[2],
                     c2 = txi[0] * teta[1] - txi[1] * teta[0];
        const double dA = sqrt(c0 * c0 + c1 * c1 + c2 * c2) * gp[2];
        for (int i = 0; i < nf; ++i) {
          L[i] += N[i] * dA;
          for (int j = 0; j < nf; ++j) M[i][j] += N[i] * N[j] * dA;
        }
      }
      const double h = F.h[f], hs = F.h[f] * F.sink[f];
      for (int i = 0; i < nf; ++i) {
        for (int j = 0; j < nf; ++j) {
          const int a = fn[i], b = fn[j];
          if (a > b) continue;  // the stored upper block (a, b) carries the pair once
          double* blk = blocks + upper_block(n, a, b) * 10;
          const double v = h * M[i][j];
          blk[0] += v;
          blk[4] += v;
          blk[8] += v;
        }
        F.load[static_cast<int64_t>(f) * 8 + i] = hs * L[i];
      }
    }
  }
}

__global__ void film_load_kernel(FilmArgs F, double* f_ext3) {
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < F.n_fnode;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int32_t k = F.fnptr[g]; k < F.fnptr[g + 1]; ++k) s += F.load[F.fnlist[k]];
    f_ext3[3 * F.fnode[g]] += s;
  }
}

unsigned film_grid(int64_t n) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, 148 * 8)));
}

}  // namespace

cudaError_t launch_films(int type, const ElemArgs& a, const FilmArgs& f, double* edata, double* f_ext3,
                         cudaStream_t s) {
  if (f.n_felem > 0) {
    film_elem_kernel<<<film_grid(f.n_felem), 128, 0, s>>>(a, type, f, edata);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (f.n_fnode > 0) {
    film_load_kernel<<<film_grid(f.n_fnode), 128, 0, s>>>(f, f_ext3);
    return cudaGetLastError();
  }
  return cudaSuccess;
}

}  // namespace cxg
