// Field recovery from a displacement field (recover_gauss_stress / recover_fields,
// src/fem/stress.cpp:147-271; linear elasticity), and the thermal-strain load vector
// (thermal_strain_load_vector, src/fem/loads.cpp:515-560; element_thermal_load,
// element.cpp:636-665).
//
// Thermal strain, when the plan has it: te_k = T_k - t_ref at the element's nodes with an
// applied temperature (0 elsewhere), eps_th = alpha sum_k N_k te_k on the normal
// components at every Gauss point; the stress is D (eps - eps_th) and the element force
// sum_q detJ w sigma_q g_a is then K_e u_e - f_th_e. In thermal-load mode the element pass
// forms D eps_th instead (no displacement), and the node pass sums f_th.
//
// Element pass: one warp per element. Lanes take Gauss points: physical gradients,
// displacement gradient, engineering strain and sigma = D eps (written out per point
// when asked); then lanes take (component) means over the Gauss points, which the hex
// and wedge families give every element node (extrapolation.hpp:34-41; C3D10 nodes get
// the corner extrapolation and midside averages of extrapolation.hpp:43-54), and
// (node, direction) internal forces f_a = sum_q detJ w sigma_q g_a (= K_e u_e).
// Node pass: one thread per node sums its incident elements' means and forces in
// element order (the order of the reference's element loop), divides the means by the
// number of incident elements and forms the reaction f_int - f_ext.
#include <cuda_runtime.h>

#include <algorithm>

#include "cxg_internal.cuh"

namespace cxg {

namespace {

constexpr int kRecWarps = 4;

// Value sets of 12 (strain, stress) per element that the node pass reads: one per node
// for C3D10 (its corner extrapolation differs per node), one (the mean) otherwise.
template <int ET>
constexpr int rec_sets() {
  return ET == C3D10 ? nodes_of(ET) : 1;
}

template <int ET>
constexpr int rec_warp_doubles() {
  constexpr int n = nodes_of(ET), nq = gauss_of(ET);
  return 7 * n + nq + nq * n * 3 + nq * 12;  // x, u, te, detJ w, gradients, strain + stress
}

// THLOAD: thermal-load mode (felem = f_th_e; no displacement, no means)
template <int ET, bool THLOAD>
__global__ void __launch_bounds__(kRecWarps * 32) rec_elem_kernel(ElemArgs A, double* gp_stress, double* emean,
                                                                  double* felem) {
  constexpr int n = nodes_of(ET), nq = gauss_of(ET);
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* x = reinterpret_cast<double*>(smem) + warp * rec_warp_doubles<ET>();
  double* uu = x + 3 * n;
  double* te = uu + 3 * n;  // [n] temperature change of the element's nodes
  double* sq = te + n;
  double* g = sq + nq;         // [nq][n][3]
  double* es = g + nq * n * 3; // [nq][12]: strain[6], stress[6]
  const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kRecWarps + warp;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kRecWarps;
  for (int64_t e = gwarp; e < A.n_elems; e += nwarps) {
    const double alpha = A.th_temp ? A.th_alpha[e] : 0.0;
    for (int t = lane; t < 3 * n; t += 32) {
      const int64_t node = A.conn[e * n + t / 3];
      x[t] = A.coords[3 * node + t % 3];
      uu[t] = THLOAD ? 0.0 : A.u[3 * node + t % 3];
      if (t % 3 == 0)
        te[t / 3] = alpha != 0.0 && (!A.th_applied || A.th_applied[node]) ? A.th_temp[node] - A.th_tref[e] : 0.0;
    }
    __syncwarp();
    const double E = A.young[e], nu = A.poisson[e];
    const double um2 = E / (1.0 + nu);
    const double lam = nu * um2 / (1.0 - 2.0 * nu), mu = um2 / 2.0;
    for (int q = lane; q < nq; q += 32) {
      double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[i][j] += x[3 * k + i] * c_dN[dn_offset(ET) + (3 * k + j) * nq + q];
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
      sq[q] = det * c_w[ET][q];
      double du[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k) {
        const double d0 = c_dN[dn_offset(ET) + (3 * k) * nq + q], d1 = c_dN[dn_offset(ET) + (3 * k + 1) * nq + q],
                     d2 = c_dN[dn_offset(ET) + (3 * k + 2) * nq + q];
        double gk[3];
        for (int i = 0; i < 3; ++i) {
          gk[i] = it[i][0] * d0 + it[i][1] * d1 + it[i][2] * d2;
          g[(q * n + k) * 3 + i] = gk[i];
        }
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) du[i][j] += gk[j] * uu[3 * k + i];
      }
      double eth = 0.0;  // alpha sum_k N_k te_k
      if (alpha != 0.0) {
        double dT = 0.0;
        for (int k = 0; k < n; ++k) dT += c_N[nn_offset(ET) + k * nq + q] * te[k];
        eth = alpha * dT;
      }
      double* st = es + 12 * q;
      st[0] = du[0][0];
      st[1] = du[1][1];
      st[2] = du[2][2];
      st[3] = du[0][1] + du[1][0];
      st[4] = du[0][2] + du[2][0];
      st[5] = du[1][2] + du[2][1];
      // elastic strain: eps - eps_th, or eps_th itself in thermal-load mode (D eps_th)
      const double e0 = THLOAD ? eth : st[0] - eth, e1 = THLOAD ? eth : st[1] - eth, e2 = THLOAD ? eth : st[2] - eth;
      const double tr = e0 + e1 + e2;
      st[6] = lam * tr + 2.0 * mu * e0;
      st[7] = lam * tr + 2.0 * mu * e1;
      st[8] = lam * tr + 2.0 * mu * e2;
      st[9] = THLOAD ? 0.0 : mu * st[3];
      st[10] = THLOAD ? 0.0 : mu * st[4];
      st[11] = THLOAD ? 0.0 : mu * st[5];
      if (gp_stress)
        for (int c = 0; c < 6; ++c) gp_stress[(e * nq + q) * 6 + c] = st[6 + c];
    }
    __syncwarp();
    if (emean) {
      if constexpr (ET == C3D10) {
        // corners: the a4 extrapolation matrix of CalculiX extrapolate.f; midsides: the
        // mean of their edge's corners (extrapolation.hpp:18-55)
        constexpr double kA4diag = 1.927050983124842, kA4off = -0.309016994374947;
        constexpr int kMid[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
        for (int t = lane; t < n * 12; t += 32) {
          const int i = t / 12, c = t % 12;
          auto corner = [&](int cn) {
            double v = 0.0;
            for (int l = 0; l < 4; ++l) v += (cn == l ? kA4diag : kA4off) * es[12 * l + c];
            return v;
          };
          emean[(e * n + i) * 12 + c] = i < 4 ? corner(i) : 0.5 * (corner(kMid[i - 4][0]) + corner(kMid[i - 4][1]));
        }
      } else {
        for (int c = lane; c < 12; c += 32) {
          double m = 0.0;
          for (int q = 0; q < nq; ++q) m += es[12 * q + c];
          emean[e * 12 + c] = m * (1.0 / nq);
        }
      }
    }
    if (felem)
      for (int t = lane; t < 3 * n; t += 32) {
        const int a = t / 3, d = t % 3;
        double f = 0.0;
        for (int q = 0; q < nq; ++q) {
          const double* S = es + 12 * q + 6;
          const double* ga = g + (q * n + a) * 3;
          // row d of sigma (Voigt xx yy zz xy xz yz) times g_a
          const double s0 = d == 0 ? S[0] : (d == 1 ? S[3] : S[4]);
          const double s1 = d == 0 ? S[3] : (d == 1 ? S[1] : S[5]);
          const double s2 = d == 0 ? S[4] : (d == 1 ? S[5] : S[2]);
          f += sq[q] * (s0 * ga[0] + s1 * ga[1] + s2 * ga[2]);
        }
        felem[e * (3 * n) + t] = f;
      }
    __syncwarp();
  }
}

template <int ET>
__global__ void rec_node_kernel(ElemArgs A, const int64_t* inc_ptr, const int32_t* inc_code, const double* emean,
                                const double* felem, const double* f_ext, double* strain, double* stress,
                                double* reaction) {
  constexpr int n = nodes_of(ET);
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < A.n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double m[12];
    double f[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < 12; ++c) m[c] = 0.0;
    const int64_t i0 = inc_ptr[a], i1 = inc_ptr[a + 1];
    for (int64_t i = i0; i < i1; ++i) {
      const int code = inc_code[i];
      const int64_t e = code / n;
      const int la = code % n;
      const int64_t set = rec_sets<ET>() == 1 ? e : e * n + la;
      if (emean)
        for (int c = 0; c < 12; ++c) m[c] += emean[set * 12 + c];
      for (int d = 0; d < 3; ++d) f[d] += felem[e * (3 * n) + 3 * la + d];
    }
    const int64_t cnt = i1 - i0;
    for (int c = 0; c < 6; ++c) {
      if (strain) strain[6 * a + c] = cnt > 0 ? m[c] / static_cast<double>(cnt) : 0.0;
      if (stress) stress[6 * a + c] = cnt > 0 ? m[6 + c] / static_cast<double>(cnt) : 0.0;
    }
    if (reaction)
      for (int d = 0; d < 3; ++d) reaction[3 * a + d] = f[d] - (f_ext ? f_ext[3 * a + d] : 0.0);
  }
}

unsigned rec_grid(int64_t n) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)));
}

template <int ET>
cudaError_t launch_recover_t(const ElemArgs& a, const int64_t* inc_ptr, const int32_t* inc_code, double* gp_stress,
                             double* emean, double* felem, const double* f_ext, double* strain, double* stress,
                             double* reaction, bool thermal_load, cudaStream_t s) {
  if (a.n_elems > 0) {
    auto kern = thermal_load ? rec_elem_kernel<ET, true> : rec_elem_kernel<ET, false>;
    const size_t smem = sizeof(double) * kRecWarps * rec_warp_doubles<ET>();
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    const int64_t blocks = std::min<int64_t>((a.n_elems + kRecWarps - 1) / kRecWarps, 148 * 8);
    kern<<<static_cast<unsigned>(std::max<int64_t>(blocks, 1)), kRecWarps * 32, smem, s>>>(a, gp_stress, emean, felem);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
  }
  if (felem && inc_ptr) {
    rec_node_kernel<ET><<<rec_grid(a.n_nodes), 256, 0, s>>>(a, inc_ptr, inc_code, emean, felem, f_ext, strain, stress,
                                                            reaction);
    return cudaGetLastError();
  }
  return cudaSuccess;
}

}  // namespace

cudaError_t launch_recover(int t, const ElemArgs& a, const int64_t* inc_ptr, const int32_t* inc_code,
                           double* gp_stress, double* emean, double* felem, const double* f_ext, double* strain,
                           double* stress, double* reaction, bool thermal_load, cudaStream_t s) {
  switch (t) {
#define CXG_REC(T)                                                                                             \
  case T:                                                                                                      \
    return launch_recover_t<T>(a, inc_ptr, inc_code, gp_stress, emean, felem, f_ext, strain, stress, reaction, \
                               thermal_load, s);
    CXG_REC(C3D4)
    CXG_REC(C3D10)
    CXG_REC(C3D8)
    CXG_REC(C3D8R)
    CXG_REC(C3D20)
    CXG_REC(C3D20R)
    CXG_REC(C3D6)
    CXG_REC(C3D15)
#undef CXG_REC
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace cxg
