// Element integration + CSR scatter kernels for sm_100a.
//
// One warp integrates one element at a time (elements strided over all warps of a
// persistent grid):
//   phase A  lanes gather the element's node coordinates, displacements and CSR
//            addressing data into the warp's shared-memory slice;
//   phase B  lane q handles Gauss point q: Jacobian, det, inverse (FP64), physical
//            gradients g_k = J^-T dN_k for every node, and in material-point mode the
//            small strain, the J2 radial return (FP64) and the tangent parameters;
//   phase C  lanes stride over the n(n+1)/2 node pairs (a <= b) of the symmetric
//            element matrix, accumulate the 3x3 Gram block sum_q s_q g_a g_b^T (and its
//            plastic counterparts) in registers, form K_ab in closed form
//              K_ab = lam* G + mu* (G^T + tr(G) I) - c M
//            (the isotropic B^T D B without the 6x6 B products of
//            src/fem/element.cpp:440-462), and store K_ab and K_ab^T in the dense
//            element matrices of the per-element API;
//   phase D  lanes stride over nodes for the internal force f_a = sum_q s_q S_q g_a.
// Precision: FP64, or "mixed" where the Gram blocks and K_ab are formed in FP32 from
// FP32 gradients while Jacobians, their inverses, the J2 update and every global
// accumulation stay FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "cxg_internal.cuh"

namespace cxg {

__constant__ double c_dN[kDnTotal];
__constant__ double c_w[8][kMaxGauss];
__constant__ double c_N[kNTotal];

namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;


// sqrt(3/2) with the literal the reference uses (src/fem/plasticity.cpp:24), so the
// yield-function value agrees with it bit for bit.
constexpr double kSqrt3_2 = 1.224744871391589;

__device__ __forceinline__ void report(DevStatus* st, int code, int64_t e) {
  atomicCAS(&st->code, 0, code);
  atomicMin(&st->bad_elem, static_cast<unsigned long long>(e));
}

// Piecewise-linear hardening (src/fem/plasticity.cpp:67-88).
__device__ __forceinline__ void hardening(const J2Mat& M, double ep, double& sy, double& h) {
  const int n = M.n;
  if (n == 1 || ep <= M.ep[0]) {
    sy = M.sy[0];
    h = 0.0;
    return;
  }
  if (ep >= M.ep[n - 1]) {
    sy = M.sy[n - 1];
    h = 0.0;
    return;
  }
  for (int i = 0; i + 1 < n; ++i) {
    if (ep >= M.ep[i] && ep <= M.ep[i + 1]) {
      h = (M.sy[i + 1] - M.sy[i]) / (M.ep[i + 1] - M.ep[i]);
      sy = M.sy[i] + h * (ep - M.ep[i]);
      return;
    }
  }
  sy = M.sy[n - 1];
  h = 0.0;
}

// Isotropic tangent in the form D = lam* 1x1 + mu* (2 I_normal + I_shear) - c n n^T.
struct Tangent {
  double lam, mu, c, mu_hg;
  double n[6];
  bool plastic;
};

// Small-strain J2 radial return with the consistent tangent (Simo-Hughes box 3.2/3.4,
// restating src/fem/plasticity.cpp:90-236). lam/mu_el: elastic_iso_D's constants;
// mu: the shear modulus the return map uses, E/(2(1+nu)). cs: committed history,
// ts: trial history out.
__device__ void j2_update(const J2Mat& M, double lam, double mu_el, double mu,
                          const double* eps, const double* cs, double* ts, double* sig,
                          Tangent& tp) {
  const double lam2mu = lam + 2.0 * mu_el;
  double el[6];
  for (int i = 0; i < 6; ++i) el[i] = eps[i] - cs[i];
  double st[6];
  st[0] = lam2mu * el[0] + lam * el[1] + lam * el[2];
  st[1] = lam * el[0] + lam2mu * el[1] + lam * el[2];
  st[2] = lam * el[0] + lam * el[1] + lam2mu * el[2];
  st[3] = mu_el * el[3];
  st[4] = mu_el * el[4];
  st[5] = mu_el * el[5];
  const double p = (st[0] + st[1] + st[2]) / 3.0;
  double s_tr[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
  double xi[6];
  for (int i = 0; i < 6; ++i) xi[i] = s_tr[i] - cs[7 + i];
  const double xi_norm = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2] +
                              2.0 * (xi[3] * xi[3] + xi[4] * xi[4] + xi[5] * xi[5]));
  const double q_tr = kSqrt3_2 * xi_norm;
  double sy0 = 0.0, h0 = 0.0;
  if (M.plastic) hardening(M, cs[6], sy0, h0);
  if (!M.plastic || q_tr - sy0 <= 0.0 || xi_norm == 0.0) {
    for (int i = 0; i < 6; ++i) sig[i] = st[i];
    for (int i = 0; i < kStateDoubles; ++i) ts[i] = cs[i];
    tp.lam = lam;
    tp.mu = mu_el;
    tp.c = 0.0;
    tp.mu_hg = mu_el;
    tp.plastic = false;
    for (int i = 0; i < 6; ++i) tp.n[i] = 0.0;
    return;
  }
  const double ep0 = cs[6];
  double dgamma = 0.0;
  for (int it = 0; it < 50; ++it) {
    double sy, h_iso;
    hardening(M, ep0 + dgamma, sy, h_iso);
    const double g = q_tr - 3.0 * mu * dgamma - M.h_kin * dgamma - sy;
    const double dg = -(3.0 * mu + M.h_kin + h_iso);
    const double step = -g / dg;
    dgamma += step;
    if (dgamma < 0.0) dgamma = 0.0;
    if (fabs(step) <= 1e-14 * (1.0 + fabs(dgamma))) break;
  }
  double nv[6];
  for (int i = 0; i < 6; ++i) nv[i] = xi[i] / xi_norm;
  const double dev_scale = 2.0 * mu * dgamma * kSqrt3_2;
  const double alpha_scale = (2.0 / 3.0) * M.h_kin * dgamma * kSqrt3_2;
  const double dep_scale = dgamma * kSqrt3_2;
  for (int i = 0; i < 6; ++i) {
    sig[i] = (s_tr[i] - dev_scale * nv[i]) + (i < 3 ? p : 0.0);
    ts[i] = cs[i] + dep_scale * nv[i] * (i < 3 ? 1.0 : 2.0);
    ts[7 + i] = cs[7 + i] + alpha_scale * nv[i];
  }
  ts[6] = ep0 + dgamma;
  double sy, h_iso;
  hardening(M, ep0 + dgamma, sy, h_iso);
  const double theta = 1.0 - (2.0 * mu * dgamma * kSqrt3_2) / xi_norm;
  const double denom = 1.0 + (h_iso + M.h_kin) / (3.0 * mu);
  const double theta_bar = 1.0 / denom - (1.0 - theta);
  // De - (1-theta) Idev - 2 mu theta_bar n n^T regrouped by structure.
  tp.lam = lam + (2.0 / 3.0) * (1.0 - theta) * mu;
  tp.mu = mu_el - (1.0 - theta) * mu;
  tp.c = 2.0 * mu * theta_bar;
  tp.mu_hg = tp.mu - tp.c * nv[3] * nv[3];
  tp.plastic = true;
  for (int i = 0; i < 6; ++i) tp.n[i] = nv[i];
}

// Flanagan-Belytschko hourglass base vectors (src/fem/element.cpp:529-534).
__constant__ double c_hg[4][8] = {
    {1, 1, -1, -1, -1, -1, 1, 1},
    {1, -1, -1, 1, -1, 1, 1, -1},
    {1, -1, 1, -1, 1, -1, 1, -1},
    {-1, 1, -1, 1, 1, -1, 1, -1},
};

template <int ET, int MODE, typename R>
struct WarpSmem {
  static constexpr int n = nodes_of(ET);
  static constexpr int nq = gauss_of(ET);
  static constexpr int GS = 3 * n + 1;
  static constexpr bool T = MODE == MODE_TANGENT;
  static constexpr bool DF = sizeof(R) == 4;  // mixed precision: diagonal blocks from row sums
  static constexpr int GD = T ? 27 : 9;
  double x[3 * n];
  double gd[DF ? n * GD : 1];  // per-node FP64 sums of the off-diagonal Gram blocks
  double gam[32];
  double kappa;
  double gc[3 * n];  // FP64 gradients at the last Gauss point (C3D8R: the centroid)
  double vol;        // w det J there (C3D8R: 8 det J = element volume)
  double u[T ? 3 * n : 1];
  double sig[T ? nq * 6 : 1];  // s_q * sigma_q (Voigt)
  int flags;                   // bit0: some Gauss point plastic
  R g[nq * GS];                // [q][d][k] physical gradients
  R s[nq];                     // w_q det J_q
  R dp[T ? nq * 4 : 1];        // s*lam*, s*mu*, s*c per Gauss point
  R m[T ? nq * GS : 1];        // N_q g_k (plastic points)
  double mu_hg;
};

// Gram blocks of node pair (a, b) over the Gauss points, in precision R:
//   elastic points only : G1 = sum_q s_q g_a g_b^T
//   with plastic points : G1 = sum_q (s lam*)_q g_a g_b^T, G2 = sum_q (s mu*)_q g_a g_b^T,
//                         G3 = sum_q (s c)_q m_a m_b^T   (m = N g, N the return direction)
template <int n, int nq, bool TAN, typename R, typename WS>
__device__ __forceinline__ void gram(const WS& W, int a, int b, bool plastic, R (&G1)[3][3], R (&G2)[3][3],
                                     R (&G3)[3][3]) {
  constexpr int GS = 3 * n + 1;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) G1[i][j] = G2[i][j] = G3[i][j] = R(0);
  if (!TAN || !plastic) {
#pragma unroll 3
    for (int q = 0; q < nq; ++q) {
      const R* gq = W.g + q * GS;
      const R s = W.s[q];
      const R ga[3] = {s * gq[a], s * gq[n + a], s * gq[2 * n + a]};
      const R gb[3] = {gq[b], gq[n + b], gq[2 * n + b]};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) G1[i][j] += ga[i] * gb[j];
    }
    return;
  }
  if (TAN) {
    for (int q = 0; q < nq; ++q) {
      const R* gq = W.g + q * GS;
      const R sl = W.dp[q * 4 + 0], sm = W.dp[q * 4 + 1], sc = W.dp[q * 4 + 2];
      const R ga[3] = {gq[a], gq[n + a], gq[2 * n + a]};
      const R gb[3] = {gq[b], gq[n + b], gq[2 * n + b]};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          G1[i][j] += (sl * ga[i]) * gb[j];
          G2[i][j] += (sm * ga[i]) * gb[j];
        }
      if (sc != R(0)) {
        const R* mq = W.m + q * GS;
        const R ma[3] = {sc * mq[a], sc * mq[n + a], sc * mq[2 * n + a]};
        const R mb[3] = {mq[b], mq[n + b], mq[2 * n + b]};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) G3[i][j] += ma[i] * mb[j];
      }
    }
  }
}

// K_ab from its Gram blocks, in FP64:
//   elastic: lam G1 + mu (G1^T + tr(G1) I)        (= B_a^T D B_b summed over the points)
//   plastic: G1 + G2^T + tr(G2) I - G3
template <typename T>
__device__ __forceinline__ void combine(const T (&G1)[3][3], const T (&G2)[3][3], const T (&G3)[3][3],
                                        bool plastic, double lam, double mu, double (&K)[3][3]) {
  if (!plastic) {
    const double tr = static_cast<double>(G1[0][0]) + static_cast<double>(G1[1][1]) + static_cast<double>(G1[2][2]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        K[i][j] = lam * static_cast<double>(G1[i][j]) + mu * static_cast<double>(G1[j][i]) + (i == j ? mu * tr : 0.0);
    return;
  }
  const double tr = static_cast<double>(G2[0][0]) + static_cast<double>(G2[1][1]) + static_cast<double>(G2[2][2]);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      K[i][j] = static_cast<double>(G1[i][j]) + static_cast<double>(G2[j][i]) + (i == j ? tr : 0.0) -
                static_cast<double>(G3[i][j]);
}

// C3D8R hourglass stiffness kappa sum_alpha gamma_alpha,a gamma_alpha,b on the block
// diagonal (src/fem/element.cpp:583-595).
template <typename WS>
__device__ __forceinline__ void add_hourglass(const WS& W, int a, int b, double (&K)[3][3]) {
  double h = 0.0;
  for (int al = 0; al < 4; ++al) h += W.gam[al * 8 + a] * W.gam[al * 8 + b];
  h *= W.kappa;
  K[0][0] += h;
  K[1][1] += h;
  K[2][2] += h;
}

// Dense element-matrix store: rows of node a / columns of node b, and (a != b) the
// transposed block into rows of b. (The assembled CSR systems are formed by the
// two-pass element pass and row gather of cxg_v2.cu.)
template <int n, bool DENSE, typename WS>
__device__ __forceinline__ void write_pair(const ElemArgs& A, const WS& W, int64_t e, int a, int b,
                                           const double (&K)[3][3]) {
  constexpr int nd = 3 * n;
  if (DENSE) {
    double* Ke = A.Ke + e * nd * nd;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        Ke[(3 * a + i) * nd + 3 * b + j] = K[i][j];
        Ke[(3 * b + j) * nd + 3 * a + i] = K[i][j];
      }
    return;
  }
}

template <int ET, int MODE, bool DENSE, typename R>
__global__ void __launch_bounds__(kThreads) element_kernel(ElemArgs A) {
  constexpr int n = nodes_of(ET);
  constexpr int nq = gauss_of(ET);
  constexpr int nd = 3 * n;
  constexpr int NPO = n * (n - 1) / 2;  // off-diagonal node pairs
  constexpr int GS = 3 * n + 1;
  constexpr bool TAN = MODE == MODE_TANGENT;
  using WS = WarpSmem<ET, MODE, R>;
  constexpr bool DIAGFIX = WS::DF;
  constexpr int GD = WS::GD;

  extern __shared__ __align__(16) unsigned char smem[];
  double* sdN = reinterpret_cast<double*>(smem);  // [n*3*nq]
  double* sw = sdN + n * 3 * nq;                  // [nq]
  unsigned short* spair = reinterpret_cast<unsigned short*>(sw + nq);
  constexpr size_t cta_bytes = ((sizeof(double) * (n * 3 * nq + nq) + 2 * NPO) + 15) / 16 * 16;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  WS& W = *reinterpret_cast<WS*>(smem + cta_bytes + warp * ((sizeof(WS) + 15) / 16 * 16));

  for (int i = threadIdx.x; i < n * 3 * nq; i += blockDim.x) sdN[i] = c_dN[dn_offset(ET) + i];
  for (int i = threadIdx.x; i < nq; i += blockDim.x) sw[i] = c_w[ET][i];
  for (int i = threadIdx.x; i < NPO; i += blockDim.x) {
    int a = 0, r = i;
    while (r >= n - 1 - a) {
      r -= n - 1 - a;
      ++a;
    }
    spair[i] = static_cast<unsigned short>(a | ((a + 1 + r) << 8));
  }
  __syncthreads();

  const int64_t gwarp = (static_cast<int64_t>(blockIdx.x) * kWarps) + warp;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kWarps;

  for (int64_t e = gwarp; e < A.n_elems; e += nwarps) {
    // ---- phase A: gather ------------------------------------------------------
    for (int t = lane; t < nd; t += 32) {
      W.x[t] = A.elem_coords[e * nd + t];
      if (TAN) W.u[t] = A.u[e * nd + t];
    }
    const double E = A.young[e];
    const double nu = A.poisson[e];
    const double um2 = E / (1.0 + nu);
    const double lam = nu * um2 / (1.0 - 2.0 * nu);
    const double mu_el = um2 / 2.0;
    const double mu_j2 = E / (2.0 * (1.0 + nu));
    __syncwarp();

    // ---- phase B: one Gauss point per lane ----------------------------------------
    bool plastic = false;
    if (lane < nq) {
      const int q = lane;
      double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll 4
      for (int k = 0; k < n; ++k) {
        const double d0 = sdN[(3 * k + 0) * nq + q], d1 = sdN[(3 * k + 1) * nq + q],
                     d2 = sdN[(3 * k + 2) * nq + q];
        for (int i = 0; i < 3; ++i) {
          const double xk = W.x[3 * k + i];
          J[i][0] = fma(xk, d0, J[i][0]);
          J[i][1] = fma(xk, d1, J[i][1]);
          J[i][2] = fma(xk, d2, J[i][2]);
        }
      }
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      if (!(det > 0.0)) report(A.status, 4 /*CXG_ERR_NEGATIVE_JACOBIAN*/, e);
      const double inv = 1.0 / det;
      // Rows of J^-T (= columns of J^-1).
      const double it[3][3] = {
          {c00 * inv, c01 * inv, c02 * inv},
          {(J[0][2] * J[2][1] - J[0][1] * J[2][2]) * inv, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv,
           (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * inv},
          {(J[0][1] * J[1][2] - J[0][2] * J[1][1]) * inv, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * inv,
           (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv}};
      const double sq = det * sw[q];
      W.s[q] = static_cast<R>(sq);
      if (ET == C3D8R) W.vol = sq;
      double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k) {
        const double d0 = sdN[(3 * k + 0) * nq + q], d1 = sdN[(3 * k + 1) * nq + q],
                     d2 = sdN[(3 * k + 2) * nq + q];
        double gk[3];
        for (int i = 0; i < 3; ++i) {
          gk[i] = it[i][0] * d0 + it[i][1] * d1 + it[i][2] * d2;
          W.g[q * GS + i * n + k] = static_cast<R>(gk[i]);
          if (ET == C3D8R) W.gc[i * n + k] = gk[i];
        }
        if (TAN) {
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) H[i][j] = fma(W.u[3 * k + i], gk[j], H[i][j]);
        }
      }
      if (TAN) {
        const double eps[6] = {H[0][0], H[1][1], H[2][2], H[0][1] + H[1][0], H[0][2] + H[2][0],
                               H[1][2] + H[2][1]};
        const int mat = A.elem_mat ? A.elem_mat[e] : 0;
        const int64_t gidx = e * nq + q;
        double cs[kStateDoubles], ts[kStateDoubles], sig[6];
        for (int c = 0; c < kStateDoubles; ++c) cs[c] = A.state_c[c * A.n_gauss + gidx];
        Tangent tp;
        j2_update(A.mats[mat], lam, mu_el, mu_j2, eps, cs, ts, sig, tp);
        for (int c = 0; c < kStateDoubles; ++c) A.state_t[c * A.n_gauss + gidx] = ts[c];
        for (int c = 0; c < 6; ++c) W.sig[q * 6 + c] = sq * sig[c];
        W.dp[q * 4 + 0] = static_cast<R>(sq * tp.lam);
        W.dp[q * 4 + 1] = static_cast<R>(sq * tp.mu);
        W.dp[q * 4 + 2] = static_cast<R>(sq * tp.c);
        plastic = tp.plastic;
        if (plastic) {
          // m_k = N g_k with N the symmetric tensor of the return direction.
          const double* nv = tp.n;
          for (int k = 0; k < n; ++k) {
            const double gx = W.g[q * GS + 0 * n + k], gy = W.g[q * GS + 1 * n + k],
                         gz = W.g[q * GS + 2 * n + k];
            W.m[q * GS + 0 * n + k] = static_cast<R>(nv[0] * gx + nv[3] * gy + nv[4] * gz);
            W.m[q * GS + 1 * n + k] = static_cast<R>(nv[3] * gx + nv[1] * gy + nv[5] * gz);
            W.m[q * GS + 2 * n + k] = static_cast<R>(nv[4] * gx + nv[5] * gy + nv[2] * gz);
          }
        }
        if (q == nq - 1) W.mu_hg = tp.mu_hg;
      }
    }
    const bool any_plastic = __any_sync(0xffffffffu, plastic);
    __syncwarp();

    // ---- C3D8R hourglass control (src/fem/element.cpp:545-579) ------------------
    if (ET == C3D8R) {
      if (lane < 4) {
        const int al = lane;
        double gx[3] = {0, 0, 0};
        for (int j = 0; j < 8; ++j)
          for (int d = 0; d < 3; ++d) gx[d] += c_hg[al][j] * W.x[3 * j + d];
        for (int j = 0; j < 8; ++j) {
          double corr = 0.0;
          for (int d = 0; d < 3; ++d) corr += gx[d] * W.gc[d * n + j];
          W.gam[al * 8 + j] = c_hg[al][j] - corr;
        }
      }
      if (lane == 0) {
        double b2 = 0.0;
        for (int j = 0; j < 8; ++j)
          for (int d = 0; d < 3; ++d) {
            const double b = W.gc[d * n + j];
            b2 += b * b;
          }
        const double vol = W.vol;  // 8 det J at the centroid
        const double mu_hg = TAN ? W.mu_hg : mu_j2;
        W.kappa = 0.05 * mu_hg * vol * b2;
      }
      __syncwarp();
    }

    // ---- phase C: node-pair blocks -------------------------------------------------
    // Off-diagonal pairs (a < b) first. In mixed precision their Gram blocks are also
    // summed per node in FP64, and the diagonal blocks are then formed as the negative
    // of those sums: every block row of the element matrix sums to zero in FP64, so the
    // rigid translations stay in the null space exactly (sum_b g_b = 0), which FP32
    // rounding of the individual products would otherwise break.
    const bool plastic_elem = TAN && any_plastic;
    if (DIAGFIX) {
      for (int t = lane; t < n * GD; t += 32) W.gd[t] = 0.0;
      __syncwarp();
    }
    for (int pi = lane; pi < NPO; pi += 32) {
      const int pr = spair[pi];
      const int a = pr & 0xff, b = pr >> 8;
      R G1[3][3], G2[3][3], G3[3][3];
      gram<n, nq, TAN>(W, a, b, plastic_elem, G1, G2, G3);
      if (DIAGFIX) {
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            atomicAdd(&W.gd[a * GD + 3 * i + j], static_cast<double>(G1[i][j]));
            atomicAdd(&W.gd[b * GD + 3 * j + i], static_cast<double>(G1[i][j]));
            if (plastic_elem) {
              atomicAdd(&W.gd[a * GD + 9 + 3 * i + j], static_cast<double>(G2[i][j]));
              atomicAdd(&W.gd[b * GD + 9 + 3 * j + i], static_cast<double>(G2[i][j]));
              atomicAdd(&W.gd[a * GD + 18 + 3 * i + j], static_cast<double>(G3[i][j]));
              atomicAdd(&W.gd[b * GD + 18 + 3 * j + i], static_cast<double>(G3[i][j]));
            }
          }
      }
      double K[3][3];
      combine(G1, G2, G3, plastic_elem, lam, mu_el, K);
      if (ET == C3D8R) add_hourglass(W, a, b, K);
      write_pair<n, DENSE>(A, W, e, a, b, K);
    }
    __syncwarp();
    for (int a = lane; a < n; a += 32) {
      double K[3][3];
      if (DIAGFIX) {
        double G1[3][3], G2[3][3], G3[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            G1[i][j] = -W.gd[a * GD + 3 * i + j];
            G2[i][j] = plastic_elem ? -W.gd[a * GD + 9 + 3 * i + j] : 0.0;
            G3[i][j] = plastic_elem ? -W.gd[a * GD + 18 + 3 * i + j] : 0.0;
          }
        combine(G1, G2, G3, plastic_elem, lam, mu_el, K);
      } else {
        R G1[3][3], G2[3][3], G3[3][3];
        gram<n, nq, TAN>(W, a, a, plastic_elem, G1, G2, G3);
        combine(G1, G2, G3, plastic_elem, lam, mu_el, K);
      }
      if (ET == C3D8R) add_hourglass(W, a, a, K);
      write_pair<n, DENSE>(A, W, e, a, a, K);
    }

    // ---- phase D: internal force (material-point mode) -----------------------------
    if (TAN) {
      for (int a = lane; a < n; a += 32) {
        double f[3] = {0, 0, 0};
        for (int q = 0; q < nq; ++q) {
          const double* S = W.sig + q * 6;
          const double gx = W.g[q * GS + a], gy = W.g[q * GS + n + a], gz = W.g[q * GS + 2 * n + a];
          f[0] += S[0] * gx + S[3] * gy + S[4] * gz;
          f[1] += S[3] * gx + S[1] * gy + S[5] * gz;
          f[2] += S[4] * gx + S[5] * gy + S[2] * gz;
        }
        if (ET == C3D8R) {
          for (int al = 0; al < 4; ++al) {
            double gu[3] = {0, 0, 0};
            for (int j = 0; j < 8; ++j)
              for (int d = 0; d < 3; ++d) gu[d] += W.gam[al * 8 + j] * W.u[3 * j + d];
            const double ka = W.kappa * W.gam[al * 8 + a];
            for (int d = 0; d < 3; ++d) f[d] += ka * gu[d];
          }
        }
        for (int d = 0; d < 3; ++d) A.fe[e * nd + 3 * a + d] = f[d];
      }
    }
    __syncwarp();
  }
}

template <int ET, int MODE, bool DENSE, typename R>
cudaError_t launch_t(const ElemArgs& a, cudaStream_t s) {
  using WS = WarpSmem<ET, MODE, R>;
  constexpr int n = nodes_of(ET), nq = gauss_of(ET), NPO = n * (n - 1) / 2;
  constexpr size_t cta_bytes = ((sizeof(double) * (n * 3 * nq + nq) + 2 * NPO) + 15) / 16 * 16;
  constexpr size_t smem = cta_bytes + kWarps * ((sizeof(WS) + 15) / 16 * 16);
  auto kern = element_kernel<ET, MODE, DENSE, R>;
  static thread_local int configured_device = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured_device != dev) {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    configured_device = dev;
  }
  int per_sm = 0, sms = 0;
  cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
  if (err != cudaSuccess) return err;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t need = (a.n_elems + kWarps - 1) / kWarps;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, static_cast<int64_t>(std::max(per_sm, 1)) * sms));
  if (a.n_elems == 0) return cudaSuccess;
  kern<<<static_cast<unsigned>(grid), kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <int ET>
cudaError_t launch_type(int mode, bool dense, int precision, const ElemArgs& a, cudaStream_t s) {
  if (!dense) return cudaErrorNotSupported;  // CSR assembly is the two-pass path
  if (mode == MODE_LINEAR)
    return precision ? launch_t<ET, MODE_LINEAR, true, float>(a, s) : launch_t<ET, MODE_LINEAR, true, double>(a, s);
  return precision ? launch_t<ET, MODE_TANGENT, true, float>(a, s) : launch_t<ET, MODE_TANGENT, true, double>(a, s);
}

__global__ void rhs_init_kernel(const int32_t* dof_eq, const double* f_ext, int64_t ndof, double* rhs) {
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < ndof;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t eq = dof_eq[g];
    if (eq >= 0) rhs[eq] = f_ext ? f_ext[g] : 0.0;
  }
}

__global__ void state_transpose_kernel(const double* src, double* dst, int64_t G, bool to_soa) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < G * kStateDoubles;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t g = i / kStateDoubles;
    const int c = static_cast<int>(i % kStateDoubles);
    if (to_soa)
      dst[c * G + g] = src[i];
    else
      dst[i] = src[c * G + g];
  }
}

std::mutex g_tables_mu;
std::vector<int> g_tables_ready;

}  // namespace

cudaError_t ensure_tables() {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  std::lock_guard<std::mutex> lock(g_tables_mu);
  if (static_cast<int>(g_tables_ready.size()) > dev && g_tables_ready[dev]) return cudaSuccess;
  std::vector<double> dn(kDnTotal, 0.0), nv(kNTotal, 0.0);
  double w[8][kMaxGauss] = {};
  for (int t = kFirstType; t <= kLastType; ++t) {
    GaussPt pts[kMaxGauss];
    const int nq = gauss_rule(t, pts);
    const int n = nodes_of(t);
    for (int q = 0; q < nq; ++q) {
      double N[kMaxNodes], d[kMaxNodes][3];
      shape_derivatives(t, pts[q].xi, pts[q].et, pts[q].ze, N, d);
      for (int k = 0; k < n; ++k) {
        for (int j = 0; j < 3; ++j) dn[dn_offset(t) + (3 * k + j) * nq + q] = d[k][j];
        nv[nn_offset(t) + k * nq + q] = N[k];
      }
      w[t][q] = pts[q].w;
    }
  }
  err = cudaMemcpyToSymbol(c_dN, dn.data(), sizeof(double) * kDnTotal);
  if (err != cudaSuccess) return err;
  err = cudaMemcpyToSymbol(c_w, w, sizeof(w));
  if (err != cudaSuccess) return err;
  err = cudaMemcpyToSymbol(c_N, nv.data(), sizeof(double) * kNTotal);
  if (err != cudaSuccess) return err;
  if (static_cast<int>(g_tables_ready.size()) <= dev) g_tables_ready.resize(dev + 1, 0);
  g_tables_ready[dev] = 1;
  return cudaSuccess;
}

cudaError_t launch_element_kernel(int t, int mode, bool dense, int precision, const ElemArgs& a,
                                  cudaStream_t s) {
  switch (t) {
    case C3D4: return launch_type<C3D4>(mode, dense, precision, a, s);
    case C3D10: return launch_type<C3D10>(mode, dense, precision, a, s);
    case C3D8: return launch_type<C3D8>(mode, dense, precision, a, s);
    case C3D8R: return launch_type<C3D8R>(mode, dense, precision, a, s);
    case C3D20: return launch_type<C3D20>(mode, dense, precision, a, s);
    case C3D20R: return launch_type<C3D20R>(mode, dense, precision, a, s);
    case C3D6: return launch_type<C3D6>(mode, dense, precision, a, s);
    case C3D15: return launch_type<C3D15>(mode, dense, precision, a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_rhs_init(const int32_t* dof_eq, const double* f_ext, int64_t ndof, double* rhs,
                            cudaStream_t s) {
  if (ndof == 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((ndof + 255) / 256, 4096);
  rhs_init_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(dof_eq, f_ext, ndof, rhs);
  return cudaGetLastError();
}

cudaError_t launch_state_transpose(const double* src, double* dst, int64_t G, bool to_soa,
                                   cudaStream_t s) {
  if (G == 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((G * kStateDoubles + 255) / 256, 8192);
  state_transpose_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(src, dst, G, to_soa);
  return cudaGetLastError();
}

}  // namespace cxg
