// Assembly in two passes, with no atomics and every CSR value written exactly once.
//
// P1 (element pass): each warp integrates EPW elements at once. Lanes first handle
// (element, Gauss point) tasks: Jacobian, its inverse and the physical gradients in
// FP64 (plus the J2 return in material-point mode, whose trial history is written
// here, once per Gauss point). Then every lane owns a 2x4 tile of node pairs of one
// element and accumulates the 8 corresponding 3x3 blocks of K_e in registers over the
// Gauss points from float4/double4 gradient loads; elastic points use the Gram form
// K_ab = lam G + mu (G^T + tr(G) I) with G = sum_q s_q g_a g_b^T, plastic elements the
// full tangent sum_q s [lam* g_a g_b^T + mu* (g_b g_a^T + (g_a.g_b) I) - c m_a m_b^T]
// (m = N g, N the return direction, formed in the tile loop from the gradients and the
// stored N of the Gauss point). The upper blocks (a <= b) go to a per-element
// buffer, FP32 in mixed precision, FP64 otherwise; the internal force goes beside them.
//
// P2 (row gather): one warp per node. It walks the node's incident elements in
// element order, adds their block rows into the node's CSR rows held in shared memory
// (plain read-modify-write: within one element every target is distinct), moves
// prescribed columns into the rhs (-K_fc u_c, src/fem/assembly.cpp:95-96), adds the
// load vector, and stores its rows once with coalesced writes. In mixed precision the
// diagonal block of each element row is formed here in FP64 as minus the sum of that
// row's off-diagonal FP32 blocks, so rigid translations stay in the null space exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "cxg_internal.cuh"

namespace cxg {

namespace {

constexpr int kT1 = 128;          // P1 threads per block
constexpr int kW1 = kT1 / 32;
constexpr double kSqrt3_2v2 = 1.224744871391589;

struct TileList {
  int count;
  unsigned char r[64];
  unsigned char c[64];
};

// Node-pair tiles of TR rows x TC columns covering the upper triangle (a <= b).
constexpr TileList make_tiles(int n, int TR, int TC) {
  TileList t{};
  const int npad = (n + 3) / 4 * 4;
  for (int r = 0; r < npad / TR; ++r)
    for (int c = 0; c < npad / TC; ++c) {
      bool any = false;
      for (int i = 0; i < TR; ++i)
        for (int j = 0; j < TC; ++j) {
          const int a = TR * r + i, b = TC * c + j;
          if (a < n && b < n && a <= b) any = true;
        }
      if (any) {
        t.r[t.count] = static_cast<unsigned char>(r);
        t.c[t.count] = static_cast<unsigned char>(c);
        ++t.count;
      }
    }
  return t;
}

// Tile shapes of the element pass (TILE codes): 0 = 2x4 (default), 1 = 2x2, 2 = 4x4.
constexpr int tile_rows(int tile) { return tile == 2 ? 4 : 2; }
constexpr int tile_cols(int tile) { return tile == 1 ? 2 : 4; }

template <int ET, int TILE = 0>
struct Geo {
  static constexpr int n = nodes_of(ET);
  static constexpr int nq = gauss_of(ET);
  static constexpr int npad = (n + 3) / 4 * 4;
  static constexpr int NB = n * (n + 1) / 2;
  static constexpr int TR = tile_rows(TILE), TC = tile_cols(TILE);
  static constexpr TileList tiles = make_tiles(n, TR, TC);
  static constexpr int NT = tiles.count;
  static constexpr int EPW = NT >= 32 ? 1 : 32 / NT;
};

__host__ __device__ constexpr int blk_index(int n, int a, int b) { return a * n - a * (a - 1) / 2 + (b - a); }

// Stored 3x3 blocks are padded to 16 bytes (10 doubles, 12 floats) so that they move
// with 128-bit accesses.
template <typename R>
__host__ __device__ constexpr int blk_stride() { return sizeof(R) == 8 ? 10 : 12; }

// Slot of element e in the element buffer, a ring of `ring` elements (the whole mesh when
// the assembly runs as one window; ring_base 0): e mod ring. Every element a window's
// passes touch lies in [ring_base, ring_base + 2 ring), so one conditional subtraction
// gives the slot, with no division in the inner loops.
__device__ __forceinline__ int64_t ring_slot(int64_t e, const V2Args& V) {
  const int64_t d = e - V.ring_base;
  return d < V.ring ? d : d - V.ring;
}

template <typename R>
__device__ __forceinline__ void store_block(R* dst, const R (&v)[9]) {
  if constexpr (sizeof(R) == 8) {
    double2* d = reinterpret_cast<double2*>(dst);
    d[0] = make_double2(v[0], v[1]);
    d[1] = make_double2(v[2], v[3]);
    d[2] = make_double2(v[4], v[5]);
    d[3] = make_double2(v[6], v[7]);
    d[4] = make_double2(v[8], 0.0);
  } else {
    float4* d = reinterpret_cast<float4*>(dst);
    d[0] = make_float4(v[0], v[1], v[2], v[3]);
    d[1] = make_float4(v[4], v[5], v[6], v[7]);
    d[2] = make_float4(v[8], 0.f, 0.f, 0.f);
  }
}

template <typename R>
__device__ __forceinline__ void load_block(const R* src, R (&v)[9]) {
  if constexpr (sizeof(R) == 8) {
    const double2* d = reinterpret_cast<const double2*>(src);
    const double2 a = __ldg(d), b = __ldg(d + 1), c = __ldg(d + 2), e = __ldg(d + 3), f = __ldg(d + 4);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y; v[6] = e.x; v[7] = e.y; v[8] = f.x;
  } else {
    const float4* d = reinterpret_cast<const float4*>(src);
    const float4 a = __ldg(d), b = __ldg(d + 1), c = __ldg(d + 2);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w; v[8] = c.x;
  }
}

__device__ __forceinline__ void hardening2(const J2Mat& M, double ep, double& sy, double& h) {
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

// J2 radial return + consistent tangent (restating src/fem/plasticity.cpp:90-236), FP64.
// Returns true on the plastic branch; lam_s/mu_s/c: tangent parameters, nv: direction.
__device__ bool j2_point(const J2Mat& M, double lam, double mu_el, double mu, const double* eps, const double* cs,
                         double* ts, double* sig, double& lam_t, double& mu_t, double& c_t, double* nv,
                         double& mu_hg) {
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
  const double s_tr[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
  double xi[6];
  for (int i = 0; i < 6; ++i) xi[i] = s_tr[i] - cs[7 + i];
  const double xi_norm = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2] +
                              2.0 * (xi[3] * xi[3] + xi[4] * xi[4] + xi[5] * xi[5]));
  const double q_tr = kSqrt3_2v2 * xi_norm;
  double sy0 = 0.0, h0 = 0.0;
  if (M.plastic) hardening2(M, cs[6], sy0, h0);
  if (!M.plastic || q_tr - sy0 <= 0.0 || xi_norm == 0.0) {
    for (int i = 0; i < 6; ++i) sig[i] = st[i];
    for (int i = 0; i < kStateDoubles; ++i) ts[i] = cs[i];
    lam_t = lam;
    mu_t = mu_el;
    c_t = 0.0;
    mu_hg = mu_el;
    return 0;
  }
  const double ep0 = cs[6];
  double dgamma = 0.0;
  for (int it = 0; it < 50; ++it) {
    double sy, h_iso;
    hardening2(M, ep0 + dgamma, sy, h_iso);
    const double g = q_tr - 3.0 * mu * dgamma - M.h_kin * dgamma - sy;
    const double dg = -(3.0 * mu + M.h_kin + h_iso);
    const double step = -g / dg;
    dgamma += step;
    if (dgamma < 0.0) dgamma = 0.0;
    if (fabs(step) <= 1e-14 * (1.0 + fabs(dgamma))) break;
  }
  for (int i = 0; i < 6; ++i) nv[i] = xi[i] / xi_norm;
  const double dev_scale = 2.0 * mu * dgamma * kSqrt3_2v2;
  const double alpha_scale = (2.0 / 3.0) * M.h_kin * dgamma * kSqrt3_2v2;
  const double dep_scale = dgamma * kSqrt3_2v2;
  for (int i = 0; i < 6; ++i) {
    sig[i] = (s_tr[i] - dev_scale * nv[i]) + (i < 3 ? p : 0.0);
    ts[i] = cs[i] + dep_scale * nv[i] * (i < 3 ? 1.0 : 2.0);
    ts[7 + i] = cs[7 + i] + alpha_scale * nv[i];
  }
  ts[6] = ep0 + dgamma;
  double sy, h_iso;
  hardening2(M, ep0 + dgamma, sy, h_iso);
  const double theta = 1.0 - (2.0 * mu * dgamma * kSqrt3_2v2) / xi_norm;
  const double denom = 1.0 + (h_iso + M.h_kin) / (3.0 * mu);
  const double theta_bar = 1.0 / denom - (1.0 - theta);
  lam_t = lam + (2.0 / 3.0) * (1.0 - theta) * mu;
  mu_t = mu_el - (1.0 - theta) * mu;
  c_t = 2.0 * mu * theta_bar;
  mu_hg = mu_t - c_t * nv[3] * nv[3];
  return true;
}

// Band around the yield surface, as a fraction of the current yield stress, inside which
// the mixed-precision path decides and returns in FP64.
constexpr float kYieldBandFp32 = 1e-3f;

// J2 return of the mixed-precision path: the same steps as j2_point
// (src/fem/plasticity.cpp:90-236) with the trial stress, the local Newton on the plastic
// multiplier, the stress and history update and the consistent-tangent parameters in
// FP32. The consistency scalar f = q_tr - sigma_y(ep0) decides the branch in FP32 only
// when |f| exceeds kYieldBandFp32 * sigma_y, clear of the FP32 rounding of q_tr; points
// inside the band, and points whose FP32 Newton does not settle, take the FP64 return:
// the function then returns kJ2Fp64 and writes nothing, and the caller runs j2_point (one
// call site, so the FP64 return is inlined once). Else it returns 1 for a plastic step and
// 0 for an elastic one. The hardening table is read in FP64 (it is indexed by the FP64
// history).
constexpr int kJ2Fp64 = 2;
__device__ __forceinline__ int j2_point_mixed(const J2Mat& M, double lam, double mu_el, double mu, const double* eps,
                               const double* cs, double* ts, double* sig, double& lam_t, double& mu_t,
                               double& c_t, double* nv, double& mu_hg) {
  const float l = static_cast<float>(lam), me = static_cast<float>(mu_el), m = static_cast<float>(mu);
  const float hk = static_cast<float>(M.h_kin);
  float el[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) el[i] = static_cast<float>(eps[i] - cs[i]);
  const float l2m = l + 2.0f * me;
  float st[6];
  st[0] = l2m * el[0] + l * el[1] + l * el[2];
  st[1] = l * el[0] + l2m * el[1] + l * el[2];
  st[2] = l * el[0] + l * el[1] + l2m * el[2];
  st[3] = me * el[3];
  st[4] = me * el[4];
  st[5] = me * el[5];
  const float p = (st[0] + st[1] + st[2]) / 3.0f;
  const float s_tr[6] = {st[0] - p, st[1] - p, st[2] - p, st[3], st[4], st[5]};
  float xi[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) xi[i] = s_tr[i] - static_cast<float>(cs[7 + i]);
  const float xi_norm = sqrtf(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2] +
                              2.0f * (xi[3] * xi[3] + xi[4] * xi[4] + xi[5] * xi[5]));
  const float sq32 = static_cast<float>(kSqrt3_2v2);
  const float q_tr = sq32 * xi_norm;
  double sy0 = 0.0, h0 = 0.0;
  if (M.plastic) hardening2(M, cs[6], sy0, h0);
  const float f = q_tr - static_cast<float>(sy0);
  if (M.plastic && fabsf(f) <= kYieldBandFp32 * static_cast<float>(sy0)) return kJ2Fp64;
  if (!M.plastic || f <= 0.0f || xi_norm == 0.0f) {
#pragma unroll
    for (int i = 0; i < 6; ++i) sig[i] = st[i];
#pragma unroll
    for (int i = 0; i < kStateDoubles; ++i) ts[i] = cs[i];
    lam_t = lam;
    mu_t = mu_el;
    c_t = 0.0;
    mu_hg = mu_el;
    return 0;
  }
  const double ep0 = cs[6];
  float dgamma = 0.0f;
  bool settled = false;
  for (int it = 0; it < 50; ++it) {
    double sy, h_iso;
    hardening2(M, ep0 + dgamma, sy, h_iso);
    const float g = q_tr - 3.0f * m * dgamma - hk * dgamma - static_cast<float>(sy);
    const float dg = -(3.0f * m + hk + static_cast<float>(h_iso));
    const float step = -g / dg;
    dgamma += step;
    if (dgamma < 0.0f) dgamma = 0.0f;
    if (fabsf(step) <= 4e-7f * dgamma) {
      settled = true;
      break;
    }
  }
  if (!settled) return kJ2Fp64;
  float n32[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) n32[i] = xi[i] / xi_norm;
  const float dev_scale = 2.0f * m * dgamma * sq32;
  const float alpha_scale = (2.0f / 3.0f) * hk * dgamma * sq32;
  const float dep_scale = dgamma * sq32;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    nv[i] = n32[i];
    sig[i] = (s_tr[i] - dev_scale * n32[i]) + (i < 3 ? p : 0.0f);
    ts[i] = cs[i] + static_cast<double>(dep_scale * n32[i] * (i < 3 ? 1.0f : 2.0f));
    ts[7 + i] = cs[7 + i] + static_cast<double>(alpha_scale * n32[i]);
  }
  ts[6] = ep0 + static_cast<double>(dgamma);
  double sy, h_iso;
  hardening2(M, ep0 + dgamma, sy, h_iso);
  const float theta = 1.0f - dev_scale / xi_norm;
  const float denom = 1.0f + (static_cast<float>(h_iso) + hk) / (3.0f * m);
  const float theta_bar = 1.0f / denom - (1.0f - theta);
  const float lt = l + (2.0f / 3.0f) * (1.0f - theta) * m;
  const float mt = me - (1.0f - theta) * m;
  const float ct = 2.0f * m * theta_bar;
  lam_t = lt;
  mu_t = mt;
  c_t = ct;
  mu_hg = mt - ct * n32[3] * n32[3];
  return 1;
}

__constant__ double c_hg2[4][8] = {
    {1, 1, -1, -1, -1, -1, 1, 1},
    {1, -1, -1, 1, -1, 1, 1, -1},
    {1, -1, 1, -1, 1, -1, 1, -1},
    {-1, 1, -1, 1, 1, -1, 1, -1},
};

template <typename R>
struct Vec4;
template <>
struct Vec4<float> {
  using T = float4;
};
template <>
struct Vec4<double> {
  using T = double4;
};

// Shared-memory layout of per-(element, Gauss point) node vectors: node k lives in
// slot(k) = k/2 for even k and npad/2 + k/2 for odd k, so the row nodes 2r + i of the
// lanes' tiles occupy consecutive slots. FP32 vectors are float4 per slot; FP64 vectors
// are split in two half planes of double2 (x,y | z,0) so consecutive slots are 16 bytes
// apart. Either way one warp-wide vector load touches distinct banks. The plane block of
// each (element, Gauss point) is followed by 16 bytes of padding: the blocks then start
// 16 (mod 128) bytes apart, so the lanes of the Gauss-point phase, one block each,
// store their vectors into 8 distinct 16-byte bank groups instead of one.
__host__ __device__ constexpr int node_slot(int k, int npad) { return (k & 1) ? npad / 2 + (k >> 1) : (k >> 1); }

template <typename R, int NPAD>
struct VecIdx {
  // elements of one plane block (b = element*nq + q), padding included
  static constexpr int kBlock = NPAD * 4 + (sizeof(R) == 4 ? 4 : 2);
  // flat index of component c of the vector in `slot` of plane block b
  __device__ __forceinline__ static int at(int b, int slot, int c) {
    if (sizeof(R) == 4) return b * kBlock + slot * 4 + c;
    return b * kBlock + (c >> 1) * (NPAD * 2) + slot * 2 + (c & 1);
  }
};

// one vector store (x, y, z, 0) of a node vector
template <typename R, int NPAD>
__device__ __forceinline__ void st3(R* base, int b, int slot, double x, double y, double z) {
  if constexpr (sizeof(R) == 4) {
    *reinterpret_cast<float4*>(base + VecIdx<R, NPAD>::at(b, slot, 0)) =
        make_float4(static_cast<float>(x), static_cast<float>(y), static_cast<float>(z), 0.f);
  } else {
    *reinterpret_cast<double2*>(base + VecIdx<R, NPAD>::at(b, slot, 0)) = make_double2(x, y);
    *reinterpret_cast<double2*>(base + VecIdx<R, NPAD>::at(b, slot, 2)) = make_double2(z, 0.0);
  }
}

template <typename R, int NPAD>
__device__ __forceinline__ void ld3(const R* base, int b, int slot, R& x, R& y, R& z) {
  if (sizeof(R) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(base + VecIdx<R, NPAD>::at(b, slot, 0));
    x = v.x;
    y = v.y;
    z = v.z;
  } else {
    const double2 v = *reinterpret_cast<const double2*>(base + VecIdx<R, NPAD>::at(b, slot, 0));
    const double2 w = *reinterpret_cast<const double2*>(base + VecIdx<R, NPAD>::at(b, slot, 2));
    x = v.x;
    y = v.y;
    z = w.x;
  }
}

template <int ET, int MODE, typename R, int TILE>
struct P1Smem {
  using G = Geo<ET, TILE>;
  static constexpr int n = G::n, nq = G::nq, npad = G::npad, EPW = G::EPW;
  static constexpr bool T = MODE == MODE_TANGENT;
  static constexpr int kVec = EPW * nq * VecIdx<R, npad>::kBlock;
  static constexpr int HG = ET == C3D8R ? EPW : 1;  // hourglass data (C3D8R only)
  R g[kVec];                                      // node vectors, see VecIdx
  R nvq[T ? EPW * nq * 8 : 4];  // return direction N (Voigt, 6 used) per plastic Gauss point
  R s[EPW][nq];
  R dp[T ? EPW : 1][T ? nq : 1][4];
  double x[EPW][3 * n];
  double u[T ? EPW : 1][T ? 3 * n : 1];
  double sig[T ? EPW : 1][T ? nq : 1][6];
  double lam[EPW], mu[EPW], mu_j2[EPW];
  double gam[HG][32];
  double kappa[HG];
  double gc[HG][3 * n];
  double vol[HG];
  double mu_hg[HG];
  int plastic[EPW];
};

template <int ET, int MODE, typename R, int TILE>
constexpr size_t p1_smem_bytes() {
  using WS = P1Smem<ET, MODE, R, TILE>;
  constexpr int n = nodes_of(ET), nq = gauss_of(ET);
  return (sizeof(double) * (n * 3 * nq + nq) + 15) / 16 * 16 + kW1 * ((sizeof(WS) + 15) / 16 * 16);
}

// Resident blocks per SM the element pass asks the register allocator for: as many as
// its shared memory allows, at most 3 (<= 170 registers per thread) for the tiles whose
// accumulators fit that budget without spilling (2x2, and 2x4 in FP32), else 2 (no
// limit below the 255-register ceiling). The mixed-precision material-point pass with
// 2x2 tiles takes 4 (<= 128 registers): it spills 28 bytes per thread there and still
// ran 10 % faster on the C3D8 J2 block, where the FP64 one lost 8 % to its spills.
template <int ET, int MODE, typename R, int TILE>
constexpr int p1_min_blocks() {
  constexpr size_t per_sm = 227 * 1024;
  constexpr int by_smem = static_cast<int>(per_sm / (p1_smem_bytes<ET, MODE, R, TILE>() + 1024));
  constexpr int cap = (TILE == 1 && MODE == MODE_TANGENT && sizeof(R) == 4)   ? 4
                      : (TILE == 1 || (TILE == 0 && sizeof(R) == 4)) ? 3
                                                                     : 2;
  return by_smem < 1 ? 1 : (by_smem > cap ? cap : by_smem);
}

// J2F32 (mixed-precision material-point pass only): the J2 return in FP32
// (j2_point_mixed) instead of FP64.
// bid / nblk: this block's index among the nblk blocks that share the element range.
template <int ET, int MODE, typename R, int TILE, bool J2F32>
__device__ __forceinline__ void p1_body(const ElemArgs& A, const V2Args& V, unsigned bid, unsigned nblk) {
  using G = Geo<ET, TILE>;
  constexpr int n = G::n, nq = G::nq, npad = G::npad, EPW = G::EPW, NT = G::NT, NB = G::NB;
  constexpr int TR = G::TR, TC = G::TC;
  constexpr bool TAN = MODE == MODE_TANGENT;
  using WS = P1Smem<ET, MODE, R, TILE>;
  extern __shared__ __align__(16) unsigned char smem[];
  double* sdN = reinterpret_cast<double*>(smem);  // [n][3][nq]
  double* sw = sdN + n * 3 * nq;
  constexpr size_t cta_bytes = (sizeof(double) * (n * 3 * nq + nq) + 15) / 16 * 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WS& W = *reinterpret_cast<WS*>(smem + cta_bytes + warp * ((sizeof(WS) + 15) / 16 * 16));
  __shared__ unsigned char s_tr[64], s_tc[64];
  for (int i = threadIdx.x; i < n * 3 * nq; i += blockDim.x) sdN[i] = c_dN[dn_offset(ET) + i];
  for (int i = threadIdx.x; i < nq; i += blockDim.x) sw[i] = c_w[ET][i];
  if (threadIdx.x == 0) {
    constexpr TileList tl = make_tiles(n, TR, TC);
    for (int i = 0; i < NT; ++i) {
      s_tr[i] = tl.r[i];
      s_tc[i] = tl.c[i];
    }
  }
  // zero the padded gradient slots once; they are never written afterwards
  for (int t = lane; t < WS::kVec; t += 32) {
    W.g[t] = R(0);
  }
  __syncthreads();

  const int64_t gwarp = static_cast<int64_t>(bid) * kW1 + warp;
  const int64_t nwarps = static_cast<int64_t>(nblk) * kW1;
  const int64_t e_end = V.e_end;  // elements [V.e_begin, V.e_end) of this window
  // The connectivity of a warp's next elements is loaded while it integrates the current
  // ones, so the coordinate gather of the next iteration waits for one round of loads.
  constexpr int PA = (EPW * n + 31) / 32;
  int conn_next[PA];
  auto load_conn = [&](int64_t e0x) {
#pragma unroll
    for (int p = 0; p < PA; ++p) {
      const int t = lane + 32 * p;
      const int64_t e = e0x + t / n;
      conn_next[p] = t < EPW * n && e < e_end ? A.conn[e * n + t % n] : -1;
    }
  };
  load_conn(V.e_begin + gwarp * EPW);
  for (int64_t e0 = V.e_begin + gwarp * EPW; e0 < e_end; e0 += nwarps * EPW) {
    // ---- phase A ---------------------------------------------------------------
#pragma unroll
    for (int p = 0; p < PA; ++p) {
      const int t = lane + 32 * p;
      const int node = conn_next[p];
      if (node >= 0) {
        const int ei = t / n, k = t % n;
        for (int d = 0; d < 3; ++d) {
          W.x[ei][3 * k + d] = A.coords[3 * static_cast<int64_t>(node) + d];
          if (TAN) W.u[ei][3 * k + d] = A.u[3 * static_cast<int64_t>(node) + d];
        }
      }
    }
    load_conn(e0 + nwarps * EPW);
    if (lane < EPW) {
      const int64_t e = e0 + lane;
      const double E = e < e_end ? A.young[e] : 1.0, nu = e < e_end ? A.poisson[e] : 0.0;
      const double um2 = E / (1.0 + nu);
      W.lam[lane] = nu * um2 / (1.0 - 2.0 * nu);
      W.mu[lane] = um2 / 2.0;
      W.mu_j2[lane] = E / (2.0 * (1.0 + nu));
      W.plastic[lane] = 0;
    }
    __syncwarp();
    // ---- phase B: (element, Gauss point) tasks ----------------------------------------
    for (int t = lane; t < EPW * nq; t += 32) {
      const int ei = t / nq, q = t % nq;
      const int64_t e = e0 + ei;
      if (e >= e_end) continue;
      double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k) {
        const double d0 = sdN[(3 * k) * nq + q], d1 = sdN[(3 * k + 1) * nq + q], d2 = sdN[(3 * k + 2) * nq + q];
        for (int i = 0; i < 3; ++i) {
          const double xk = W.x[ei][3 * k + i];
          J[i][0] = fma(xk, d0, J[i][0]);
          J[i][1] = fma(xk, d1, J[i][1]);
          J[i][2] = fma(xk, d2, J[i][2]);
        }
      }
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
      const double sq = det * sw[q];
      W.s[ei][q] = static_cast<R>(sq);
      if constexpr (ET == C3D8R) W.vol[ei] = sq;
      double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < n; ++k) {
        const double d0 = sdN[(3 * k) * nq + q], d1 = sdN[(3 * k + 1) * nq + q], d2 = sdN[(3 * k + 2) * nq + q];
        double gk[3];
        for (int i = 0; i < 3; ++i) {
          gk[i] = it[i][0] * d0 + it[i][1] * d1 + it[i][2] * d2;
          if constexpr (ET == C3D8R) W.gc[ei][i * n + k] = gk[i];
        }
        st3<R, npad>(W.g, ei * nq + q, node_slot(k, npad), gk[0], gk[1], gk[2]);
        if (TAN)
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) H[i][j] = fma(W.u[ei][3 * k + i], gk[j], H[i][j]);
      }
      if (TAN) {
        const double eps[6] = {H[0][0], H[1][1], H[2][2], H[0][1] + H[1][0], H[0][2] + H[2][0], H[1][2] + H[2][1]};
        const int mat = A.elem_mat ? A.elem_mat[e] : 0;
        const int64_t gidx = e * nq + q;
        double cs[kStateDoubles], ts[kStateDoubles], sig[6], nv[6] = {0, 0, 0, 0, 0, 0};
        // plastic strain and equivalent plastic strain always; the back stress only when
        // some material moves it (state_comps 13), else it is zero
        const bool back = A.state_comps > 7;
#pragma unroll
        for (int c = 0; c < 7; ++c) cs[c] = A.state_c[c * A.n_gauss + gidx];
        if (back) {
#pragma unroll
          for (int c = 7; c < kStateDoubles; ++c) cs[c] = A.state_c[c * A.n_gauss + gidx];
        } else {
#pragma unroll
          for (int c = 7; c < kStateDoubles; ++c) cs[c] = 0.0;
        }
        double lt, mt, ct, mhg;
        // FP64 return, or with J2F32 the FP32 return (with the FP64 band near yield)
        const int r = (sizeof(R) == 8 || !J2F32) ? kJ2Fp64
                                     : j2_point_mixed(A.mats[mat], W.lam[ei], W.mu[ei], W.mu_j2[ei], eps, cs, ts, sig,
                                                      lt, mt, ct, nv, mhg);
        const bool pl = r == kJ2Fp64
                            ? j2_point(A.mats[mat], W.lam[ei], W.mu[ei], W.mu_j2[ei], eps, cs, ts, sig, lt, mt, ct, nv, mhg)
                            : r != 0;
#pragma unroll
        for (int c = 0; c < 7; ++c) A.state_t[c * A.n_gauss + gidx] = ts[c];
        if (back) {
#pragma unroll
          for (int c = 7; c < kStateDoubles; ++c) A.state_t[c * A.n_gauss + gidx] = ts[c];
        }
        for (int c = 0; c < 6; ++c) W.sig[ei][q][c] = sq * sig[c];
        W.dp[ei][q][0] = static_cast<R>(sq * lt);
        W.dp[ei][q][1] = static_cast<R>(sq * mt);
        W.dp[ei][q][2] = static_cast<R>(sq * ct);
        if (pl) {
          W.plastic[ei] = 1;
#pragma unroll
          for (int c = 0; c < 6; ++c) W.nvq[(ei * nq + q) * 8 + c] = static_cast<R>(nv[c]);
        }
        if constexpr (ET == C3D8R) {
          if (q == nq - 1) W.mu_hg[ei] = mhg;
        }
      }
    }
    __syncwarp();
    // ---- C3D8R hourglass vectors (src/fem/element.cpp:545-579) ------------------------
    if constexpr (ET == C3D8R) {
      for (int t = lane; t < EPW * 4; t += 32) {
        const int ei = t / 4, al = t % 4;
        double gx[3] = {0, 0, 0};
        for (int j = 0; j < 8; ++j)
          for (int d = 0; d < 3; ++d) gx[d] += c_hg2[al][j] * W.x[ei][3 * j + d];
        for (int j = 0; j < 8; ++j) {
          double corr = 0.0;
          for (int d = 0; d < 3; ++d) corr += gx[d] * W.gc[ei][d * n + j];
          W.gam[ei][al * 8 + j] = c_hg2[al][j] - corr;
        }
      }
      if (lane < EPW) {
        double b2 = 0.0;
        for (int t = 0; t < 3 * n; ++t) b2 += W.gc[lane][t] * W.gc[lane][t];
        W.kappa[lane] = 0.05 * (TAN ? W.mu_hg[lane] : W.mu_j2[lane]) * W.vol[lane] * b2;
      }
      __syncwarp();
    }
    // ---- phase C: TR x TC node-pair tiles ---------------------------------------------
    // Staged stores (FP64 linear mode, one tile per lane, the element's blocks fit the
    // gradient area): once every tile is done the gradient vectors are dead, so the lanes
    // put their blocks there unpadded and the warp writes the padded element buffer with
    // consecutive 16-byte stores, instead of every lane writing its own 80-byte blocks
    // across the element's buffer (about one cache line per lane and store instruction).
    // Measured on C3D20 64^3: FP64 6.25 -> 6.10 ms per assembly; in FP32 the staging
    // raised the 2x4 tile's registers from 126 to 168 and lost, so FP32 stores directly.
    constexpr bool STAGE =
        MODE == MODE_LINEAR && sizeof(R) == 8 && EPW * NT <= 32 && EPW * NB * 9 <= WS::kVec;
    R acc[TR][TC][9];
    for (int task = lane; task < EPW * NT; task += 32) {
      const int ei = task / NT, ti = task % NT;
      const int64_t e = e0 + ei;
      if (e < e_end) {
        const int a0 = TR * s_tr[ti], b0 = TC * s_tc[ti];
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
          for (int j = 0; j < TC; ++j)
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[i][j][k] = R(0);
        const bool pl = TAN && W.plastic[ei];
        if (!pl) {
#pragma unroll 3
          for (int q = 0; q < nq; ++q) {
            const R s = W.s[ei][q];
            R ga[TR][3], gb[TC][3];
#pragma unroll
            for (int i = 0; i < TR; ++i) {
              ld3<R, npad>(W.g, ei * nq + q, node_slot(a0 + i, npad), ga[i][0], ga[i][1], ga[i][2]);
              ga[i][0] *= s;
              ga[i][1] *= s;
              ga[i][2] *= s;
            }
#pragma unroll
            for (int j = 0; j < TC; ++j)
              ld3<R, npad>(W.g, ei * nq + q, node_slot(b0 + j, npad), gb[j][0], gb[j][1], gb[j][2]);
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
              for (int j = 0; j < TC; ++j)
#pragma unroll
                for (int x = 0; x < 3; ++x)
#pragma unroll
                  for (int y = 0; y < 3; ++y) acc[i][j][3 * x + y] += ga[i][x] * gb[j][y];
          }
          const R lam = static_cast<R>(W.lam[ei]), mu = static_cast<R>(W.mu[ei]);
#pragma unroll
          for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
              R Gm[9];
#pragma unroll
              for (int k = 0; k < 9; ++k) Gm[k] = acc[i][j][k];
              const R tr = Gm[0] + Gm[4] + Gm[8];
#pragma unroll
              for (int x = 0; x < 3; ++x)
#pragma unroll
                for (int y = 0; y < 3; ++y)
                  acc[i][j][3 * x + y] = lam * Gm[3 * x + y] + mu * Gm[3 * y + x] + (x == y ? mu * tr : R(0));
            }
        } else if (TAN) {
          for (int q = 0; q < nq; ++q) {
            const R sl = W.dp[ei][q][0], sm = W.dp[ei][q][1], sc = W.dp[ei][q][2];
            R ga[TR][3], gb[TC][3];
#pragma unroll
            for (int i = 0; i < TR; ++i)
              ld3<R, npad>(W.g, ei * nq + q, node_slot(a0 + i, npad), ga[i][0], ga[i][1], ga[i][2]);
#pragma unroll
            for (int j = 0; j < TC; ++j)
              ld3<R, npad>(W.g, ei * nq + q, node_slot(b0 + j, npad), gb[j][0], gb[j][1], gb[j][2]);
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
              for (int j = 0; j < TC; ++j) {
                const R dot = sm * (ga[i][0] * gb[j][0] + ga[i][1] * gb[j][1] + ga[i][2] * gb[j][2]);
#pragma unroll
                for (int x = 0; x < 3; ++x)
#pragma unroll
                  for (int y = 0; y < 3; ++y)
                    acc[i][j][3 * x + y] += (sl * ga[i][x]) * gb[j][y] + (sm * gb[j][x]) * ga[i][y] + (x == y ? dot : R(0));
              }
            if (sc != R(0)) {
              // m = N g for the tile's nodes, from the stored return direction
              const R* N = W.nvq + (ei * nq + q) * 8;
              const R n0 = N[0], n1 = N[1], n2 = N[2], n3 = N[3], n4 = N[4], n5 = N[5];
              R ma[TR][3], mb[TC][3];
#pragma unroll
              for (int i = 0; i < TR; ++i) {
                ma[i][0] = n0 * ga[i][0] + n3 * ga[i][1] + n4 * ga[i][2];
                ma[i][1] = n3 * ga[i][0] + n1 * ga[i][1] + n5 * ga[i][2];
                ma[i][2] = n4 * ga[i][0] + n5 * ga[i][1] + n2 * ga[i][2];
              }
#pragma unroll
              for (int j = 0; j < TC; ++j) {
                mb[j][0] = n0 * gb[j][0] + n3 * gb[j][1] + n4 * gb[j][2];
                mb[j][1] = n3 * gb[j][0] + n1 * gb[j][1] + n5 * gb[j][2];
                mb[j][2] = n4 * gb[j][0] + n5 * gb[j][1] + n2 * gb[j][2];
              }
#pragma unroll
              for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j)
#pragma unroll
                  for (int x = 0; x < 3; ++x)
#pragma unroll
                    for (int y = 0; y < 3; ++y) acc[i][j][3 * x + y] -= (sc * ma[i][x]) * mb[j][y];
            }
          }
        }
        if constexpr (!STAGE) {
          R* out = reinterpret_cast<R*>(V.edata) + ring_slot(e, V) * (NB * blk_stride<R>());
#pragma unroll
          for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
              const int a = a0 + i, b = b0 + j;
              if (a < n && b < n && a <= b) {
                R h = R(0);
                if constexpr (ET == C3D8R) {
                  double hd = 0.0;
                  for (int al = 0; al < 4; ++al) hd += W.gam[ei][al * 8 + a] * W.gam[ei][al * 8 + b];
                  h = static_cast<R>(hd * W.kappa[ei]);
                }
                R bv[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) bv[k] = acc[i][j][k] + ((k % 4 == 0) ? h : R(0));
                store_block<R>(out + blk_index(n, a, b) * blk_stride<R>(), bv);
              }
            }
        }
      }
    }
    if constexpr (STAGE) {
      static_assert(ET != C3D8R, "staged stores carry no hourglass term");
      constexpr int BS = blk_stride<R>(), PER = 16 / static_cast<int>(sizeof(R)), CPB = BS / PER;
      __syncwarp();  // every lane is done reading the gradient vectors
      R* stg = W.g;  // EPW x NB blocks of 9 values
      if (lane < EPW * NT) {
        const int ei = lane / NT, ti = lane % NT;
        if (e0 + ei < e_end) {
          const int a0 = TR * s_tr[ti], b0 = TC * s_tc[ti];
#pragma unroll
          for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) {
              const int a = a0 + i, b = b0 + j;
              if (a < n && b < n && a <= b) {
                R* d = stg + (ei * NB + blk_index(n, a, b)) * 9;
#pragma unroll
                for (int k = 0; k < 9; ++k) d[k] = acc[i][j][k];
              }
            }
        }
      }
      __syncwarp();
      for (int ei = 0; ei < EPW && e0 + ei < e_end; ++ei) {
        R* out = reinterpret_cast<R*>(V.edata) + ring_slot(e0 + ei, V) * (NB * BS);
        const R* sb = stg + ei * NB * 9;
        for (int pc = lane; pc < NB * CPB; pc += 32) {
          const int k = pc / CPB, part = pc % CPB;
          R v[4];
#pragma unroll
          for (int t = 0; t < PER; ++t) {
            const int j = part * PER + t;
            v[t] = j < 9 ? sb[k * 9 + j] : R(0);
          }
          if constexpr (sizeof(R) == 4) {
            *reinterpret_cast<float4*>(out + k * BS + part * PER) = make_float4(v[0], v[1], v[2], v[3]);
          } else {
            *reinterpret_cast<double2*>(out + k * BS + part * PER) = make_double2(v[0], v[1]);
          }
        }
      }
      __syncwarp();  // the next elements' Gauss-point phase rewrites the gradient area
    }
    // ---- phase D: internal force per element (material-point mode) --------------------
    if (TAN) {
      for (int t = lane; t < EPW * n; t += 32) {
        const int ei = t / n, a = t % n;
        const int64_t e = e0 + ei;
        if (e >= e_end) continue;
        double f[3] = {0, 0, 0};
        for (int q = 0; q < nq; ++q) {
          const double* S = W.sig[ei][q];
          R rx, ry, rz;
          ld3<R, npad>(W.g, ei * nq + q, node_slot(a, npad), rx, ry, rz);
          const double gx = rx, gy = ry, gz = rz;
          f[0] += S[0] * gx + S[3] * gy + S[4] * gz;
          f[1] += S[3] * gx + S[1] * gy + S[5] * gz;
          f[2] += S[4] * gx + S[5] * gy + S[2] * gz;
        }
        if constexpr (ET == C3D8R) {
          for (int al = 0; al < 4; ++al) {
            double gu[3] = {0, 0, 0};
            for (int j = 0; j < 8; ++j)
              for (int d = 0; d < 3; ++d) gu[d] += W.gam[ei][al * 8 + j] * W.u[ei][3 * j + d];
            const double ka = W.kappa[ei] * W.gam[ei][al * 8 + a];
            for (int d = 0; d < 3; ++d) f[d] += ka * gu[d];
          }
        }
        for (int d = 0; d < 3; ++d) V.fdata[ring_slot(e, V) * (3 * n) + 3 * a + d] = f[d];
      }
    }
    __syncwarp();
  }
}

template <int ET, int MODE, typename R, int TILE, bool J2F32>
__global__ void __launch_bounds__(kT1, (p1_min_blocks<ET, MODE, R, TILE>())) p1_kernel(ElemArgs A, V2Args V) {
  p1_body<ET, MODE, R, TILE, J2F32>(A, V, blockIdx.x, gridDim.x);
}

// ---- P2: row gather ------------------------------------------------------------------
// One warp per node a. The node's three rows are staged in shared memory at full width:
// row i holds 3 entries for each node of a's adjacency list (position s, from the
// element slot map), every component, free or not. Lanes form EG groups of GS lanes
// (GS = 16 for elements of at most 16 nodes, else 32); lane lb of group s handles column node lb of incident element
// k + s, so EG elements are applied per pass, each group into its own copy of the rows
// (within one element every target is distinct: plain adds, no atomics). The inner
// loop is one block fetch and 9 adds per lane. Every group copy is zeroed and read once
// per node, which for the short rows of the <= 8-node families costs more shared-memory
// traffic than the idle lanes of two 16-lane groups (measured on the C3D8 tangent
// gather, two groups against four: FP64 10 %, mixed 12 % faster). The epilogue
// reads every staged entry as the sum of the group copies in group order, and
//  - in mixed precision forms the diagonal block of node a as minus the FP64 sum of
//    all off-diagonal FP32 blocks in its rows (27 lanes: 9 entries x 3 phases, added in
//    a fixed order), so rigid translations stay in the null space of K to FP64 accuracy;
//  - stores the free rows: interior nodes (every neighbour fully free) as staged, with
//    coalesced writes; the others lane by neighbour, at the compressed columns a warp
//    scan of the neighbours' free-component counts gives, moving the prescribed
//    columns into the rhs (-K_fc u_c, src/fem/assembly.cpp:95-96).
// The node's incident-element codes come in with one coalesced load per 32 elements and
// are handed out by shuffles.
template <int ET, bool DIAGFIX>
struct P2Geo {
  static constexpr int n = nodes_of(ET);
  static constexpr int GS = n <= 16 ? 16 : 32;
  static constexpr int EG = 32 / GS;
  // lanes n .. n + 2 of a group are idle in the block loop and gather the three
  // components of the element forces (all families but C3D15, whose 16-lane groups
  // leave one lane, and whose diagonal-block lane takes them)
  static constexpr bool FIDLE = n + 3 <= GS;
};

template <typename R>
struct P2Pass {
  double v[9];
  int64_t e;
  int la, slotv;
  bool active;
};

template <int ET, typename R, bool WIN>
__device__ __forceinline__ void p2_fetch(const ElemArgs& A, const V2Args& V, const R* ed, int code, bool active,
                                         int lb, P2Pass<R>& p) {
  constexpr int n = nodes_of(ET), NB = n * (n + 1) / 2;
  p.active = active;
  p.e = code / n;
  p.la = code % n;
  if (active) {
    p.slotv = __ldg(A.slot + (p.e * n + p.la) * n + lb);
    const bool tr = lb < p.la;
    R raw[9];
    load_block<R>(ed + (WIN ? ring_slot(p.e, V) : p.e) * (NB * blk_stride<R>()) +
                      (tr ? blk_index(n, lb, p.la) : blk_index(n, p.la, lb)) * blk_stride<R>(),
                  raw);
#pragma unroll
    for (int q = 0; q < 9; ++q) p.v[q] = static_cast<double>(tr ? raw[3 * (q % 3) + q / 3] : raw[q]);
  } else {
    p.slotv = 0;
#pragma unroll
    for (int q = 0; q < 9; ++q) p.v[q] = 0.0;
  }
}

template <int ET, bool TAN, typename R, bool DIAGFIX, bool WIN>
__device__ __forceinline__ void p2_body(const ElemArgs& A, const V2Args& V, unsigned bid, unsigned nblk) {
  constexpr int n = nodes_of(ET);
  constexpr int GS = P2Geo<ET, DIAGFIX>::GS, EG = P2Geo<ET, DIAGFIX>::EG;
  constexpr unsigned kAll = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int stride = static_cast<int>(V.row_stride);  // doubles of one row-buffer copy
  double* buf = reinterpret_cast<double*>(smem) + warp * (EG * stride);
  const int64_t gwarp = static_cast<int64_t>(bid) * (blockDim.x >> 5) + warp;
  const int64_t nwarps = static_cast<int64_t>(nblk) * (blockDim.x >> 5);
  const R* ed = reinterpret_cast<const R*>(V.edata);
  const int sub = lane / GS, lb = lane % GS;
  const bool lane_ok = lb < n;
  double* mine = buf + sub * stride;
  // nodes [V.n_begin, V.n_end) of this window's node list (node_order, WIN), or of the mesh
  const int64_t n_begin = WIN ? V.n_begin : 0, n_end = WIN ? V.n_end : A.n_nodes;
  // per-node scalars, all loaded at the node's start
  struct NodeInfo {
    int64_t a, i0, i1, base;
    int ma, L, K;
  };
  auto node_info = [&](int64_t idx) {
    NodeInfo t;
    t.a = WIN ? static_cast<int64_t>(V.node_order[idx]) : idx;
    t.ma = A.node_mask[t.a];
    t.K = A.adj_len[t.a];
    t.i0 = V.inc_ptr[t.a];
    t.i1 = V.inc_ptr[t.a + 1];
    t.base = A.node_base[t.a];
    t.L = static_cast<int>(A.node_rowlen[t.a]);
    return t;
  };
  for (int64_t idx = n_begin + gwarp; idx < n_end; idx += nwarps) {
    const NodeInfo cur_node = node_info(idx);
    const int64_t a = cur_node.a;
    const int ma = cur_node.ma;
    const int K = cur_node.K;  // neighbours, a itself included
    const int W = 3 * K;                               // full-width row length
    const int total = 3 * W;
    const int64_t i0 = cur_node.i0, i1 = cur_node.i1;
    const int L = cur_node.L;
    // every copy starts 16-byte aligned (stride is even) and holds at least total + 1
    // doubles when total is odd
    for (int g = 0; g < EG; ++g)
      for (int t = lane; 2 * t < total; t += 32)
        reinterpret_cast<double2*>(buf + g * stride)[t] = make_double2(0.0, 0.0);
    __syncwarp();
    constexpr bool FIDLE = P2Geo<ET, DIAGFIX>::FIDLE;
    // a's internal force: component lb - n on lanes lb = n .. n + 2 (FIDLE), else all
    // three on the lane of each element's diagonal block
    double fs[FIDLE ? 1 : 3] = {};
    int slot_aa = 0;  // position of node a in its own adjacency list (DIAGFIX)
    for (int64_t c0 = i0; c0 < i1; c0 += 32) {
      const int cnt = static_cast<int>(i1 - c0 < 32 ? i1 - c0 : 32);
      const int code_l = lane < cnt ? __ldg(V.inc_code + c0 + lane) : 0;
      for (int k = 0; k < cnt; k += EG) {
        P2Pass<R> cur;
        p2_fetch<ET, R, WIN>(A, V, ed, __shfl_sync(kAll, code_l, (k + sub) & 31), lane_ok && k + sub < cnt, lb, cur);
        if (cur.active && (!DIAGFIX || lb != cur.la)) {
          double* c = mine + 3 * cur.slotv;
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            c[i * W] += cur.v[3 * i];
            c[i * W + 1] += cur.v[3 * i + 1];
            c[i * W + 2] += cur.v[3 * i + 2];
          }
        }
        if constexpr (TAN && FIDLE) {
          if (lb >= n && lb < n + 3 && k + sub < cnt)
            fs[0] += __ldg(V.fdata + (WIN ? ring_slot(cur.e, V) : cur.e) * (3 * n) + 3 * cur.la + (lb - n));
        } else if constexpr (TAN) {
          if (cur.active && lb == cur.la)
#pragma unroll
            for (int d = 0; d < 3; ++d)
              fs[d] += __ldg(V.fdata + (WIN ? ring_slot(cur.e, V) : cur.e) * (3 * n) + 3 * cur.la + d);
        }
        if (DIAGFIX && cur.active && lb == cur.la) slot_aa = cur.slotv;
        __syncwarp();
      }
    }
    // staged entry t: the group copies summed in group order
    auto staged = [&](int t) {
      double v = buf[t];
#pragma unroll
      for (int g = 1; g < EG; ++g) v += buf[g * stride + t];
      return v;
    };
    if (DIAGFIX) {
      // diagonal block of node a: minus the FP64 sum of every off-diagonal block in its
      // rows. Lane 9 p + q (p < 3) sums entry q of the blocks of neighbours p, p + 3,
      // ... in neighbour order; lane q then adds the three phases in phase order.
      slot_aa = static_cast<int>(__reduce_max_sync(kAll, static_cast<unsigned>(slot_aa)));
      const int q = lane % 9, p = lane / 9, qi = q / 3, qj = q - 3 * qi;
      double d = 0.0;
      if (p < 3)
        for (int s = p; s < K; s += 3)
          if (s != slot_aa) d += staged(qi * W + 3 * s + qj);
      const double d1 = __shfl_sync(kAll, d, (lane + 9) & 31), d2 = __shfl_sync(kAll, d, (lane + 18) & 31);
      if (lane < 9 && i1 > i0) buf[qi * W + 3 * slot_aa + qj] = -((d + d1) + d2);
      __syncwarp();
    }
    // Interior nodes (every neighbour fully free, L == W) store the staged rows as they
    // are, coalesced. At the others each lane takes a neighbour: a warp scan of the
    // neighbours' free-component counts gives its first compressed column, its free
    // columns are stored there and its prescribed columns go to the rhs.
    double rr[3] = {0.0, 0.0, 0.0};
    double* orow0 = A.vals + cur_node.base;
    if (L == W) {
      double* orow = orow0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (!((ma >> i) & 1)) continue;
        for (int c = lane; c < L; c += 32) {
          const double v = staged(i * W + c);
          orow[c] = V.accumulate ? orow[c] + v : v;
        }
        orow += L;
      }
    } else {
      const int32_t* nbr = A.bnd_node + A.bnd_ptr[a];
      int carry = 0;
      for (int s0 = 0; s0 < K; s0 += 32) {
        const int s = s0 + lane;
        const bool ok = s < K;
        const int b = ok ? __ldg(nbr + s) : 0;
        const int mb = ok ? static_cast<int>(A.node_mask[b]) : 0;
        const int pc = __popc(mb);
        int incl = pc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int y = __shfl_up_sync(kAll, incl, off);
          if (lane >= off) incl += y;
        }
        const int c = carry + incl - pc;
        carry += __shfl_sync(kAll, incl, 31);
        if (ok) {
#pragma unroll
          for (int jj = 0; jj < 3; ++jj) {
            if ((mb >> jj) & 1) {
              const int col = c + __popc(mb & ((1 << jj) - 1));
              int ri = 0;
#pragma unroll
              for (int i = 0; i < 3; ++i) {
                if (!((ma >> i) & 1)) continue;
                double* o = orow0 + static_cast<int64_t>(ri) * L + col;
                const double v = staged(i * W + 3 * s + jj);
                *o = V.accumulate ? *o + v : v;
                ++ri;
              }
            } else {
              const double pv = A.prescribed[3 * static_cast<int64_t>(b) + jj];
              if (pv != 0.0) {
#pragma unroll
                for (int i = 0; i < 3; ++i) rr[i] -= staged(i * W + 3 * s + jj) * pv;
              }
            }
          }
        }
      }
    }
    if (A.rhs) {
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        double v = rr[r];
        // interior nodes have no prescribed columns: every lane's term is +0.0
        if (L != W)
          for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kAll, v, off);
        if (lane == 0 && ((ma >> r) & 1)) {
          const int64_t eq = A.node_eq0[a] + __popc(ma & ((1 << r) - 1));
          const double prev = V.accumulate ? A.rhs[eq] : (V.f_ext ? V.f_ext[3 * a + r] : 0.0);
          A.rhs[eq] = prev + v;
        }
      }
    }
    if (TAN && A.f_int) {
      if constexpr (FIDLE) {
        // group partials (each in incidence order) added in group order
        double v = fs[0];
#pragma unroll
        for (int g = 1; g < EG; ++g) v += __shfl_sync(kAll, fs[0], (lane + g * GS) & 31);
        if (lane >= n && lane < n + 3) {
          const int d = lane - n;
          A.f_int[3 * a + d] = (V.accumulate ? A.f_int[3 * a + d] : 0.0) + v;
        }
      } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double v = fs[d];
          for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kAll, v, off);
          if (lane == 0) A.f_int[3 * a + d] = (V.accumulate ? A.f_int[3 * a + d] : 0.0) + v;
        }
      }
    }
    __syncwarp();
  }
}

// Blocks of at most 8 warps, compiled without a register budget (48-72 registers).
// WIN: the windowed schedule (node list and element ring); the one-window gather is
// compiled without either, so it keeps the registers of a plain node loop.
template <int ET, bool TAN, typename R, bool DIAGFIX, bool WIN>
__global__ void p2_kernel(ElemArgs A, V2Args V) {
  p2_body<ET, TAN, R, DIAGFIX, WIN>(A, V, blockIdx.x, gridDim.x);
}

// The gather of the <= 8-node families, compiled for 5 resident 8-warp blocks per SM
// (<= 48 registers): their row buffers are small, so registers, not shared memory, bound
// their resident warps, and the latency-bound gather runs faster with more of them.
template <int ET, bool TAN, typename R, bool DIAGFIX, bool WIN>
__global__ void __launch_bounds__(256, 5) p2_kernel_small(ElemArgs A, V2Args V) {
  p2_body<ET, TAN, R, DIAGFIX, WIN>(A, V, blockIdx.x, gridDim.x);
}

int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Persistent grid: blocks_per_sm (0 = as many as are resident) blocks on every SM,
// capped by the work available.
int64_t persistent_grid(int64_t need, int resident, int blocks_per_sm) {
  const int per_sm = blocks_per_sm > 0 ? std::min(blocks_per_sm, std::max(resident, 1)) : std::max(resident, 1);
  return std::max<int64_t>(1, std::min<int64_t>(need, static_cast<int64_t>(per_sm) * sm_count()));
}

template <int ET, int MODE, typename R, int TILE>
cudaError_t launch_p1_tile(const ElemArgs& a, const V2Args& v, const LaunchCfg& cfg, cudaStream_t s) {
  constexpr size_t smem = p1_smem_bytes<ET, MODE, R, TILE>();
  static_assert(smem <= 227 * 1024, "element pass shared memory");
  auto kern = p1_kernel<ET, MODE, R, TILE, false>;
  if constexpr (MODE == MODE_TANGENT && sizeof(R) == 4) {
    if (cfg.j2_fp32) kern = p1_kernel<ET, MODE, R, TILE, true>;
  }
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kT1, smem);
  if (err != cudaSuccess) return err;
  constexpr int EPW = Geo<ET, TILE>::EPW;
  const int64_t count = v.e_end - v.e_begin;
  const int64_t need = (count + kW1 * EPW - 1) / (kW1 * EPW);
  const int64_t grid = persistent_grid(need, per_sm, cfg.p1_blocks_per_sm);
  if (count <= 0) return cudaSuccess;
  kern<<<static_cast<unsigned>(grid), kT1, smem, s>>>(a, v);
  return cudaGetLastError();
}

// Tile shapes instantiated: 2x4 and 2x2 everywhere, 4x4 in the linear pass with FP32
// accumulators.
template <int ET, int MODE, typename R>
cudaError_t launch_p1_t(const ElemArgs& a, const V2Args& v, const LaunchCfg& cfg, cudaStream_t s) {
  if (cfg.tile == 1) return launch_p1_tile<ET, MODE, R, 1>(a, v, cfg, s);
  if constexpr (MODE == MODE_LINEAR && sizeof(R) == 4) {
    if (cfg.tile == 2) return launch_p1_tile<ET, MODE, R, 2>(a, v, cfg, s);
  }
  if (cfg.tile != 0) return cudaErrorInvalidValue;
  return launch_p1_tile<ET, MODE, R, 0>(a, v, cfg, s);
}

template <int ET, bool TAN, typename R, bool DF>
cudaError_t launch_p2_t(const ElemArgs& a, V2Args v, const LaunchCfg& cfg, cudaStream_t s) {
  auto kern = v.node_order ? p2_kernel<ET, TAN, R, DF, true> : p2_kernel<ET, TAN, R, DF, false>;
  if constexpr (nodes_of(ET) <= 8)
    kern = v.node_order ? p2_kernel_small<ET, TAN, R, DF, true> : p2_kernel_small<ET, TAN, R, DF, false>;
  // warps per block: as many as fit in ~160 KB of row buffers, up to 8 (or the
  // configured count when it fits). Per warp: EG full-width copies of three rows of
  // 3 x max_adj doubles. (Shared memory beyond that comes out of the L1 cache the
  // scattered block loads reuse.)
  const int64_t stride = std::max<int64_t>(2, (9 * v.max_adj + 1) / 2 * 2);
  const int64_t wbytes = P2Geo<ET, DF>::EG * stride * 8;
  int warps = cfg.p2_warps > 0 ? std::min(cfg.p2_warps, 8) : 8;
  while (warps > 1 && warps * wbytes > 160 * 1024) warps /= 2;
  const size_t smem = static_cast<size_t>(warps) * wbytes;
  if (smem > 220 * 1024) return cudaErrorInvalidConfiguration;
  v.row_stride = stride;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem);
  if (err != cudaSuccess) return err;
  const int64_t count = v.n_end - v.n_begin;
  if (count <= 0) return cudaSuccess;
  const int64_t need = (count + warps - 1) / warps;
  const int64_t grid = persistent_grid(need, per_sm, cfg.p2_blocks_per_sm);
  kern<<<static_cast<unsigned>(grid), warps * 32, smem, s>>>(a, v);
  return cudaGetLastError();
}

template <int ET>
cudaError_t launch_v2_pair(int mode, int precision, const ElemArgs& a, const V2Args& v, const LaunchCfg& c,
                           cudaStream_t s);

// Every window's element pass and row gather in order on one stream: the row gather of
// window w reads element blocks that stay in the ring (and in L2) until the element
// pass of window w+1 overwrites the slots of elements no later node needs.
template <int ET>
cudaError_t launch_v2_type(int mode, int precision, const ElemArgs& a, const V2Args& v, const LaunchCfg& c,
                           cudaStream_t s) {
  if (v.n_win <= 1) return launch_v2_pair<ET>(mode, precision, a, v, c, s);
  V2Args w = v;
  for (int32_t k = 0; k < v.n_win; ++k) {
    w.e_begin = v.win_e[k];
    w.e_end = v.win_e[k + 1];
    // both passes of window k touch elements in [e_end - ring, e_end) only
    const int64_t lo = std::max<int64_t>(0, w.e_end - v.ring);
    w.ring_base = lo / v.ring * v.ring;
    w.n_begin = v.win_n[k];
    w.n_end = v.win_n[k + 1];
    const cudaError_t err = launch_v2_pair<ET>(mode, precision, a, w, c, s);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

template <int ET>
cudaError_t launch_v2_pair(int mode, int precision, const ElemArgs& a, const V2Args& v, const LaunchCfg& c,
                           cudaStream_t s) {
  cudaError_t err = cudaSuccess;
  if (mode == MODE_LINEAR) {
    if (c.passes & 1)
      err = precision ? launch_p1_t<ET, MODE_LINEAR, float>(a, v, c, s) : launch_p1_t<ET, MODE_LINEAR, double>(a, v, c, s);
    if (err != cudaSuccess || !(c.passes & 2)) return err;
    return precision ? launch_p2_t<ET, false, float, true>(a, v, c, s) : launch_p2_t<ET, false, double, false>(a, v, c, s);
  }
  if (c.passes & 1)
    err = precision ? launch_p1_t<ET, MODE_TANGENT, float>(a, v, c, s) : launch_p1_t<ET, MODE_TANGENT, double>(a, v, c, s);
  if (err != cudaSuccess || !(c.passes & 2)) return err;
  return precision ? launch_p2_t<ET, true, float, true>(a, v, c, s) : launch_p2_t<ET, true, double, false>(a, v, c, s);
}

// ---- scalar-block element pass (mass, geometric stiffness) ---------------------------
// Every 3x3 block of these operators is a scalar times I: m_ab = sum_q rho detJ w N_a N_b
// (element_mass, src/fem/element.cpp:786-812), its row sums on the diagonal for the
// lumped mass (element.cpp:814-831), k_ab = sum_q detJ w g_a . sigma_q . g_b
// (element_geometric_stiffness + accumulate_kgeo, element.cpp:482-508, 833-854). One
// warp per element: lanes take Gauss points for detJ (and the gradients), then node
// pairs (a <= b) for the scalar sums; the blocks go to the FP64 element buffer the row
// gather reads. The conduction matrix k_ab = sum_q k detJ w g_a . g_b
// (element_conduction, element.cpp:745-765) has the same shape and takes kind 4; its
// plan carries the temperature as component 0 of every node.
constexpr int kScalarWarps = 4;

template <int ET, int KIND>
constexpr int scalar_warp_doubles() {
  constexpr int n = nodes_of(ET), nq = gauss_of(ET);
  return 3 * n + nq + (KIND >= 3 ? nq * n * 3 : 0) + (KIND == 3 ? nq * 6 : 0);
}

template <int ET, int KIND>
__global__ void __launch_bounds__(kScalarWarps * 32) scalar_kernel(ElemArgs A, V2Args V, const double* density,
                                                                   const double* gp_stress) {
  constexpr int n = nodes_of(ET), nq = gauss_of(ET), NB = n * (n + 1) / 2;
  constexpr bool GEO = KIND == 3, GRAD = KIND >= 3;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned char s_pa[NB], s_pb[NB];
  for (int p = threadIdx.x; p < NB; p += blockDim.x) {
    int a = 0, r = p;
    while (r >= n - a) {
      r -= n - a;
      ++a;
    }
    s_pa[p] = static_cast<unsigned char>(a);
    s_pb[p] = static_cast<unsigned char>(a + r);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* x = reinterpret_cast<double*>(smem) + warp * scalar_warp_doubles<ET, KIND>();
  double* sq = x + 3 * n;   // [nq] rho detJ w (mass), detJ w (geometric), k detJ w (conduction)
  double* g = sq + nq;      // [nq][n][3] physical gradients (geometric)
  double* sig = g + nq * n * 3;  // [nq][6] stress (geometric)
  const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kScalarWarps + warp;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kScalarWarps;
  for (int64_t e = gwarp; e < A.n_elems; e += nwarps) {
    for (int t = lane; t < 3 * n; t += 32) x[t] = A.coords[3 * static_cast<int64_t>(A.conn[e * n + t / 3]) + t % 3];
    __syncwarp();
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
      if (!GRAD) {
        sq[q] = density[e] * det * c_w[ET][q];
      } else {
        sq[q] = GEO ? det * c_w[ET][q] : density[e] * det * c_w[ET][q];
        const double inv = 1.0 / det;
        const double it[3][3] = {
            {c00 * inv, c01 * inv, c02 * inv},
            {(J[0][2] * J[2][1] - J[0][1] * J[2][2]) * inv, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv,
             (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * inv},
            {(J[0][1] * J[1][2] - J[0][2] * J[1][1]) * inv, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * inv,
             (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv}};
        for (int k = 0; k < n; ++k) {
          const double d0 = c_dN[dn_offset(ET) + (3 * k) * nq + q], d1 = c_dN[dn_offset(ET) + (3 * k + 1) * nq + q],
                       d2 = c_dN[dn_offset(ET) + (3 * k + 2) * nq + q];
          for (int i = 0; i < 3; ++i) g[(q * n + k) * 3 + i] = it[i][0] * d0 + it[i][1] * d1 + it[i][2] * d2;
        }
        if (GEO)
          for (int c = 0; c < 6; ++c) sig[q * 6 + c] = gp_stress ? gp_stress[(e * nq + q) * 6 + c] : 0.0;
      }
    }
    __syncwarp();
    double* out = reinterpret_cast<double*>(V.edata) + e * (NB * blk_stride<double>());
    for (int p = lane; p < NB; p += 32) {
      const int a = s_pa[p], b = s_pb[p];
      double val = 0.0;
      if (KIND == 1) {
        for (int q = 0; q < nq; ++q) val += sq[q] * c_N[nn_offset(ET) + a * nq + q] * c_N[nn_offset(ET) + b * nq + q];
      } else if (KIND == 2) {
        if (a == b)
          for (int bb = 0; bb < n; ++bb) {
            double m = 0.0;
            for (int q = 0; q < nq; ++q)
              m += sq[q] * c_N[nn_offset(ET) + a * nq + q] * c_N[nn_offset(ET) + bb * nq + q];
            val += m;
          }
      } else if (KIND == 4) {
        for (int q = 0; q < nq; ++q) {
          const double* ga = g + (q * n + a) * 3;
          const double* gb = g + (q * n + b) * 3;
          val += sq[q] * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
        }
      } else {
        for (int q = 0; q < nq; ++q) {
          const double* ga = g + (q * n + a) * 3;
          const double* gb = g + (q * n + b) * 3;
          const double* sg = sig + q * 6;
          const double se = sg[0] * ga[0] * gb[0] + sg[1] * ga[1] * gb[1] + sg[2] * ga[2] * gb[2] +
                            sg[3] * (ga[0] * gb[1] + ga[1] * gb[0]) + sg[4] * (ga[0] * gb[2] + ga[2] * gb[0]) +
                            sg[5] * (ga[1] * gb[2] + ga[2] * gb[1]);
          val += sq[q] * se;
        }
      }
      const double bv[9] = {val, 0.0, 0.0, 0.0, val, 0.0, 0.0, 0.0, val};
      store_block<double>(out + p * blk_stride<double>(), bv);
    }
    __syncwarp();
  }
}

template <int ET, int KIND>
cudaError_t launch_scalar_t(const ElemArgs& a, const V2Args& v, const double* density, const double* gp_stress,
                            cudaStream_t s) {
  if (a.n_elems == 0) return cudaSuccess;
  auto kern = scalar_kernel<ET, KIND>;
  const size_t smem = sizeof(double) * kScalarWarps * scalar_warp_doubles<ET, KIND>();
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kScalarWarps * 32, smem);
  if (err != cudaSuccess) return err;
  const int64_t grid = persistent_grid((a.n_elems + kScalarWarps - 1) / kScalarWarps, per_sm, 0);
  kern<<<static_cast<unsigned>(grid), kScalarWarps * 32, smem, s>>>(a, v, density, gp_stress);
  return cudaGetLastError();
}

template <int ET>
cudaError_t launch_scalar_type(int kind, const ElemArgs& a, const V2Args& v, const double* density,
                               const double* gp_stress, cudaStream_t s) {
  switch (kind) {
    case 1: return launch_scalar_t<ET, 1>(a, v, density, gp_stress, s);
    case 2: return launch_scalar_t<ET, 2>(a, v, density, gp_stress, s);
    case 3: return launch_scalar_t<ET, 3>(a, v, density, gp_stress, s);
    case 4: return launch_scalar_t<ET, 4>(a, v, density, gp_stress, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

size_t v2_bytes_per_element(int t, int precision, bool tangent) {
  return v2_edata_bytes(t, 1, precision) + (tangent ? sizeof(double) * 3 * nodes_of(t) : 0);
}

size_t v2_edata_bytes(int t, int64_t n_elems, int precision) {
  const int n = nodes_of(t);
  return static_cast<size_t>(n_elems) * (n * (n + 1) / 2) *
         (precision ? blk_stride<float>() * sizeof(float) : blk_stride<double>() * sizeof(double));
}

cudaError_t launch_v2(int t, int mode, int precision, const ElemArgs& a, const V2Args& v, cudaStream_t s,
                      const LaunchCfg& c) {
  switch (t) {
    case C3D4: return launch_v2_type<C3D4>(mode, precision, a, v, c, s);
    case C3D10: return launch_v2_type<C3D10>(mode, precision, a, v, c, s);
    case C3D8: return launch_v2_type<C3D8>(mode, precision, a, v, c, s);
    case C3D8R: return launch_v2_type<C3D8R>(mode, precision, a, v, c, s);
    case C3D20: return launch_v2_type<C3D20>(mode, precision, a, v, c, s);
    case C3D20R: return launch_v2_type<C3D20R>(mode, precision, a, v, c, s);
    case C3D6: return launch_v2_type<C3D6>(mode, precision, a, v, c, s);
    case C3D15: return launch_v2_type<C3D15>(mode, precision, a, v, c, s);
    default: return cudaErrorInvalidValue;
  }
}

// ---- one launch per pass for a batch of element-type groups ---------------------------
// Slot k of a pass is one group (one element type, the concatenated models of that type)
// and owns blocks [blk0_k, blk0_{k+1}) of the grid. A block reads its slot's arguments
// in place from the kernel's parameter space (a copy in shared memory measured slower:
// the bodies' shared-memory stores made every argument a reload) and runs the group's
// element-pass or row-gather body with its index among the slot's blocks in place of
// blockIdx. The bodies are the ones the
// per-group kernels inline, so every value is the same bit for bit; the kernel holds
// the largest register count of its bodies, which is what a group pays for sharing
// the launch.
struct BatchSlot {
  ElemArgs a;
  V2Args v;
  int64_t blk0;
  int32_t type, tile;
};
struct BatchPass {
  BatchSlot s[kMaxBatchSlots];
  int32_t n;
};
static_assert(sizeof(BatchPass) <= 4096, "batch pass arguments exceed the kernel parameter space");

// Slot of this block (block-uniform).
__device__ __forceinline__ int slot_of(const BatchPass& P) {
  int k = 0;
  while (k + 1 < P.n && static_cast<int64_t>(blockIdx.x) >= P.s[k + 1].blk0) ++k;
  return k;
}

// This block's index among its slot's blocks, and their count.
__device__ __forceinline__ void slot_blocks(const BatchPass& P, int k, unsigned& bid, unsigned& nblk) {
  const int64_t end = k + 1 < P.n ? P.s[k + 1].blk0 : static_cast<int64_t>(gridDim.x);
  bid = blockIdx.x - static_cast<unsigned>(P.s[k].blk0);
  nblk = static_cast<unsigned>(end - P.s[k].blk0);
}

template <int ET, int MODE, typename R, int TILE, bool J2F32>
__device__ __forceinline__ void p1_slot(const ElemArgs& A, const V2Args& V, unsigned bid, unsigned nblk) {
  p1_body<ET, MODE, R, TILE, J2F32>(A, V, bid, nblk);
}

// The batch kernels carry the tiles whose accumulators fit 168 registers, so that 3
// blocks of 4 warps stay resident per SM whatever families share the launch: 2x2
// everywhere and 2x4 in the mixed-precision linear pass.
bool batch_tile_ok(int mode, int precision, int tile) {
  return tile == 1 || (tile == 0 && mode == MODE_LINEAR && precision);
}

template <int ET, int MODE, typename R, bool J2F32>
__device__ __forceinline__ void p1_slot_tile(int tile, const ElemArgs& A, const V2Args& V, unsigned bid, unsigned nblk) {
  if constexpr (MODE == MODE_LINEAR && sizeof(R) == 4) {
    if (tile == 0) {
      p1_slot<ET, MODE, R, 0, J2F32>(A, V, bid, nblk);
      return;
    }
  }
  p1_slot<ET, MODE, R, 1, J2F32>(A, V, bid, nblk);
}

template <int MODE, typename R, bool J2F32>
__global__ void __launch_bounds__(kT1, 3) p1_batch_kernel(const __grid_constant__ BatchPass P) {
  // the slot's arguments are read in place from the (read-only) parameter space
  const int k = slot_of(P);
  const BatchSlot& S = P.s[k];
  unsigned bid, nblk;
  slot_blocks(P, k, bid, nblk);
  switch (S.type) {
    case C3D4: p1_slot_tile<C3D4, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D10: p1_slot_tile<C3D10, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D8: p1_slot_tile<C3D8, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D8R: p1_slot_tile<C3D8R, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D20: p1_slot_tile<C3D20, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D20R: p1_slot_tile<C3D20R, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D6: p1_slot_tile<C3D6, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    case C3D15: p1_slot_tile<C3D15, MODE, R, J2F32>(S.tile, S.a, S.v, bid, nblk); break;
    default: break;
  }
}

template <int ET, bool TAN, typename R, bool DF>
__device__ __forceinline__ void p2_slot(const ElemArgs& A, const V2Args& V, unsigned bid, unsigned nblk) {
  p2_body<ET, TAN, R, DF, false>(A, V, bid, nblk);
}

template <bool TAN, typename R, bool DF>
__global__ void p2_batch_kernel(const __grid_constant__ BatchPass P) {
  const int k = slot_of(P);
  const BatchSlot& S = P.s[k];
  unsigned bid, nblk;
  slot_blocks(P, k, bid, nblk);
  switch (S.type) {
    case C3D4: p2_slot<C3D4, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D10: p2_slot<C3D10, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D8: p2_slot<C3D8, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D8R: p2_slot<C3D8R, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D20: p2_slot<C3D20, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D20R: p2_slot<C3D20R, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D6: p2_slot<C3D6, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    case C3D15: p2_slot<C3D15, TAN, R, DF>(S.a, S.v, bid, nblk); break;
    default: break;
  }
}

// Per-(family, tile) figures the launcher needs at run time.
struct P1Shape {
  size_t smem = 0;
  int epw = 1;
};
template <int ET, int MODE, typename R, int TILE>
P1Shape p1_shape_of() {
  return {p1_smem_bytes<ET, MODE, R, TILE>(), Geo<ET, TILE>::EPW};
}
template <int ET, int MODE, typename R>
P1Shape p1_shape_tile(int tile) {
  if constexpr (MODE == MODE_LINEAR && sizeof(R) == 4) {
    if (tile == 0) return p1_shape_of<ET, MODE, R, 0>();
  }
  return p1_shape_of<ET, MODE, R, 1>();
}
template <int MODE, typename R>
P1Shape p1_shape(int t, int tile) {
  switch (t) {
    case C3D4: return p1_shape_tile<C3D4, MODE, R>(tile);
    case C3D10: return p1_shape_tile<C3D10, MODE, R>(tile);
    case C3D8: return p1_shape_tile<C3D8, MODE, R>(tile);
    case C3D8R: return p1_shape_tile<C3D8R, MODE, R>(tile);
    case C3D20: return p1_shape_tile<C3D20, MODE, R>(tile);
    case C3D20R: return p1_shape_tile<C3D20R, MODE, R>(tile);
    case C3D6: return p1_shape_tile<C3D6, MODE, R>(tile);
    default: return p1_shape_tile<C3D15, MODE, R>(tile);
  }
}
// Row-buffer copies per warp of the row gather (P2Geo::EG): two 16-lane groups for the
// families of at most 16 nodes, one 32-lane group above.
int p2_groups_of(int t) { return nodes_of(t) <= 16 ? 2 : 1; }

// Blocks of a persistent grid of `total` blocks shared out in proportion to the
// slots' weights, at least one and at most `need` per slot.
void share_blocks(const double* weight, const int64_t* need, int n, int64_t total, int64_t* grid) {
  double sum = 0.0;
  for (int k = 0; k < n; ++k) sum += weight[k] > 0.0 ? weight[k] : 0.0;
  for (int k = 0; k < n; ++k) {
    const double f = sum > 0.0 ? std::max(weight[k], 0.0) / sum : 1.0 / n;
    const int64_t g = static_cast<int64_t>(std::llround(f * static_cast<double>(total)));
    grid[k] = std::max<int64_t>(1, std::min<int64_t>(need[k], g));
  }
}

template <int MODE, typename R, bool J2F32>
cudaError_t launch_p1_batch(const BatchSlotIn* in, int n, cudaStream_t s) {
  auto kern = p1_batch_kernel<MODE, R, J2F32>;
  BatchPass P{};
  size_t smem = 0;
  int64_t need[kMaxBatchSlots], grid[kMaxBatchSlots];
  double w[kMaxBatchSlots];
  for (int k = 0; k < n; ++k) {
    const P1Shape sh = p1_shape<MODE, R>(in[k].type, in[k].cfg.tile);
    smem = std::max(smem, sh.smem);
    const int64_t count = in[k].v.e_end - in[k].v.e_begin;
    need[k] = std::max<int64_t>(1, (count + kW1 * sh.epw - 1) / (kW1 * sh.epw));
    w[k] = in[k].p1_weight;
  }
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kT1, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  share_blocks(w, need, n, static_cast<int64_t>(per_sm) * sm_count(), grid);
  int64_t blk = 0;
  for (int k = 0; k < n; ++k) {
    P.s[k].a = in[k].a;
    P.s[k].v = in[k].v;
    P.s[k].blk0 = blk;
    P.s[k].type = in[k].type;
    P.s[k].tile = in[k].cfg.tile;
    blk += grid[k];
  }
  P.n = n;
  kern<<<static_cast<unsigned>(blk), kT1, smem, s>>>(P);
  return cudaGetLastError();
}

template <bool TAN, typename R, bool DF>
cudaError_t launch_p2_batch(const BatchSlotIn* in, int n, cudaStream_t s) {
  auto kern = p2_batch_kernel<TAN, R, DF>;
  BatchPass P{};
  // one block shape for every slot: the most warps every slot's row buffers allow in
  // ~160 KB, at most 8 (or the smallest configured count)
  int warps = 8;
  int64_t wbytes_max = 0;
  for (int k = 0; k < n; ++k) {
    const int64_t stride = std::max<int64_t>(2, (9 * in[k].v.max_adj + 1) / 2 * 2);
    const int64_t wbytes = p2_groups_of(in[k].type) * stride * 8;
    wbytes_max = std::max(wbytes_max, wbytes);
    if (in[k].cfg.p2_warps > 0) warps = std::min(warps, in[k].cfg.p2_warps);
  }
  while (warps > 1 && warps * wbytes_max > 160 * 1024) warps /= 2;
  const size_t smem = static_cast<size_t>(warps) * wbytes_max;
  if (smem > 220 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int64_t need[kMaxBatchSlots], grid[kMaxBatchSlots];
  double w[kMaxBatchSlots];
  for (int k = 0; k < n; ++k) {
    const int64_t count = in[k].v.n_end - in[k].v.n_begin;
    need[k] = std::max<int64_t>(1, (count + warps - 1) / warps);
    w[k] = in[k].p2_weight;
  }
  share_blocks(w, need, n, static_cast<int64_t>(per_sm) * sm_count(), grid);
  int64_t blk = 0;
  for (int k = 0; k < n; ++k) {
    P.s[k].a = in[k].a;
    P.s[k].v = in[k].v;
    P.s[k].v.row_stride = std::max<int64_t>(2, (9 * in[k].v.max_adj + 1) / 2 * 2);
    P.s[k].blk0 = blk;
    P.s[k].type = in[k].type;
    P.s[k].tile = in[k].cfg.tile;
    blk += grid[k];
  }
  P.n = n;
  kern<<<static_cast<unsigned>(blk), warps * 32, smem, s>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_v2_batch(int mode, int precision, const BatchSlotIn* in, int n, int passes, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (n > kMaxBatchSlots) return cudaErrorInvalidValue;
  const bool j2f32 = mode == MODE_TANGENT && precision && in[0].cfg.j2_fp32;
  for (int k = 0; k < n; ++k) {
    if (in[k].type < kFirstType || in[k].type > kLastType || in[k].v.n_win > 1 || in[k].v.node_order)
      return cudaErrorInvalidValue;
    if ((mode == MODE_TANGENT && precision && (in[k].cfg.j2_fp32 != 0) != j2f32) ||
        !batch_tile_ok(mode, precision, in[k].cfg.tile))
      return cudaErrorInvalidValue;
  }
  cudaError_t err = cudaSuccess;
  if (passes & 1) {
    if (mode == MODE_LINEAR)
      err = precision ? launch_p1_batch<MODE_LINEAR, float, false>(in, n, s)
                      : launch_p1_batch<MODE_LINEAR, double, false>(in, n, s);
    else if (precision)
      err = j2f32 ? launch_p1_batch<MODE_TANGENT, float, true>(in, n, s)
                  : launch_p1_batch<MODE_TANGENT, float, false>(in, n, s);
    else
      err = launch_p1_batch<MODE_TANGENT, double, false>(in, n, s);
    if (err != cudaSuccess) return err;
  }
  if (passes & 2) {
    if (mode == MODE_LINEAR)
      err = precision ? launch_p2_batch<false, float, true>(in, n, s) : launch_p2_batch<false, double, false>(in, n, s);
    else
      err = precision ? launch_p2_batch<true, float, true>(in, n, s) : launch_p2_batch<true, double, false>(in, n, s);
  }
  return err;
}

cudaError_t launch_scalar_pass(int t, int kind, const ElemArgs& a, const V2Args& v, const double* density,
                               const double* gp_stress, cudaStream_t s) {
  switch (t) {
    case C3D4: return launch_scalar_type<C3D4>(kind, a, v, density, gp_stress, s);
    case C3D10: return launch_scalar_type<C3D10>(kind, a, v, density, gp_stress, s);
    case C3D8: return launch_scalar_type<C3D8>(kind, a, v, density, gp_stress, s);
    case C3D8R: return launch_scalar_type<C3D8R>(kind, a, v, density, gp_stress, s);
    case C3D20: return launch_scalar_type<C3D20>(kind, a, v, density, gp_stress, s);
    case C3D20R: return launch_scalar_type<C3D20R>(kind, a, v, density, gp_stress, s);
    case C3D6: return launch_scalar_type<C3D6>(kind, a, v, density, gp_stress, s);
    case C3D15: return launch_scalar_type<C3D15>(kind, a, v, density, gp_stress, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace cxg
