/* cxo — CPU restatement of CalculiX++'s element-integration / J2 / assembly path.
 * TEST INFRASTRUCTURE ONLY (see cxo.h). Every function names the reference file:line
 * it restates. Operation order follows the reference so that, compiled with
 * -ffp-contract=off, results are bit-identical to the reference's own code. */
#include "cxo.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static _Thread_local char g_err[256];

static int fail(const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return -1;
}

const char* cxo_last_error(void) { return g_err; }

enum { T_C3D4 = 0, T_C3D10 = 1, T_C3D8 = 2, T_C3D8R = 3, T_C3D20 = 4, T_C3D20R = 5, T_C3D6 = 6, T_C3D15 = 7 };
#define MAXN 20

/* include/calculixpp/core/element.hpp:24-44 */
int cxo_nodes_per_element(int type) {
  switch (type) {
    case T_C3D8: case T_C3D8R: return 8;
    case T_C3D20: case T_C3D20R: return 20;
    case T_C3D6: return 6;
    case T_C3D15: return 15;
    case T_C3D4: return 4;
    case T_C3D10: return 10;
    default: return 0;
  }
}

/* ---- Gauss rules: src/fem/element.cpp:22-126 ------------------------------------ */
static const double kG2 = 0.577350269189625764;
static const double kG3 = 0.774596669241483377;

int cxo_gauss_rule(int type, double* out) {
  int n = 0;
#define GP(a, b, c, w) do { out[4*n] = (a); out[4*n+1] = (b); out[4*n+2] = (c); out[4*n+3] = (w); ++n; } while (0)
  switch (type) {
    case T_C3D8:
    case T_C3D20R:
      /* 2x2x2, xi fastest (element.cpp:32-37) */
      for (int c = 0; c < 2; ++c)
        for (int b = 0; b < 2; ++b)
          for (int a = 0; a < 2; ++a)
            GP(a ? kG2 : -kG2, b ? kG2 : -kG2, c ? kG2 : -kG2, 1.0);
      break;
    case T_C3D8R:
      GP(0.0, 0.0, 0.0, 8.0); /* element.cpp:40 */
      break;
    case T_C3D20: {
      /* 3x3x3 Gauss-Legendre (element.cpp:43-62) */
      const double nodes[3] = {-kG3, 0.0, kG3};
      const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
      for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
          for (int a = 0; a < 3; ++a) GP(nodes[a], nodes[b], nodes[c], wts[a] * wts[b] * wts[c]);
      break;
    }
    case T_C3D6:
      GP(1.0 / 3.0, 1.0 / 3.0, -kG2, 0.5); /* element.cpp:68-71 */
      GP(1.0 / 3.0, 1.0 / 3.0, kG2, 0.5);
      break;
    case T_C3D15: {
      const double kT = 1.0 / 6.0, kU = 2.0 / 3.0; /* element.cpp:72-77 */
      GP(kT, kT, -kG2, kT); GP(kU, kT, -kG2, kT); GP(kT, kU, -kG2, kT);
      GP(kT, kT, kG2, kT); GP(kU, kT, kG2, kT); GP(kT, kU, kG2, kT);
      break;
    }
    case T_C3D4:
      GP(0.25, 0.25, 0.25, 1.0 / 6.0); /* element.cpp:14 */
      break;
    case T_C3D10: {
      const double kA = 0.138196601125010515, kB = 0.585410196624968454; /* element.cpp:10-20 */
      GP(kA, kA, kA, 1.0 / 24.0); GP(kB, kA, kA, 1.0 / 24.0);
      GP(kA, kB, kA, 1.0 / 24.0); GP(kA, kA, kB, 1.0 / 24.0);
      break;
    }
    default:
      return 0;
  }
#undef GP
  return n;
}

/* ---- shape functions: src/fem/element.cpp:160-359 ------------------------------- */
static const int kHexSign[8][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1},
};
static const int kMidHex[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                   {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
static const int kEdgeAxis[12] = {0, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2};

static void shape_c3d8(double xi, double et, double ze, double* N, double* dN) {
  for (int k = 0; k < 8; ++k) {
    const double sg = kHexSign[k][0], sh = kHexSign[k][1], sr = kHexSign[k][2];
    const double g = 1.0 + sg * xi, h = 1.0 + sh * et, r = 1.0 + sr * ze;
    N[k] = g * h * r / 8.0;
    dN[3 * k + 0] = sg * h * r / 8.0;
    dN[3 * k + 1] = sh * g * r / 8.0;
    dN[3 * k + 2] = sr * g * h / 8.0;
  }
}

static void shape_c3d20(double xi, double et, double ze, double* N, double* dN) {
  const double p[3] = {xi, et, ze};
  for (int k = 0; k < 8; ++k) {
    const double sgn[3] = {kHexSign[k][0], kHexSign[k][1], kHexSign[k][2]};
    const double g = 1.0 + sgn[0] * xi, h = 1.0 + sgn[1] * et, r = 1.0 + sgn[2] * ze;
    const double q = sgn[0] * xi + sgn[1] * et + sgn[2] * ze - 2.0;
    N[k] = g * h * r * q / 8.0;
    const double fac[3] = {g, h, r};
    for (int d = 0; d < 3; ++d) {
      double others = 1.0;
      for (int m = 0; m < 3; ++m)
        if (m != d) others *= fac[m];
      dN[3 * k + d] = (sgn[d] * others * q + g * h * r * sgn[d]) / 8.0;
    }
  }
  for (int j = 0; j < 12; ++j) {
    const int node = 8 + j;
    const int a = kEdgeAxis[j];
    const int c0 = kMidHex[j][0];
    const double sgn[3] = {kHexSign[c0][0], kHexSign[c0][1], kHexSign[c0][2]};
    const double pa = p[a];
    double plane = 1.0;
    for (int m = 0; m < 3; ++m)
      if (m != a) plane *= 1.0 + sgn[m] * p[m];
    N[node] = (1.0 - pa * pa) * plane / 4.0;
    for (int d = 0; d < 3; ++d) {
      if (d == a) {
        dN[3 * node + d] = (-2.0 * pa) * plane / 4.0;
      } else {
        double other = 1.0;
        for (int m = 0; m < 3; ++m)
          if (m != a && m != d) other *= 1.0 + sgn[m] * p[m];
        dN[3 * node + d] = (1.0 - pa * pa) * sgn[d] * other / 4.0;
      }
    }
  }
}

static void shape_c3d6(double xi, double et, double ze, double* N, double* dN) {
  const double a = 1.0 - xi - et;
  const double m = 0.5 * (1.0 - ze), p = 0.5 * (1.0 + ze);
  const double n6[6] = {a * m, xi * m, et * m, a * p, xi * p, et * p};
  const double d6[18] = {-m, -m, -0.5 * a, m, 0.0, -0.5 * xi, 0.0, m, -0.5 * et,
                         -p, -p, 0.5 * a,  p, 0.0, 0.5 * xi,  0.0, p, 0.5 * et};
  memcpy(N, n6, sizeof n6);
  memcpy(dN, d6, sizeof d6);
}

static void shape_c3d15(double xi, double et, double ze, double* N, double* dN) {
  const double a = 1.0 - xi - et;
  const double omz = 1.0 - ze, opz = 1.0 + ze, omz2 = 1.0 - ze * ze;
  N[0] = -0.5 * a * omz * (2 * xi + 2 * et + ze);
  N[1] = 0.5 * xi * omz * (2 * xi - 2 - ze);
  N[2] = 0.5 * et * omz * (2 * et - 2 - ze);
  N[3] = -0.5 * a * opz * (2 * xi + 2 * et - ze);
  N[4] = 0.5 * xi * opz * (2 * xi - 2 + ze);
  N[5] = 0.5 * et * opz * (2 * et - 2 + ze);
  N[6] = 2 * xi * a * omz;
  N[7] = 2 * xi * et * omz;
  N[8] = 2 * et * a * omz;
  N[9] = 2 * xi * a * opz;
  N[10] = 2 * xi * et * opz;
  N[11] = 2 * et * a * opz;
  N[12] = a * omz2;
  N[13] = xi * omz2;
  N[14] = et * omz2;
  const double dxi[15] = {0.5 * omz * (4 * xi + 4 * et + ze - 2),
                          0.5 * omz * (4 * xi - ze - 2),
                          0.0,
                          0.5 * opz * (4 * xi + 4 * et - ze - 2),
                          0.5 * opz * (4 * xi + ze - 2),
                          0.0,
                          2 * omz * (1 - 2 * xi - et),
                          2 * et * omz,
                          -2 * et * omz,
                          2 * opz * (1 - 2 * xi - et),
                          2 * et * opz,
                          -2 * et * opz,
                          -omz2,
                          omz2,
                          0.0};
  const double det[15] = {0.5 * omz * (4 * xi + 4 * et + ze - 2),
                          0.0,
                          0.5 * omz * (4 * et - ze - 2),
                          0.5 * opz * (4 * xi + 4 * et - ze - 2),
                          0.0,
                          0.5 * opz * (4 * et + ze - 2),
                          -2 * xi * omz,
                          2 * xi * omz,
                          2 * omz * (1 - xi - 2 * et),
                          -2 * xi * opz,
                          2 * xi * opz,
                          2 * opz * (1 - xi - 2 * et),
                          -omz2,
                          0.0,
                          omz2};
  double dz[15];
  dz[0] = -0.5 * a * (-1.0 * (2 * xi + 2 * et + ze) + omz * 1.0);
  dz[1] = 0.5 * xi * (-1.0 * (2 * xi - 2 - ze) + omz * (-1.0));
  dz[2] = 0.5 * et * (-1.0 * (2 * et - 2 - ze) + omz * (-1.0));
  dz[3] = -0.5 * a * (1.0 * (2 * xi + 2 * et - ze) + opz * (-1.0));
  dz[4] = 0.5 * xi * (1.0 * (2 * xi - 2 + ze) + opz * (1.0));
  dz[5] = 0.5 * et * (1.0 * (2 * et - 2 + ze) + opz * (1.0));
  dz[6] = -2 * xi * a;
  dz[7] = -2 * xi * et;
  dz[8] = -2 * et * a;
  dz[9] = 2 * xi * a;
  dz[10] = 2 * xi * et;
  dz[11] = 2 * et * a;
  dz[12] = a * (-2 * ze);
  dz[13] = xi * (-2 * ze);
  dz[14] = et * (-2 * ze);
  for (int k = 0; k < 15; ++k) {
    dN[3 * k] = dxi[k];
    dN[3 * k + 1] = det[k];
    dN[3 * k + 2] = dz[k];
  }
}

/* shape_c3d4 / shape_c3d10, element.cpp:130-158: volume coordinates, a = 1-xi-et-ze. */
static void shape_c3d4(double xi, double et, double ze, double* N, double* dN) {
  N[0] = 1.0 - xi - et - ze; N[1] = xi; N[2] = et; N[3] = ze;
  const double d[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 3; ++j) dN[3 * k + j] = d[k][j];
}

static void shape_c3d10(double xi, double et, double ze, double* N, double* dN) {
  const double a = 1.0 - xi - et - ze;
  N[0] = (2 * a - 1) * a;  N[1] = xi * (2 * xi - 1); N[2] = et * (2 * et - 1); N[3] = ze * (2 * ze - 1);
  N[4] = 4 * xi * a;       N[5] = 4 * xi * et;       N[6] = 4 * et * a;        N[7] = 4 * ze * a;
  N[8] = 4 * xi * ze;      N[9] = 4 * et * ze;
  const double d[10][3] = {{1 - 4 * a, 1 - 4 * a, 1 - 4 * a}, {4 * xi - 1, 0, 0}, {0, 4 * et - 1, 0},
                           {0, 0, 4 * ze - 1}, {4 * (a - xi), -4 * xi, -4 * xi}, {4 * et, 4 * xi, 0},
                           {-4 * et, 4 * (a - et), -4 * et}, {-4 * ze, -4 * ze, 4 * (a - ze)},
                           {4 * ze, 0, 4 * xi}, {0, 4 * ze, 4 * et}};
  for (int k = 0; k < 10; ++k)
    for (int j = 0; j < 3; ++j) dN[3 * k + j] = d[k][j];
}

int cxo_shape(int type, double xi, double et, double ze, double* N, double* dN) {
  switch (type) {
    case T_C3D8: case T_C3D8R: shape_c3d8(xi, et, ze, N, dN); return 8;
    case T_C3D20: case T_C3D20R: shape_c3d20(xi, et, ze, N, dN); return 20;
    case T_C3D6: shape_c3d6(xi, et, ze, N, dN); return 6;
    case T_C3D15: shape_c3d15(xi, et, ze, N, dN); return 15;
    case T_C3D4: shape_c3d4(xi, et, ze, N, dN); return 4;
    case T_C3D10: shape_c3d10(xi, et, ze, N, dN); return 10;
    default: return 0;
  }
}

/* ---- physical gradients: src/fem/element.cpp:80-102, 361-380 ------------------- */
static int gradients_from_shape(int n, const double* dN, const double* x, double* g,
                                double* det_out) {
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
  if (det <= 0.0) return fail("non-positive element Jacobian (bad connectivity?)");
  const double inv = 1.0 / det;
  const double Jinv[3][3] = {
      {c00 * inv, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * inv,
       (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * inv},
      {c01 * inv, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * inv,
       (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * inv},
      {c02 * inv, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * inv,
       (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * inv},
  };
  double invT[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) invT[i][j] = Jinv[j][i];
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < 3; ++i) {
      double v = 0.0;
      for (int j = 0; j < 3; ++j) v += invT[i][j] * dN[3 * k + j];
      g[3 * k + i] = v;
    }
  *det_out = det;
  return 0;
}

int cxo_physical_gradients(int type, double xi, double et, double ze,
                           const double* coords, double* grad, double* det) {
  double N[MAXN], dN[3 * MAXN];
  const int n = cxo_shape(type, xi, et, ze, N, dN);
  if (n == 0) return fail("unsupported element type");
  return gradients_from_shape(n, dN, coords, grad, det);
}

/* element.cpp:424-433 */
int cxo_element_volume(int type, const double* coords, double* vol) {
  double gp[4 * 27], g[3 * MAXN], det;
  const int ng = cxo_gauss_rule(type, gp);
  double v = 0.0;
  for (int q = 0; q < ng; ++q) {
    if (cxo_physical_gradients(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], coords, g, &det))
      return -1;
    v += det * gp[4 * q + 3];
  }
  *vol = v;
  return 0;
}

/* ---- constitutive pieces --------------------------------------------------------- */
/* element.cpp:382-392 */
static double b_entry(int row, const double* gk, int dir) {
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

/* element.cpp:410-422 */
static void elastic_D(double E, double nu, double* D) {
  const double um2 = E / (1.0 + nu);
  const double lam = nu * um2 / (1.0 - 2.0 * nu);
  const double mu = um2 / 2.0;
  const double lam2mu = lam + um2;
  memset(D, 0, 36 * sizeof(double));
  D[0] = D[7] = D[14] = lam2mu;
  D[1] = D[2] = D[6] = D[8] = D[12] = D[13] = lam;
  D[21] = D[28] = D[35] = mu;
}

/* element.cpp:440-462 */
static void accumulate_ktangent(const double* g, int ndof, const double* D, double scale,
                                double* Ke) {
  for (int a = 0; a < ndof; ++a) {
    const int ka = a / 3, da = a % 3;
    double DBa[6];
    for (int row = 0; row < 6; ++row) {
      double v = 0.0;
      for (int r = 0; r < 6; ++r) v += D[6 * row + r] * b_entry(r, g + 3 * ka, da);
      DBa[row] = v;
    }
    for (int b = a; b < ndof; ++b) {
      const int kb = b / 3, db = b % 3;
      double v = 0.0;
      for (int row = 0; row < 6; ++row) v += b_entry(row, g + 3 * kb, db) * DBa[row];
      Ke[a * ndof + b] += scale * v;
    }
  }
}

/* element.cpp:465-475 */
static void accumulate_fint(const double* g, int ndof, const double* sigma, double scale,
                            double* fe) {
  for (int a = 0; a < ndof; ++a) {
    const int ka = a / 3, da = a % 3;
    double v = 0.0;
    for (int row = 0; row < 6; ++row) v += b_entry(row, g + 3 * ka, da) * sigma[row];
    fe[a] += scale * v;
  }
}

/* element.cpp:511-518 */
static void mirror_upper(int ndof, double* Ke) {
  for (int a = 0; a < ndof; ++a)
    for (int b = a + 1; b < ndof; ++b) Ke[b * ndof + a] = Ke[a * ndof + b];
}

/* element.cpp:394-408 */
static void strain_from_gradients(const double* g, int n, const double* ue, double* eps) {
  double du[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < n; ++k) v += g[3 * k + j] * ue[3 * k + i];
      du[i][j] = v;
    }
  eps[0] = du[0][0];
  eps[1] = du[1][1];
  eps[2] = du[2][2];
  eps[3] = du[0][1] + du[1][0];
  eps[4] = du[0][2] + du[2][0];
  eps[5] = du[1][2] + du[2][1];
}

/* ---- C3D8R hourglass control: element.cpp:529-610 ------------------------------- */
static const double kHgGamma[4][8] = {
    {1, 1, -1, -1, -1, -1, 1, 1},
    {1, -1, -1, 1, -1, 1, 1, -1},
    {1, -1, 1, -1, 1, -1, 1, -1},
    {-1, 1, -1, 1, 1, -1, 1, -1},
};

typedef struct {
  double gamma[4][8];
  double kappa;
} hourglass_t;

static int build_hourglass(const double* x, double mu, hourglass_t* hg) {
  double N[8], dN[24], b[24], det;
  shape_c3d8(0.0, 0.0, 0.0, N, dN);
  if (gradients_from_shape(8, dN, x, b, &det)) return -1;
  const double vol = 8.0 * det;
  for (int al = 0; al < 4; ++al) {
    double gx[3] = {0, 0, 0};
    for (int j = 0; j < 8; ++j)
      for (int d = 0; d < 3; ++d) gx[d] += kHgGamma[al][j] * x[3 * j + d];
    for (int j = 0; j < 8; ++j) {
      double corr = 0.0;
      for (int d = 0; d < 3; ++d) corr += gx[d] * b[3 * j + d];
      hg->gamma[al][j] = kHgGamma[al][j] - corr;
    }
  }
  double b2 = 0.0;
  for (int j = 0; j < 8; ++j)
    for (int d = 0; d < 3; ++d) b2 += b[3 * j + d] * b[3 * j + d];
  const double c_hg = 0.05;
  hg->kappa = c_hg * mu * vol * b2;
  return 0;
}

static void accumulate_hourglass(const hourglass_t* hg, double* Ke) {
  for (int al = 0; al < 4; ++al)
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) {
        const double kij = hg->kappa * hg->gamma[al][i] * hg->gamma[al][j];
        for (int d = 0; d < 3; ++d) {
          const int a = i * 3 + d, bc = j * 3 + d;
          if (bc >= a) Ke[a * 24 + bc] += kij;
        }
      }
}

static void accumulate_hourglass_force(const hourglass_t* hg, const double* ue, double* fe) {
  for (int al = 0; al < 4; ++al) {
    double gu[3] = {0, 0, 0};
    for (int j = 0; j < 8; ++j)
      for (int d = 0; d < 3; ++d) gu[d] += hg->gamma[al][j] * ue[3 * j + d];
    for (int i = 0; i < 8; ++i)
      for (int d = 0; d < 3; ++d) fe[i * 3 + d] += hg->kappa * hg->gamma[al][i] * gu[d];
  }
}

/* ---- element_stiffness: element.cpp:614-634 ------------------------------------- */
int cxo_element_stiffness(int type, const double* x, double E, double nu, double* Ke) {
  const int n = cxo_nodes_per_element(type);
  if (n == 0) return fail("unsupported element type");
  const int ndof = 3 * n;
  double D[36], gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det;
  elastic_D(E, nu, D);
  memset(Ke, 0, (size_t)ndof * ndof * sizeof(double));
  const int ng = cxo_gauss_rule(type, gp);
  for (int q = 0; q < ng; ++q) {
    cxo_shape(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
    if (gradients_from_shape(n, dN, x, g, &det)) return -1;
    accumulate_ktangent(g, ndof, D, det * gp[4 * q + 3], Ke);
  }
  if (type == T_C3D8R) {
    const double mu = E / (2.0 * (1.0 + nu));
    hourglass_t hg;
    if (build_hourglass(x, mu, &hg)) return -1;
    accumulate_hourglass(&hg, Ke);
  }
  mirror_upper(ndof, Ke);
  return 0;
}

/* ---- J2 plasticity: src/fem/plasticity.cpp:20-236 ------------------------------- */
static const double kSqrt3_2 = 1.224744871391589;

typedef struct {
  double E, nu, mu, h_kin;
  int n;
  const double* ep;
  double sy[64];
  double De[36];
} j2_t;

/* plasticity.cpp:42-65 */
static int j2_init(const cxo_material* m, j2_t* j) {
  if (m->n_plastic <= 0) return fail("J2PlasticMaterial needs a non-empty *PLASTIC table");
  if (m->n_plastic > 64) return fail("*PLASTIC table longer than 64 points");
  j->E = m->E;
  j->nu = m->nu;
  j->mu = m->E / (2.0 * (1.0 + m->nu));
  j->h_kin = m->h_kin;
  j->n = m->n_plastic;
  j->ep = m->eqplastic;
  for (int i = 0; i < j->n; ++i) j->sy[i] = m->yield[i];
  if (m->hardening == 1 || m->hardening == 2) {
    if (j->h_kin == 0.0 && j->n >= 2 && j->ep[1] > j->ep[0])
      j->h_kin = (j->sy[1] - j->sy[0]) / (j->ep[1] - j->ep[0]);
    if (m->hardening == 1)
      for (int i = 0; i < j->n; ++i) j->sy[i] = j->sy[0];
  }
  elastic_D(m->E, m->nu, j->De);
  return 0;
}

/* plasticity.cpp:67-88 */
static void j2_hardening(const j2_t* j, double ep, double* sigma_y, double* h_iso) {
  const int n = j->n;
  if (n == 1 || ep <= j->ep[0]) {
    *sigma_y = j->sy[0];
    *h_iso = 0.0;
    return;
  }
  if (ep >= j->ep[n - 1]) {
    *sigma_y = j->sy[n - 1];
    *h_iso = 0.0;
    return;
  }
  for (int i = 0; i + 1 < n; ++i) {
    if (ep >= j->ep[i] && ep <= j->ep[i + 1]) {
      *h_iso = (j->sy[i + 1] - j->sy[i]) / (j->ep[i + 1] - j->ep[i]);
      *sigma_y = j->sy[i] + *h_iso * (ep - j->ep[i]);
      return;
    }
  }
  *sigma_y = j->sy[n - 1];
  *h_iso = 0.0;
}

static double contract6(const double* s) {
  return s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
}

/* plasticity.cpp:90-236. committed/trial: eps_p[6], ep, alpha[6]. */
static void j2_evaluate(const j2_t* j, const double* strain, const double* cs, double* ts,
                        double* stress, double* tangent) {
  double el[6], sig_tr[6], s_tr[6], xi[6];
  for (int i = 0; i < 6; ++i) el[i] = strain[i] - cs[i];
  for (int i = 0; i < 6; ++i) {
    double v = 0.0;
    for (int k = 0; k < 6; ++k) v += j->De[6 * i + k] * el[k];
    sig_tr[i] = v;
  }
  {
    const double p = (sig_tr[0] + sig_tr[1] + sig_tr[2]) / 3.0;
    s_tr[0] = sig_tr[0] - p;
    s_tr[1] = sig_tr[1] - p;
    s_tr[2] = sig_tr[2] - p;
    s_tr[3] = sig_tr[3];
    s_tr[4] = sig_tr[4];
    s_tr[5] = sig_tr[5];
  }
  for (int i = 0; i < 6; ++i) xi[i] = s_tr[i] - cs[7 + i];
  const double xi_norm = sqrt(contract6(xi));
  const double q_tr = kSqrt3_2 * xi_norm;
  double sy0, h0;
  j2_hardening(j, cs[6], &sy0, &h0);
  const double f_tr = q_tr - sy0;
  if (f_tr <= 0.0 || xi_norm == 0.0) {
    memcpy(stress, sig_tr, sizeof sig_tr);
    memcpy(tangent, j->De, 36 * sizeof(double));
    memcpy(ts, cs, 13 * sizeof(double));
    return;
  }
  const double ep0 = cs[6];
  double dgamma = 0.0;
  for (int it = 0; it < 50; ++it) {
    double sy, h_iso;
    j2_hardening(j, ep0 + dgamma, &sy, &h_iso);
    const double g = q_tr - 3.0 * j->mu * dgamma - j->h_kin * dgamma - sy;
    const double dg = -(3.0 * j->mu + j->h_kin + h_iso);
    const double step = -g / dg;
    dgamma += step;
    if (dgamma < 0.0) dgamma = 0.0;
    if (fabs(step) <= 1e-14 * (1.0 + fabs(dgamma))) break;
  }
  double n[6];
  for (int i = 0; i < 6; ++i) n[i] = xi[i] / xi_norm;
  const double dev_scale = 2.0 * j->mu * dgamma * kSqrt3_2;
  const double alpha_scale = (2.0 / 3.0) * j->h_kin * dgamma * kSqrt3_2;
  const double mean = (sig_tr[0] + sig_tr[1] + sig_tr[2]) / 3.0;
  for (int i = 0; i < 6; ++i) {
    const double dev = s_tr[i] - dev_scale * n[i];
    stress[i] = dev + (i < 3 ? mean : 0.0);
  }
  const double dep_scale = dgamma * kSqrt3_2;
  for (int i = 0; i < 6; ++i) {
    const double dep_i = dep_scale * n[i] * (i < 3 ? 1.0 : 2.0);
    ts[i] = cs[i] + dep_i;
    ts[7 + i] = cs[7 + i] + alpha_scale * n[i];
  }
  ts[6] = ep0 + dgamma;
  double sy, h_iso;
  j2_hardening(j, ep0 + dgamma, &sy, &h_iso);
  const double theta = 1.0 - (2.0 * j->mu * dgamma * kSqrt3_2) / xi_norm;
  const double denom = 1.0 + (h_iso + j->h_kin) / (3.0 * j->mu);
  const double theta_bar = 1.0 / denom - (1.0 - theta);
  double Idev[36];
  memset(Idev, 0, sizeof Idev);
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) Idev[6 * i + k] = 2.0 * j->mu * ((i == k ? 1.0 : 0.0) - 1.0 / 3.0);
  for (int i = 3; i < 6; ++i) Idev[6 * i + i] = j->mu;
  for (int i = 0; i < 6; ++i)
    for (int k = 0; k < 6; ++k)
      tangent[6 * i + k] = j->De[6 * i + k] - (1.0 - theta) * Idev[6 * i + k] -
                           2.0 * j->mu * theta_bar * n[i] * n[k];
}

/* Linear elasticity (element.cpp:859-871) or J2 (plasticity.cpp:90). */
int cxo_material_evaluate(const cxo_material* m, const double* strain, const double* cs,
                          double* ts, double* stress, double* tangent) {
  if (m->n_plastic > 0) {
    j2_t j;
    if (j2_init(m, &j)) return -1;
    j2_evaluate(&j, strain, cs, ts, stress, tangent);
    return 0;
  }
  elastic_D(m->E, m->nu, tangent);
  for (int i = 0; i < 6; ++i) {
    double v = 0.0;
    for (int k = 0; k < 6; ++k) v += tangent[6 * i + k] * strain[k];
    stress[i] = v;
  }
  memcpy(ts, cs, 13 * sizeof(double));
  return 0;
}

/* ---- element_tangent_force: element.cpp:708-743 --------------------------------- */
static int tangent_force(int type, const double* x, const double* ue, const cxo_material* m,
                         const j2_t* j, const double* sc, double* st, double* Ke, double* fe) {
  const int n = cxo_nodes_per_element(type);
  const int ndof = 3 * n;
  double gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det, eps[6], sig[6], D[36];
  memset(Ke, 0, (size_t)ndof * ndof * sizeof(double));
  memset(fe, 0, (size_t)ndof * sizeof(double));
  double De[36];
  if (!j) elastic_D(m->E, m->nu, De);
  const int ng = cxo_gauss_rule(type, gp);
  double mu_hg = 0.0;
  for (int q = 0; q < ng; ++q) {
    cxo_shape(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
    if (gradients_from_shape(n, dN, x, g, &det)) return -1;
    const double scale = det * gp[4 * q + 3];
    strain_from_gradients(g, n, ue, eps);
    if (j) {
      j2_evaluate(j, eps, sc + 13 * q, st + 13 * q, sig, D);
    } else {
      memcpy(D, De, sizeof D);
      for (int i = 0; i < 6; ++i) {
        double v = 0.0;
        for (int k = 0; k < 6; ++k) v += D[6 * i + k] * eps[k];
        sig[i] = v;
      }
      memcpy(st + 13 * q, sc + 13 * q, 13 * sizeof(double));
    }
    accumulate_ktangent(g, ndof, D, scale, Ke);
    accumulate_fint(g, ndof, sig, scale, fe);
    mu_hg = D[21];
  }
  if (type == T_C3D8R) {
    hourglass_t hg;
    if (build_hourglass(x, mu_hg, &hg)) return -1;
    accumulate_hourglass(&hg, Ke);
    accumulate_hourglass_force(&hg, ue, fe);
  }
  mirror_upper(ndof, Ke);
  return 0;
}

int cxo_element_tangent_force(int type, const double* x, const double* ue,
                              const cxo_material* m, const double* sc, double* st,
                              double* Ke, double* fe) {
  if (cxo_nodes_per_element(type) == 0) return fail("unsupported element type");
  j2_t j;
  if (m->n_plastic > 0 && j2_init(m, &j)) return -1;
  return tangent_force(type, x, ue, m, m->n_plastic > 0 ? &j : NULL, sc, st, Ke, fe);
}

/* ---- assembly: src/fem/assembly.cpp:19-257, 385-423 ----------------------------- */
struct cxo_system {
  int32_t n_free;
  int64_t nnz;
  int64_t* row_ptr;
  int32_t* col_idx;
  double* vals;
  double* rhs;
};

/* constraint_transform.cpp:78-82 (SPC-only: free DOFs numbered in global order) */
int32_t cxo_dof_map(int64_t n_nodes, int64_t n_spc, const int32_t* spc_node,
                    const int32_t* spc_comp, const double* spc_val, int32_t* dof_eq,
                    double* prescribed) {
  const int64_t ndof = 3 * n_nodes;
  for (int64_t g = 0; g < ndof; ++g) {
    dof_eq[g] = 0;
    prescribed[g] = 0.0;
  }
  for (int64_t i = 0; i < n_spc; ++i) {
    const int64_t g = 3 * (int64_t)spc_node[i] + spc_comp[i];
    dof_eq[g] = -1;
    prescribed[g] = spc_val[i];
  }
  int32_t n_free = 0;
  for (int64_t g = 0; g < ndof; ++g) dof_eq[g] = dof_eq[g] < 0 ? -1 : n_free++;
  return n_free;
}

typedef struct {
  int64_t* key;
  double* val;
  int64_t n, cap;
} triplets_t;

static int trip_push(triplets_t* t, int64_t key, double v) {
  if (t->n == t->cap) {
    const int64_t nc = t->cap ? 2 * t->cap : 1 << 16;
    int64_t* k = realloc(t->key, (size_t)nc * sizeof(int64_t));
    if (!k) return fail("out of memory");
    t->key = k;
    double* vv = realloc(t->val, (size_t)nc * sizeof(double));
    if (!vv) return fail("out of memory");
    t->val = vv;
    t->cap = nc;
  }
  t->key[t->n] = key;
  t->val[t->n] = v;
  ++t->n;
  return 0;
}

/* Stable LSD radix sort of (key, val) by key; keys are non-negative. */
static int radix_sort(triplets_t* t) {
  const int64_t n = t->n;
  int64_t maxk = 0;
  for (int64_t i = 0; i < n; ++i)
    if (t->key[i] > maxk) maxk = t->key[i];
  int64_t* k2 = malloc((size_t)(n ? n : 1) * sizeof(int64_t));
  double* v2 = malloc((size_t)(n ? n : 1) * sizeof(double));
  if (!k2 || !v2) {
    free(k2);
    free(v2);
    return fail("out of memory");
  }
  for (int shift = 0; shift < 64 && (maxk >> shift) != 0; shift += 11) {
    int64_t cnt[2049];
    memset(cnt, 0, sizeof cnt);
    for (int64_t i = 0; i < n; ++i) ++cnt[((t->key[i] >> shift) & 2047) + 1];
    for (int b = 0; b < 2048; ++b) cnt[b + 1] += cnt[b];
    for (int64_t i = 0; i < n; ++i) {
      const int64_t p = cnt[(t->key[i] >> shift) & 2047]++;
      k2[p] = t->key[i];
      v2[p] = t->val[i];
    }
    int64_t* tk = t->key;
    t->key = k2;
    k2 = tk;
    double* tv = t->val;
    t->val = v2;
    v2 = tv;
  }
  free(k2);
  free(v2);
  return 0;
}

/* scatter_block for an SPC-only transform (assembly.cpp:76-100): free rows receive
 * kab at (eqA, eqB) for free columns and -kab*u_c into rhs for prescribed columns;
 * exact zeros are skipped. */
static int scatter(const double* Ke, int ndof, const int64_t* gd, const int32_t* dof_eq,
                   const double* prescribed, int32_t n_free, triplets_t* t, double* rhs) {
  for (int a = 0; a < ndof; ++a) {
    const int32_t ea = dof_eq[gd[a]];
    const double ca = ea < 0 ? prescribed[gd[a]] : 0.0;
    if (ea < 0 && ca == 0.0) continue;
    for (int b = 0; b < ndof; ++b) {
      const double kab = Ke[a * ndof + b];
      if (kab == 0.0) continue;
      if (ea < 0) continue; /* prescribed row: no free terms */
      const int32_t eb = dof_eq[gd[b]];
      if (eb >= 0) {
        if (trip_push(t, (int64_t)ea * n_free + eb, 1.0 * kab * 1.0)) return -1;
      } else {
        const double cb = prescribed[gd[b]];
        if (cb != 0.0) rhs[ea] -= 1.0 * kab * cb;
      }
    }
  }
  return 0;
}

static cxo_system* finish(triplets_t* t, int32_t n_free, double* rhs) {
  cxo_system* s = calloc(1, sizeof *s);
  if (!s || radix_sort(t)) {
    free(s);
    return NULL;
  }
  int64_t nnz = 0;
  for (int64_t i = 0; i < t->n; ++i)
    if (i == 0 || t->key[i] != t->key[i - 1]) ++nnz;
  s->n_free = n_free;
  s->nnz = nnz;
  s->row_ptr = calloc((size_t)n_free + 1, sizeof(int64_t));
  s->col_idx = malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
  s->vals = malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
  s->rhs = rhs;
  int64_t p = -1;
  for (int64_t i = 0; i < t->n; ++i) {
    if (i == 0 || t->key[i] != t->key[i - 1]) {
      ++p;
      const int32_t r = (int32_t)(t->key[i] / n_free);
      s->col_idx[p] = (int32_t)(t->key[i] % n_free);
      s->vals[p] = 0.0;
      ++s->row_ptr[r + 1];
    }
    s->vals[p] += t->val[i];
  }
  for (int32_t r = 0; r < n_free; ++r) s->row_ptr[r + 1] += s->row_ptr[r];
  free(t->key);
  free(t->val);
  return s;
}

/* add_external_load (assembly.cpp:200-208) */
static void add_external(const double* f_ext, int64_t ndof, const int32_t* dof_eq,
                         double* rhs) {
  if (!f_ext) return;
  for (int64_t g = 0; g < ndof; ++g) {
    if (f_ext[g] == 0.0) continue;
    if (dof_eq[g] >= 0) rhs[dof_eq[g]] += 1.0 * f_ext[g];
  }
}

static cxo_system* assemble(int64_t n_nodes, const double* coords, int64_t n_elems,
                            const int32_t* types, const int64_t* conn_ptr,
                            const int32_t* conn, const int32_t* elem_mat,
                            const cxo_material* mats, const int32_t* dof_eq,
                            const double* prescribed, int32_t n_free, const double* f_ext,
                            const double* u, const double* sc, double* st, double* f_int) {
  triplets_t t = {0};
  double* rhs = calloc((size_t)n_free + 1, sizeof(double));
  double x[3 * MAXN], ue[3 * MAXN], Ke[60 * 60], fe[60];
  int64_t gd[60];
  int64_t gp_off = 0;
  if (f_int) memset(f_int, 0, (size_t)(3 * n_nodes) * sizeof(double));
  for (int64_t e = 0; e < n_elems; ++e) {
    const int type = types[e];
    const int n = cxo_nodes_per_element(type);
    if (n == 0 || conn_ptr[e + 1] - conn_ptr[e] != n) {
      fail("unsupported element type or bad connectivity length");
      goto error;
    }
    const int32_t* c = conn + conn_ptr[e];
    for (int k = 0; k < n; ++k) {
      if (c[k] < 0 || c[k] >= n_nodes) {
        fail("element references unknown node");
        goto error;
      }
      for (int d = 0; d < 3; ++d) {
        x[3 * k + d] = coords[3 * (int64_t)c[k] + d];
        gd[3 * k + d] = 3 * (int64_t)c[k] + d;
        if (u) ue[3 * k + d] = u[3 * (int64_t)c[k] + d];
      }
    }
    const cxo_material* m = &mats[elem_mat[e]];
    double gpb[4 * 27];
    const int ng = cxo_gauss_rule(type, gpb);
    if (u) {
      if (cxo_element_tangent_force(type, x, ue, m, sc + 13 * gp_off, st + 13 * gp_off, Ke, fe))
        goto error;
    } else {
      if (cxo_element_stiffness(type, x, m->E, m->nu, Ke)) goto error;
    }
    gp_off += ng;
    if (scatter(Ke, 3 * n, gd, dof_eq, prescribed, n_free, &t, rhs)) goto error;
    if (f_int)
      for (int a = 0; a < 3 * n; ++a) f_int[gd[a]] += fe[a];
  }
  add_external(f_ext, 3 * n_nodes, dof_eq, rhs);
  {
    cxo_system* s = finish(&t, n_free, rhs);
    if (!s) goto error;
    return s;
  }
error:
  free(t.key);
  free(t.val);
  free(rhs);
  return NULL;
}

cxo_system* cxo_assemble_linear(int64_t n_nodes, const double* coords, int64_t n_elems,
                                const int32_t* types, const int64_t* conn_ptr,
                                const int32_t* conn, const int32_t* elem_mat,
                                const cxo_material* mats, const int32_t* dof_eq,
                                const double* prescribed, int32_t n_free,
                                const double* f_ext) {
  return assemble(n_nodes, coords, n_elems, types, conn_ptr, conn, elem_mat, mats, dof_eq,
                  prescribed, n_free, f_ext, NULL, NULL, NULL, NULL);
}

cxo_system* cxo_assemble_tangent(int64_t n_nodes, const double* coords, int64_t n_elems,
                                 const int32_t* types, const int64_t* conn_ptr,
                                 const int32_t* conn, const int32_t* elem_mat,
                                 const cxo_material* mats, const int32_t* dof_eq,
                                 const double* prescribed, int32_t n_free,
                                 const double* f_ext, const double* u, const double* sc,
                                 double* st, double* f_int) {
  if (!u || !sc || !st || !f_int) {
    fail("tangent assembly needs u, committed state, trial state and f_int");
    return NULL;
  }
  return assemble(n_nodes, coords, n_elems, types, conn_ptr, conn, elem_mat, mats, dof_eq,
                  prescribed, n_free, f_ext, u, sc, st, f_int);
}

/* ---- mass and geometric (initial-stress) stiffness ------------------------------ */
/* element_mass, src/fem/element.cpp:786-812: M[3a+d][3b+d] += (rho detJ w) N_a N_b. */
int cxo_element_mass(int type, const double* x, double rho, double* Me) {
  const int n = cxo_nodes_per_element(type);
  if (n == 0) return fail("unsupported element type");
  const int ndof = 3 * n;
  memset(Me, 0, sizeof(double) * (size_t)ndof * (size_t)ndof);
  if (rho == 0.0) return 0;
  double gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det;
  const int ng = cxo_gauss_rule(type, gp);
  for (int q = 0; q < ng; ++q) {
    cxo_shape(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
    if (gradients_from_shape(n, dN, x, g, &det)) return -1;
    const double scale = rho * det * gp[4 * q + 3];
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        const double m = scale * N[a] * N[b];
        for (int d = 0; d < 3; ++d) Me[(3 * a + d) * ndof + 3 * b + d] += m;
      }
  }
  return 0;
}

/* element_mass_lumped, element.cpp:814-831: the diagonal takes the row sum of the
 * consistent mass. */
int cxo_element_mass_lumped(int type, const double* x, double rho, double* Ml) {
  const int n = cxo_nodes_per_element(type);
  if (n == 0) return fail("unsupported element type");
  const int ndof = 3 * n;
  double Mc[60 * 60];
  if (cxo_element_mass(type, x, rho, Mc)) return -1;
  memset(Ml, 0, sizeof(double) * (size_t)ndof * (size_t)ndof);
  for (int i = 0; i < ndof; ++i) {
    double row = 0.0;
    for (int j = 0; j < ndof; ++j) row += Mc[i * ndof + j];
    Ml[i * ndof + i] = row;
  }
  return 0;
}

/* element_geometric_stiffness + accumulate_kgeo, element.cpp:482-508, 833-854:
 * K[3a+d][3b+d] += (detJ w) (g_a . sigma . g_b) on the upper triangle, then mirrored.
 * gp_stress holds one Voigt6 per Gauss point (may be NULL: zero field). */
int cxo_element_geometric_stiffness(int type, const double* x, const double* gp_stress, double* Ke) {
  const int n = cxo_nodes_per_element(type);
  if (n == 0) return fail("unsupported element type");
  const int ndof = 3 * n;
  memset(Ke, 0, sizeof(double) * (size_t)ndof * (size_t)ndof);
  double gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det;
  const int ng = cxo_gauss_rule(type, gp);
  for (int q = 0; q < ng; ++q) {
    cxo_shape(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
    if (gradients_from_shape(n, dN, x, g, &det)) return -1;
    static const double zero6[6] = {0, 0, 0, 0, 0, 0};
    const double* sg = gp_stress ? gp_stress + 6 * q : zero6;
    const double scale = det * gp[4 * q + 3];
    for (int a = 0; a < n; ++a) {
      const double* ga = g + 3 * a;
      for (int b = a; b < n; ++b) {
        const double* gb = g + 3 * b;
        const double senergy = sg[0] * ga[0] * gb[0] + sg[1] * ga[1] * gb[1] + sg[2] * ga[2] * gb[2] +
                               sg[3] * (ga[0] * gb[1] + ga[1] * gb[0]) +
                               sg[4] * (ga[0] * gb[2] + ga[2] * gb[0]) +
                               sg[5] * (ga[1] * gb[2] + ga[2] * gb[1]);
        const double v = scale * senergy;
        for (int d = 0; d < 3; ++d) {
          const int ia = 3 * a + d, ib = 3 * b + d;
          if (ib >= ia) Ke[ia * ndof + ib] += v;
        }
      }
    }
  }
  mirror_upper(ndof, Ke);
  return 0;
}

/* assemble_mass / assemble_geometric_stiffness, src/fem/assembly.cpp:259-331: the same
 * SPC-only scatter as the stiffness with the rhs side effect discarded (the returned
 * rhs is zero). kind 1: consistent mass, 2: lumped mass, 3: geometric stiffness.
 * density[E] per element (kinds 1, 2); gp_stress[6 * G] (kind 3, element order). */
cxo_system* cxo_assemble_scalar(int kind, int64_t n_nodes, const double* coords, int64_t n_elems,
                                const int32_t* types, const int64_t* conn_ptr, const int32_t* conn,
                                const double* density, const double* gp_stress, const int32_t* dof_eq,
                                const double* prescribed, int32_t n_free) {
  triplets_t t = {0};
  double* rhs = calloc((size_t)n_free + 1, sizeof(double));
  double* dummy = calloc((size_t)n_free + 1, sizeof(double));
  double x[3 * MAXN], Ke[60 * 60];
  int64_t gd[60];
  int64_t gp_off = 0;
  for (int64_t e = 0; e < n_elems; ++e) {
    const int type = types[e];
    const int n = cxo_nodes_per_element(type);
    if (n == 0 || conn_ptr[e + 1] - conn_ptr[e] != n) {
      fail("unsupported element type or bad connectivity length");
      goto error;
    }
    const int32_t* c = conn + conn_ptr[e];
    for (int k = 0; k < n; ++k) {
      if (c[k] < 0 || c[k] >= n_nodes) {
        fail("element references unknown node");
        goto error;
      }
      for (int d = 0; d < 3; ++d) {
        x[3 * k + d] = coords[3 * (int64_t)c[k] + d];
        gd[3 * k + d] = 3 * (int64_t)c[k] + d;
      }
    }
    double gpb[4 * 27];
    const int ng = cxo_gauss_rule(type, gpb);
    int rc;
    if (kind == 1)
      rc = cxo_element_mass(type, x, density[e], Ke);
    else if (kind == 2)
      rc = cxo_element_mass_lumped(type, x, density[e], Ke);
    else
      rc = cxo_element_geometric_stiffness(type, x, gp_stress ? gp_stress + 6 * gp_off : NULL, Ke);
    if (rc) goto error;
    gp_off += ng;
    if (scatter(Ke, 3 * n, gd, dof_eq, prescribed, n_free, &t, dummy)) goto error;
  }
  free(dummy);
  {
    cxo_system* s = finish(&t, n_free, rhs);
    if (!s) goto error2;
    return s;
  }
error:
  free(dummy);
error2:
  free(t.key);
  free(t.val);
  free(rhs);
  return NULL;
}

/* ---- heat conduction: element_conduction (element.cpp:745-765) and
 * assemble_conduction (src/fem/thermal.cpp:92-141) without films: one temperature DOF
 * per node, prescribed temperatures eliminated into the rhs, nodal flux added at the
 * free nodes. */
int cxo_element_conduction(int type, const double* x, double k, double* Kt) {
  const int n = cxo_nodes_per_element(type);
  if (n == 0) return fail("unsupported element type");
  memset(Kt, 0, sizeof(double) * (size_t)n * (size_t)n);
  double gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det;
  const int ng = cxo_gauss_rule(type, gp);
  for (int q = 0; q < ng; ++q) {
    cxo_shape(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
    if (gradients_from_shape(n, dN, x, g, &det)) return -1;
    const double scale = k * det * gp[4 * q + 3];
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        const double dot = g[3 * a] * g[3 * b] + g[3 * a + 1] * g[3 * b + 1] + g[3 * a + 2] * g[3 * b + 2];
        Kt[a * n + b] += scale * dot;
      }
  }
  return 0;
}

/* ---- element faces: src/fem/loads.cpp:13-190, 313-389 --------------------------- */
/* face node tables (0-based), loads.cpp:16-46: tet (T3/T6), hex (Q4/Q8), wedge */
static const int kFaceTet[4][6] = {{0, 2, 1, 6, 5, 4}, {0, 1, 3, 4, 8, 7}, {1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}};
static const int kFaceHex[6][8] = {{0, 1, 2, 3, 8, 9, 10, 11},   {4, 7, 6, 5, 15, 14, 13, 12},
                                   {0, 4, 5, 1, 16, 12, 17, 8},  {1, 5, 6, 2, 17, 13, 18, 9},
                                   {2, 6, 7, 3, 18, 14, 19, 10}, {3, 7, 4, 0, 19, 15, 16, 11}};
static const int kFaceWedge[5][8] = {{0, 2, 1, 8, 7, 6, -1, -1},
                                     {3, 4, 5, 12, 13, 14, -1, -1},
                                     {0, 1, 4, 3, 6, 10, 12, 9},
                                     {1, 2, 5, 4, 7, 11, 13, 10},
                                     {2, 0, 3, 5, 8, 9, 14, 11}};

/* face_kind_of, loads.cpp:317-350: local face nodes fn, count *nf, *quad; -1 on error */
static int face_kind(int type, int face, int* fn, int* nf, int* quad) {
  const int* row = NULL;
  switch (type) {
    case T_C3D4:
    case T_C3D10:
      if (face < 1 || face > 4) return fail("tet face must be 1..4");
      *nf = type == T_C3D4 ? 3 : 6;
      *quad = 0;
      row = kFaceTet[face - 1];
      break;
    case T_C3D8:
    case T_C3D8R:
    case T_C3D20:
    case T_C3D20R:
      if (face < 1 || face > 6) return fail("hex face must be 1..6");
      *nf = (type == T_C3D8 || type == T_C3D8R) ? 4 : 8;
      *quad = 1;
      row = kFaceHex[face - 1];
      break;
    case T_C3D6:
    case T_C3D15:
      if (face < 1 || face > 5) return fail("wedge face must be 1..5");
      *quad = face > 2;
      *nf = face <= 2 ? (type == T_C3D6 ? 3 : 6) : (type == T_C3D6 ? 4 : 8);
      row = kFaceWedge[face - 1];
      break;
    default:
      return fail("unsupported element type for surface load");
  }
  for (int i = 0; i < *nf; ++i) fn[i] = row[i];
  return 0;
}

/* face_shape, loads.cpp:83-138: T3/T6 in barycentric (a, b), Q4/Q8 on [-1,1]^2 */
static void face_shape(int quad, int nf, double a, double b, double* N, double* dxi, double* deta) {
  for (int i = 0; i < 8; ++i) N[i] = dxi[i] = deta[i] = 0.0;
  if (!quad) {
    const double l1 = 1.0 - a - b, l2 = a, l3 = b;
    if (nf == 3) {
      N[0] = l1; N[1] = l2; N[2] = l3;
      dxi[0] = -1; dxi[1] = 1; dxi[2] = 0;
      deta[0] = -1; deta[1] = 0; deta[2] = 1;
      return;
    }
    N[0] = l1 * (2 * l1 - 1); N[1] = l2 * (2 * l2 - 1); N[2] = l3 * (2 * l3 - 1);
    N[3] = 4 * l1 * l2; N[4] = 4 * l2 * l3; N[5] = 4 * l3 * l1;
    dxi[0] = -(4 * l1 - 1); dxi[1] = 4 * l2 - 1; dxi[2] = 0; dxi[3] = 4 * (l1 - l2); dxi[4] = 4 * l3; dxi[5] = -4 * l3;
    deta[0] = -(4 * l1 - 1); deta[1] = 0; deta[2] = 4 * l3 - 1; deta[3] = -4 * l2; deta[4] = 4 * l2;
    deta[5] = 4 * (l1 - l3);
    return;
  }
  static const int sgn[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  if (nf == 4) {
    for (int k = 0; k < 4; ++k) {
      const double g = 1.0 + sgn[k][0] * a, h = 1.0 + sgn[k][1] * b;
      N[k] = 0.25 * g * h;
      dxi[k] = 0.25 * sgn[k][0] * h;
      deta[k] = 0.25 * sgn[k][1] * g;
    }
    return;
  }
  for (int k = 0; k < 4; ++k) {
    const double sa = sgn[k][0], sb = sgn[k][1];
    const double g = 1.0 + sa * a, h = 1.0 + sb * b;
    N[k] = 0.25 * g * h * (sa * a + sb * b - 1.0);
    dxi[k] = 0.25 * (sa * h * (sa * a + sb * b - 1.0) + g * h * sa);
    deta[k] = 0.25 * (sb * g * (sa * a + sb * b - 1.0) + g * h * sb);
  }
  static const int edge_axis[4] = {0, 1, 0, 1};
  static const double edge_fix[4] = {-1, 1, 1, -1};
  for (int e = 0; e < 4; ++e) {
    const int node = 4 + e;
    if (edge_axis[e] == 0) {
      const double sb = edge_fix[e];
      N[node] = 0.5 * (1.0 - a * a) * (1.0 + sb * b);
      dxi[node] = 0.5 * (-2.0 * a) * (1.0 + sb * b);
      deta[node] = 0.5 * (1.0 - a * a) * sb;
    } else {
      const double sa = edge_fix[e];
      N[node] = 0.5 * (1.0 + sa * a) * (1.0 - b * b);
      dxi[node] = 0.5 * sa * (1.0 - b * b);
      deta[node] = 0.5 * (1.0 + sa * a) * (-2.0 * b);
    }
  }
}

/* face_surface_integrals, loads.cpp:361-389: mass[nf*nf] = int N_i N_j dA and
 * load[nf] = int N_i dA over face `face` of an element with node coordinates x; the
 * 3-point triangle rule or the 2x2 quad rule (loads.cpp:54-66), dA = |t_xi x t_eta| w. */
static int face_surface_integrals(int type, int face, const double* x, int* fn, int* nf_out, double* mass,
                                  double* load) {
  static const double kTri[3][3] = {{1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
                                    {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                                    {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
  const double qg = 0.577350269189625764;
  const double kQuad[4][3] = {{-qg, -qg, 1.0}, {qg, -qg, 1.0}, {qg, qg, 1.0}, {-qg, qg, 1.0}};
  int nf = 0, quad = 0;
  if (face_kind(type, face, fn, &nf, &quad)) return -1;
  *nf_out = nf;
  for (int i = 0; i < nf; ++i) load[i] = 0.0;
  for (int i = 0; i < nf * nf; ++i) mass[i] = 0.0;
  const int ng = quad ? 4 : 3;
  for (int q = 0; q < ng; ++q) {
    const double* gp = quad ? kQuad[q] : kTri[q];
    double N[8], dxi[8], deta[8], txi[3] = {0, 0, 0}, teta[3] = {0, 0, 0};
    face_shape(quad, nf, gp[0], gp[1], N, dxi, deta);
    for (int i = 0; i < nf; ++i)
      for (int d = 0; d < 3; ++d) {
        txi[d] += dxi[i] * x[3 * fn[i] + d];
        teta[d] += deta[i] * x[3 * fn[i] + d];
      }
    const double nrm[3] = {txi[1] * teta[2] - txi[2] * teta[1], txi[2] * teta[0] - txi[0] * teta[2],
                           txi[0] * teta[1] - txi[1] * teta[0]};
    const double dA = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]) * gp[2];
    for (int i = 0; i < nf; ++i) {
      const double Ni = N[i];
      load[i] += Ni * dA;
      for (int j = 0; j < nf; ++j) mass[i * nf + j] += Ni * N[j] * dA;
    }
  }
  return 0;
}

/* assemble_conduction, thermal.cpp:92-141, with *FILM faces (thermal.cpp:113-126): after
 * the elements, each film adds h * mass to the matrix (scattered like an element block)
 * and h * T_sink * load to the free rhs rows; then the nodal flux. */
cxo_system* cxo_assemble_conduction_films(int64_t n_nodes, const double* coords, int64_t n_elems,
                                          const int32_t* types, const int64_t* conn_ptr, const int32_t* conn,
                                          const double* conductivity, const int32_t* t_dof_eq,
                                          const double* t_prescribed, int32_t n_free, const double* flux,
                                          int64_t n_films, const int64_t* film_elem, const int32_t* film_face,
                                          const double* film_h, const double* film_sink) {
  triplets_t t = {0};
  double* rhs = calloc((size_t)n_free + 1, sizeof(double));
  double x[3 * MAXN], Kt[MAXN * MAXN];
  int64_t gd[MAXN];
  for (int64_t e = 0; e < n_elems; ++e) {
    const int n = cxo_nodes_per_element(types[e]);
    const int32_t* c = conn + conn_ptr[e];
    if (n == 0 || conn_ptr[e + 1] - conn_ptr[e] != n) {
      fail("unsupported element type or bad connectivity length");
      goto error;
    }
    for (int k = 0; k < n; ++k) {
      if (c[k] < 0 || c[k] >= n_nodes) {
        fail("element references unknown node");
        goto error;
      }
      gd[k] = c[k];
      for (int d = 0; d < 3; ++d) x[3 * k + d] = coords[3 * (int64_t)c[k] + d];
    }
    if (cxo_element_conduction(types[e], x, conductivity[e], Kt)) goto error;
    if (scatter(Kt, n, gd, t_dof_eq, t_prescribed, n_free, &t, rhs)) goto error;
  }
  for (int64_t f = 0; f < n_films; ++f) {
    const int64_t e = film_elem[f];
    if (e < 0 || e >= n_elems) {
      fail("*FILM references unknown element");
      goto error;
    }
    const int n = cxo_nodes_per_element(types[e]);
    const int32_t* c = conn + conn_ptr[e];
    for (int k = 0; k < n; ++k)
      for (int d = 0; d < 3; ++d) x[3 * k + d] = coords[3 * (int64_t)c[k] + d];
    int fn[8], nf = 0;
    double mass[64], load[8], hM[64];
    int64_t fg[8];
    if (face_surface_integrals(types[e], film_face[f], x, fn, &nf, mass, load)) goto error;
    for (int i = 0; i < nf * nf; ++i) hM[i] = film_h[f] * mass[i];
    for (int i = 0; i < nf; ++i) fg[i] = c[fn[i]];
    if (scatter(hM, nf, fg, t_dof_eq, t_prescribed, n_free, &t, rhs)) goto error;
    for (int i = 0; i < nf; ++i) {
      const int32_t eq = t_dof_eq[fg[i]];
      if (eq >= 0) rhs[eq] += film_h[f] * film_sink[f] * load[i];
    }
  }
  if (flux)
    for (int64_t i = 0; i < n_nodes; ++i)
      if (t_dof_eq[i] >= 0) rhs[t_dof_eq[i]] += flux[i];
  {
    cxo_system* s = finish(&t, n_free, rhs);
    if (!s) goto error;
    return s;
  }
error:
  free(t.key);
  free(t.val);
  free(rhs);
  return NULL;
}

cxo_system* cxo_assemble_conduction(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                                    const int64_t* conn_ptr, const int32_t* conn, const double* conductivity,
                                    const int32_t* t_dof_eq, const double* t_prescribed, int32_t n_free,
                                    const double* flux) {
  return cxo_assemble_conduction_films(n_nodes, coords, n_elems, types, conn_ptr, conn, conductivity, t_dof_eq,
                                       t_prescribed, n_free, flux, 0, NULL, NULL, NULL, NULL);
}

/* ---- field recovery and thermal strain: src/fem/stress.cpp, src/fem/loads.cpp ---- */
/* strain_stress_at, stress.cpp:19-42: du[i][j] = sum_k g_k[j] u_k[i], engineering strain,
 * sigma = D (eps - eps_th) with eps_th = {eth, eth, eth, 0, 0, 0}. */
static void strain_stress_at(const double* g, int n, const double* ue, const double* D, double eth, double* strain,
                             double* stress) {
  const double eps_th[6] = {eth, eth, eth, 0.0, 0.0, 0.0};
  double du[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < n; ++k) v += g[3 * k + j] * ue[3 * k + i];
      du[i][j] = v;
    }
  strain[0] = du[0][0];
  strain[1] = du[1][1];
  strain[2] = du[2][2];
  strain[3] = du[0][1] + du[1][0];
  strain[4] = du[0][2] + du[2][0];
  strain[5] = du[1][2] + du[2][1];
  for (int i = 0; i < 6; ++i) {
    double v = 0.0;
    for (int j = 0; j < 6; ++j) v += D[6 * i + j] * (strain[j] - eps_th[j]);
    stress[i] = v;
  }
}

static int gather_element(int64_t n_nodes, const double* coords, const int32_t* c, int n, const double* u,
                          double* x, double* ue) {
  for (int k = 0; k < n; ++k) {
    if (c[k] < 0 || c[k] >= n_nodes) return fail("element references unknown node");
    for (int d = 0; d < 3; ++d) {
      x[3 * k + d] = coords[3 * (int64_t)c[k] + d];
      ue[3 * k + d] = u[3 * (int64_t)c[k] + d];
    }
  }
  return 0;
}

/* Thermal-strain inputs of one element (NULL node_temp: none). te_k = T_k - t_ref where
 * node k has an applied temperature, 0 elsewhere (element_temp_change, stress.cpp:76-91;
 * thermal_strain_load_vector takes T = t_ref at such nodes, loads.cpp:537-541, the same
 * te). alpha is the element's expansion coefficient as the caller evaluated its table at
 * the element's mean temperature (element_alpha, stress.cpp:97-105; loads.cpp:548-550),
 * 0 without *EXPANSION. Returns 1 when some te_k is nonzero and alpha is nonzero. */
static int element_te(const double* node_temp, const uint8_t* node_applied, const double* elem_alpha,
                      const double* elem_tref, int64_t e, const int32_t* c, int n, double* te, double* alpha) {
  int any = 0;
  *alpha = node_temp && elem_alpha ? elem_alpha[e] : 0.0;
  for (int k = 0; k < n; ++k) {
    te[k] = 0.0;
    if (node_temp && (!node_applied || node_applied[c[k]])) te[k] = node_temp[c[k]] - elem_tref[e];
    if (te[k] != 0.0) any = 1;
  }
  return any && *alpha != 0.0;
}

/* element_thermal_load, element.cpp:636-665: fe = sum_q det w B^T D eps_th,
 * eps_th = alpha sum_k N_k te_k on the normal components. */
static int element_thermal_load(int type, const double* x, const double* D, double alpha, const double* te,
                                double* fe) {
  double gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det;
  const int n = cxo_nodes_per_element(type), ndof = 3 * n;
  memset(fe, 0, sizeof(double) * (size_t)ndof);
  const int ng = cxo_gauss_rule(type, gp);
  for (int q = 0; q < ng; ++q) {
    cxo_shape(type, gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
    if (gradients_from_shape(n, dN, x, g, &det)) return -1;
    double dT = 0.0;
    for (int k = 0; k < n; ++k) dT += N[k] * te[k];
    const double eth = alpha * dT;
    const double eps_th[6] = {eth, eth, eth, 0.0, 0.0, 0.0};
    double sig_th[6];
    for (int i = 0; i < 6; ++i) {
      double v = 0.0;
      for (int j = 0; j < 6; ++j) v += D[6 * i + j] * eps_th[j];
      sig_th[i] = v;
    }
    accumulate_fint(g, ndof, sig_th, det * gp[4 * q + 3], fe);
  }
  return 0;
}

/* thermal_strain_load_vector, loads.cpp:515-560: f[3 * n_nodes] = sum over the elements
 * with an expansion coefficient and a temperature change of element_thermal_load. */
int cxo_thermal_strain_load(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                            const int64_t* conn_ptr, const int32_t* conn, const double* young, const double* poisson,
                            const double* node_temp, const uint8_t* node_applied, const double* elem_alpha,
                            const double* elem_tref, double* f) {
  double x[3 * MAXN], D[36], te[MAXN], fe[3 * MAXN], alpha;
  memset(f, 0, sizeof(double) * 3 * (size_t)n_nodes);
  for (int64_t e = 0; e < n_elems; ++e) {
    const int n = cxo_nodes_per_element(types[e]);
    const int32_t* c = conn + conn_ptr[e];
    if (n == 0 || conn_ptr[e + 1] - conn_ptr[e] != n) return fail("unsupported element type or bad connectivity");
    for (int k = 0; k < n; ++k) {
      if (c[k] < 0 || c[k] >= n_nodes) return fail("element references unknown node");
      for (int d = 0; d < 3; ++d) x[3 * k + d] = coords[3 * (int64_t)c[k] + d];
    }
    if (!element_te(node_temp, node_applied, elem_alpha, elem_tref, e, c, n, te, &alpha)) continue;
    elastic_D(young[e], poisson[e], D);
    if (element_thermal_load(types[e], x, D, alpha, te, fe)) return -1;
    for (int a = 0; a < 3 * n; ++a) f[3 * (int64_t)c[a / 3] + a % 3] += fe[a];
  }
  return 0;
}

/* recover_gauss_stress, stress.cpp:147-187: out[6 * G] (element order, Gauss-rule order);
 * young/poisson per element. */
int cxo_recover_gauss_stress_th(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                                const int64_t* conn_ptr, const int32_t* conn, const double* young,
                                const double* poisson, const double* node_temp, const uint8_t* node_applied,
                                const double* elem_alpha, const double* elem_tref, const double* u, double* out) {
  double x[3 * MAXN], ue[3 * MAXN], D[36], gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det, strain[6];
  double te[MAXN], alpha;
  int64_t off = 0;
  for (int64_t e = 0; e < n_elems; ++e) {
    const int n = cxo_nodes_per_element(types[e]);
    if (n == 0 || conn_ptr[e + 1] - conn_ptr[e] != n) return fail("unsupported element type or bad connectivity");
    if (gather_element(n_nodes, coords, conn + conn_ptr[e], n, u, x, ue)) return -1;
    elastic_D(young[e], poisson[e], D);
    const int th = element_te(node_temp, node_applied, elem_alpha, elem_tref, e, conn + conn_ptr[e], n, te, &alpha);
    const int ng = cxo_gauss_rule(types[e], gp);
    for (int q = 0; q < ng; ++q, ++off) {
      cxo_shape(types[e], gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
      if (gradients_from_shape(n, dN, x, g, &det)) return -1;
      double dT = 0.0;
      for (int k = 0; k < n; ++k) dT += N[k] * (th ? te[k] : 0.0);
      strain_stress_at(g, n, ue, D, th ? alpha * dT : 0.0, strain, out + 6 * off);
    }
  }
  return 0;
}

int cxo_recover_gauss_stress(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                             const int64_t* conn_ptr, const int32_t* conn, const double* young,
                             const double* poisson, const double* u, double* out) {
  return cxo_recover_gauss_stress_th(n_nodes, coords, n_elems, types, conn_ptr, conn, young, poisson, NULL, NULL,
                                     NULL, NULL, u, out);
}

/* recover_fields, stress.cpp:189-271 (elastic): nodal strain/stress averaged over the
 * incident elements, reaction = f_int - f_ext with f_int = sum_e (K_e u_e - f_th_e)
 * (accumulate_internal_force, stress.cpp:56-75); thermal inputs as element_te. */
int cxo_recover_fields_th(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                          const int64_t* conn_ptr, const int32_t* conn, const double* young, const double* poisson,
                          const double* node_temp, const uint8_t* node_applied, const double* elem_alpha,
                          const double* elem_tref, const double* u, const double* f_ext, double* strain_out,
                          double* stress_out, double* reaction) {
  double x[3 * MAXN], ue[3 * MAXN], D[36], gp[4 * 27], N[MAXN], dN[3 * MAXN], g[3 * MAXN], det;
  double Ke[60 * 60], gs[27][6], ge[27][6], te[MAXN], fth[3 * MAXN], alpha;
  int* count = calloc((size_t)n_nodes, sizeof(int));
  double* f_int = calloc((size_t)(3 * n_nodes), sizeof(double));
  if (!count || !f_int) {
    free(count);
    free(f_int);
    return fail("out of memory");
  }
  memset(strain_out, 0, sizeof(double) * 6 * (size_t)n_nodes);
  memset(stress_out, 0, sizeof(double) * 6 * (size_t)n_nodes);
  int rc = 0;
  for (int64_t e = 0; e < n_elems && !rc; ++e) {
    const int n = cxo_nodes_per_element(types[e]);
    const int32_t* c = conn + conn_ptr[e];
    if (n == 0 || conn_ptr[e + 1] - conn_ptr[e] != n) {
      rc = fail("unsupported element type or bad connectivity");
      break;
    }
    if ((rc = gather_element(n_nodes, coords, c, n, u, x, ue))) break;
    elastic_D(young[e], poisson[e], D);
    /* thermal strain and its equivalent load (stress.cpp:207-213) */
    const int th = element_te(node_temp, node_applied, elem_alpha, elem_tref, e, c, n, te, &alpha);
    if (th && (rc = element_thermal_load(types[e], x, D, alpha, te, fth))) break;
    if ((rc = cxo_element_stiffness(types[e], x, young[e], poisson[e], Ke))) break;
    const int ndof = 3 * n;
    /* f_int_e = K_e u_e - f_th_e (accumulate_internal_force, stress.cpp:56-75) */
    for (int a = 0; a < ndof; ++a) {
      double v = 0.0;
      for (int b = 0; b < ndof; ++b) v += Ke[a * ndof + b] * ue[b];
      if (th) v -= fth[a];
      f_int[3 * (int64_t)c[a / 3] + a % 3] += v;
    }
    const int ng = cxo_gauss_rule(types[e], gp);
    for (int q = 0; q < ng; ++q) {
      cxo_shape(types[e], gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], N, dN);
      if ((rc = gradients_from_shape(n, dN, x, g, &det))) break;
      double dT = 0.0;
      for (int k = 0; k < n; ++k) dT += N[k] * (th ? te[k] : 0.0);
      strain_stress_at(g, n, ue, D, th ? alpha * dT : 0.0, ge[q], gs[q]);
    }
    if (rc) break;
    /* extrapolate_gp_to_nodes (extrapolation.hpp:26-55): C3D10 corners by the a4 matrix
     * of CalculiX extrapolate.f, midsides the mean of their edge's corners; the other
     * families the Gauss-point mean at every node (a single point for C3D4). */
    double ne[MAXN][6], ns[MAXN][6];
    if (types[e] == T_C3D10) {
      static const double kA4diag = 1.927050983124842, kA4off = -0.309016994374947;
      static const int kMid[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
      for (int cn = 0; cn < 4; ++cn)
        for (int k = 0; k < 6; ++k) {
          double ve = 0.0, vs = 0.0;
          for (int l = 0; l < 4; ++l) {
            ve += (cn == l ? kA4diag : kA4off) * ge[l][k];
            vs += (cn == l ? kA4diag : kA4off) * gs[l][k];
          }
          ne[cn][k] = ve;
          ns[cn][k] = vs;
        }
      for (int m = 0; m < 6; ++m)
        for (int k = 0; k < 6; ++k) {
          ne[4 + m][k] = 0.5 * (ne[kMid[m][0]][k] + ne[kMid[m][1]][k]);
          ns[4 + m][k] = 0.5 * (ns[kMid[m][0]][k] + ns[kMid[m][1]][k]);
        }
    } else {
      double ms[6] = {0}, me[6] = {0};
      for (int q = 0; q < ng; ++q)
        for (int k = 0; k < 6; ++k) {
          me[k] += ge[q][k];
          ms[k] += gs[q][k];
        }
      const double inv = ng ? 1.0 / (double)ng : 0.0;
      for (int k = 0; k < 6; ++k) {
        me[k] *= inv;
        ms[k] *= inv;
      }
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 6; ++k) {
          ne[i][k] = me[k];
          ns[i][k] = ms[k];
        }
    }
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 6; ++k) {
        strain_out[6 * (int64_t)c[i] + k] += ne[i][k];
        stress_out[6 * (int64_t)c[i] + k] += ns[i][k];
      }
      ++count[c[i]];
    }
  }
  if (!rc) {
    for (int64_t i = 0; i < n_nodes; ++i)
      if (count[i] > 0)
        for (int k = 0; k < 6; ++k) {
          strain_out[6 * i + k] /= count[i];
          stress_out[6 * i + k] /= count[i];
        }
    for (int64_t i = 0; i < 3 * n_nodes; ++i) reaction[i] = f_int[i] - (f_ext ? f_ext[i] : 0.0);
  }
  free(count);
  free(f_int);
  return rc;
}

int cxo_recover_fields(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                       const int64_t* conn_ptr, const int32_t* conn, const double* young, const double* poisson,
                       const double* u, const double* f_ext, double* strain_out, double* stress_out,
                       double* reaction) {
  return cxo_recover_fields_th(n_nodes, coords, n_elems, types, conn_ptr, conn, young, poisson, NULL, NULL, NULL, NULL,
                               u, f_ext, strain_out, stress_out, reaction);
}

int cxo_system_info(const cxo_system* s, int32_t* n_free, int64_t* nnz) {
  *n_free = s->n_free;
  *nnz = s->nnz;
  return 0;
}

int cxo_system_copy(const cxo_system* s, int64_t* row_ptr, int32_t* col_idx, double* vals,
                    double* rhs) {
  memcpy(row_ptr, s->row_ptr, ((size_t)s->n_free + 1) * sizeof(int64_t));
  memcpy(col_idx, s->col_idx, (size_t)s->nnz * sizeof(int32_t));
  memcpy(vals, s->vals, (size_t)s->nnz * sizeof(double));
  memcpy(rhs, s->rhs, (size_t)s->n_free * sizeof(double));
  return 0;
}

void cxo_system_free(cxo_system* s) {
  if (!s) return;
  free(s->row_ptr);
  free(s->col_idx);
  free(s->vals);
  free(s->rhs);
  free(s);
}

/* ---- per-element compliance derivative by central differences ------------------- */
int cxo_element_compliance_grad_fd(int type, const double* coords, const double* ue,
                                   double E, double nu, double h, double* dcdX) {
  const int n = cxo_nodes_per_element(type);
  if (n == 0) return fail("unsupported element type");
  const int ndof = 3 * n;
  double xp[3 * MAXN], Kp[60 * 60], Km[60 * 60];
  for (int v = 0; v < ndof; ++v) {
    memcpy(xp, coords, (size_t)ndof * sizeof(double));
    xp[v] = coords[v] + h;
    if (cxo_element_stiffness(type, xp, E, nu, Kp)) return -1;
    xp[v] = coords[v] - h;
    if (cxo_element_stiffness(type, xp, E, nu, Km)) return -1;
    double s = 0.0;
    for (int a = 0; a < ndof; ++a) {
      double r = 0.0;
      for (int b = 0; b < ndof; ++b) r += (Kp[a * ndof + b] - Km[a * ndof + b]) * ue[b];
      s += ue[a] * r;
    }
    dcdX[v] = -s / (2.0 * h);
  }
  return 0;
}
