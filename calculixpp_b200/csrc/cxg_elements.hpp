// Element families of the hot path: Gauss rules and shape-function derivatives.
//
// Evaluated once on the host in double precision to fill the constant tables the
// kernels read (natural derivatives dN_k/dxi at every Gauss point are the same for all
// elements of a family, so the device never re-evaluates shape functions).
//
// The quadrature rules are the reference's (src/fem/element.cpp:22-126): 2x2x2 Gauss
// at +-1/sqrt(3) with unit weights, centroid with weight 8, 3x3x3 Gauss-Legendre at
// 0,+-sqrt(3/5) with weights 8/9, 5/9, and the wedge triangle-x-line rules; points are
// ordered xi fastest, then eta, then zeta. The shape functions are the standard
// isoparametric ones of CalculiX's shape8h/shape20h/shape6w/shape15w
// (element.cpp:160-330), written here from node natural coordinates: trilinear and
// serendipity hexahedra, linear and quadratic wedges over area coordinates, linear and
// quadratic tetrahedra over volume coordinates (shape4tet / shape10tet, element.cpp:130-158).
#pragma once

#include <cmath>
#include <cstdint>

namespace cxg {

enum ElemType : int32_t { C3D4 = 0, C3D10 = 1, C3D8 = 2, C3D8R = 3, C3D20 = 4, C3D20R = 5, C3D6 = 6, C3D15 = 7 };
constexpr int kFirstType = C3D4, kLastType = C3D15;

constexpr int kMaxNodes = 20;
constexpr int kMaxGauss = 27;

constexpr int nodes_of(int t) {
  return (t == C3D8 || t == C3D8R) ? 8 : (t == C3D20 || t == C3D20R) ? 20 : t == C3D6 ? 6 : t == C3D15 ? 15
         : t == C3D4 ? 4 : t == C3D10 ? 10 : 0;
}
constexpr int gauss_of(int t) {
  return t == C3D8 ? 8 : t == C3D8R ? 1 : t == C3D20 ? 27 : t == C3D20R ? 8 : t == C3D6 ? 2 : t == C3D15 ? 6
         : t == C3D4 ? 1 : t == C3D10 ? 4 : 0;
}
constexpr bool supported(int t) { return nodes_of(t) != 0; }

struct GaussPt {
  double xi, et, ze, w;
};

// Gauss rule of family t into pts[]; returns the point count.
inline int gauss_rule(int t, GaussPt* pts) {
  const double g2 = 1.0 / std::sqrt(3.0);
  const double g3 = std::sqrt(3.0 / 5.0);
  int n = 0;
  if (t == C3D8 || t == C3D20R) {
    for (int c = 0; c < 2; ++c)
      for (int b = 0; b < 2; ++b)
        for (int a = 0; a < 2; ++a) pts[n++] = {a ? g2 : -g2, b ? g2 : -g2, c ? g2 : -g2, 1.0};
  } else if (t == C3D8R) {
    pts[n++] = {0.0, 0.0, 0.0, 8.0};
  } else if (t == C3D20) {
    const double x[3] = {-g3, 0.0, g3};
    const double w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for (int c = 0; c < 3; ++c)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) pts[n++] = {x[a], x[b], x[c], w[a] * w[b] * w[c]};
  } else if (t == C3D6) {
    pts[n++] = {1.0 / 3.0, 1.0 / 3.0, -g2, 0.5};
    pts[n++] = {1.0 / 3.0, 1.0 / 3.0, g2, 0.5};
  } else if (t == C3D4) {
    pts[n++] = {0.25, 0.25, 0.25, 1.0 / 6.0};
  } else if (t == C3D10) {
    // 4-point tetrahedral rule: abscissae a = (5 - sqrt 5)/20 and b = 1 - 3a, the
    // decimal values of src/fem/element.cpp:10-20.
    const double a = 0.138196601125010515, b = 0.585410196624968454;
    pts[n++] = {a, a, a, 1.0 / 24.0};
    pts[n++] = {b, a, a, 1.0 / 24.0};
    pts[n++] = {a, b, a, 1.0 / 24.0};
    pts[n++] = {a, a, b, 1.0 / 24.0};
  } else if (t == C3D15) {
    const double tri[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
    for (int c = 0; c < 2; ++c)
      for (int k = 0; k < 3; ++k) pts[n++] = {tri[k][0], tri[k][1], c ? g2 : -g2, 1.0 / 6.0};
  }
  return n;
}

// Natural coordinates of the 20 serendipity-hexahedron nodes (corners then the edge
// midsides 9-20 of CalculiX ordering); the first 8 are the trilinear hex's nodes.
inline void hex_node_coords(double (*p)[3]) {
  static const int c[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                              {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  static const int e[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                               {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int k = 0; k < 8; ++k)
    for (int d = 0; d < 3; ++d) p[k][d] = c[k][d];
  for (int j = 0; j < 12; ++j)
    for (int d = 0; d < 3; ++d) p[8 + j][d] = 0.5 * (c[e[j][0]][d] + c[e[j][1]][d]);
}

// Natural derivatives dN[k][d] (and values N[k]) of family t at (xi, et, ze).
inline int shape_derivatives(int t, double xi, double et, double ze, double* N, double (*dN)[3]) {
  const double q[3] = {xi, et, ze};
  if (t == C3D8 || t == C3D8R || t == C3D20 || t == C3D20R) {
    double p[20][3];
    hex_node_coords(p);
    const int n = nodes_of(t);
    for (int k = 0; k < n; ++k) {
      double f[3], df[3];
      const bool corner = k < 8;
      if (!corner || n == 8) {
        // Product of one 1-D factor per axis: (1 + p q)/2 at a nonzero natural
        // coordinate, (1 - q^2) at a zero one (edge midside).
        for (int d = 0; d < 3; ++d) {
          if (p[k][d] != 0.0) {
            f[d] = 0.5 * (1.0 + p[k][d] * q[d]);
            df[d] = 0.5 * p[k][d];
          } else {
            f[d] = 1.0 - q[d] * q[d];
            df[d] = -2.0 * q[d];
          }
        }
        // hex8: (1/2)^3 prod(1 + p q) = N; edge midside: (1/2)^2 (1 - q_a^2) prod(1 + p q).
        N[k] = f[0] * f[1] * f[2];
        dN[k][0] = df[0] * f[1] * f[2];
        dN[k][1] = f[0] * df[1] * f[2];
        dN[k][2] = f[0] * f[1] * df[2];
      } else {
        // Serendipity corner: (1/8) prod(1 + p_d q_d) (p.q - 2).
        double g[3];
        for (int d = 0; d < 3; ++d) g[d] = 1.0 + p[k][d] * q[d];
        const double lin = p[k][0] * q[0] + p[k][1] * q[1] + p[k][2] * q[2] - 2.0;
        const double prod = g[0] * g[1] * g[2];
        N[k] = 0.125 * prod * lin;
        for (int d = 0; d < 3; ++d) {
          double others = 1.0;
          for (int m = 0; m < 3; ++m)
            if (m != d) others *= g[m];
          dN[k][d] = 0.125 * (p[k][d] * others * lin + prod * p[k][d]);
        }
      }
    }
    return n;
  }
  // Tetrahedra: volume coordinates L = (1 - xi - et - ze, xi, et, ze).
  if (t == C3D4 || t == C3D10) {
    const double L[4] = {1.0 - xi - et - ze, xi, et, ze};
    const double dL[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    if (t == C3D4) {
      for (int k = 0; k < 4; ++k) {
        N[k] = L[k];
        for (int d = 0; d < 3; ++d) dN[k][d] = dL[k][d];
      }
      return 4;
    }
    // corners L_i (2 L_i - 1); midsides 4 L_i L_j on edges (0,1) (1,2) (2,0) (0,3) (1,3) (2,3)
    for (int k = 0; k < 4; ++k) {
      N[k] = L[k] * (2.0 * L[k] - 1.0);
      for (int d = 0; d < 3; ++d) dN[k][d] = (4.0 * L[k] - 1.0) * dL[k][d];
    }
    static const int edge[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    for (int m = 0; m < 6; ++m) {
      const int i = edge[m][0], j = edge[m][1];
      N[4 + m] = 4.0 * L[i] * L[j];
      for (int d = 0; d < 3; ++d) dN[4 + m][d] = 4.0 * (dL[i][d] * L[j] + L[i] * dL[j][d]);
    }
    return 10;
  }
  // Wedges: area coordinates L = (1 - xi - et, xi, et), dL/dxi = (-1,1,0), dL/det = (-1,0,1).
  const double L[3] = {1.0 - xi - et, xi, et};
  const double dLx[3] = {-1.0, 1.0, 0.0}, dLy[3] = {-1.0, 0.0, 1.0};
  if (t == C3D6) {
    for (int c = 0; c < 2; ++c) {
      const double sz = c ? 1.0 : -1.0;
      const double h = 0.5 * (1.0 + sz * ze), dh = 0.5 * sz;
      for (int i = 0; i < 3; ++i) {
        const int k = 3 * c + i;
        N[k] = L[i] * h;
        dN[k][0] = dLx[i] * h;
        dN[k][1] = dLy[i] * h;
        dN[k][2] = L[i] * dh;
      }
    }
    return 6;
  }
  if (t == C3D15) {
    // Corners: (1/2) L_i (1 + s z)(2 L_i + s z - 2).
    for (int c = 0; c < 2; ++c) {
      const double s = c ? 1.0 : -1.0;
      for (int i = 0; i < 3; ++i) {
        const int k = 3 * c + i;
        const double h = 1.0 + s * ze, r = 2.0 * L[i] + s * ze - 2.0;
        N[k] = 0.5 * L[i] * h * r;
        dN[k][0] = 0.5 * dLx[i] * h * (r + 2.0 * L[i]);
        dN[k][1] = 0.5 * dLy[i] * h * (r + 2.0 * L[i]);
        dN[k][2] = 0.5 * L[i] * s * (r + h);
      }
    }
    // Triangle-edge midsides on the two end faces: 2 L_i L_j (1 + s z).
    static const int tri_edge[3][2] = {{0, 1}, {1, 2}, {2, 0}};
    for (int c = 0; c < 2; ++c) {
      const double s = c ? 1.0 : -1.0;
      for (int m = 0; m < 3; ++m) {
        const int k = 6 + 3 * c + m;
        const int i = tri_edge[m][0], j = tri_edge[m][1];
        const double h = 1.0 + s * ze;
        N[k] = 2.0 * L[i] * L[j] * h;
        dN[k][0] = 2.0 * (dLx[i] * L[j] + L[i] * dLx[j]) * h;
        dN[k][1] = 2.0 * (dLy[i] * L[j] + L[i] * dLy[j]) * h;
        dN[k][2] = 2.0 * L[i] * L[j] * s;
      }
    }
    // Vertical-edge midsides: L_i (1 - z^2).
    for (int i = 0; i < 3; ++i) {
      const int k = 12 + i;
      const double h = 1.0 - ze * ze;
      N[k] = L[i] * h;
      dN[k][0] = dLx[i] * h;
      dN[k][1] = dLy[i] * h;
      dN[k][2] = L[i] * (-2.0 * ze);
    }
    return 15;
  }
  return 0;
}

}  // namespace cxg
