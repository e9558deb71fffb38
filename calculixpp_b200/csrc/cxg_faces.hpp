// Element faces for surface terms (*FILM): local face nodes, face shape functions and
// the face quadrature of the reference's surface loads (src/fem/loads.cpp:13-190,
// 313-389). The node orders follow CalculiX (ifacet / ifaceq / ifacew, corners so that
// t_xi x t_eta points outward, then midsides); they are element-definition data, so they
// are the same tables. Host and device.
#pragma once

#include <cstdint>

#include "cxg_elements.hpp"

namespace cxg {

// Local nodes of face `face` (1-based) of an element of `type`: fn[0..nf), quad face or
// triangle. Returns false for a face number outside the family's range.
__host__ __device__ inline bool face_nodes_of(int type, int face, int* fn, int* nf, bool* quad) {
  constexpr int kTet[4][6] = {{0, 2, 1, 6, 5, 4}, {0, 1, 3, 4, 8, 7}, {1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}};
  constexpr int kHex[6][8] = {{0, 1, 2, 3, 8, 9, 10, 11},   {4, 7, 6, 5, 15, 14, 13, 12},
                              {0, 4, 5, 1, 16, 12, 17, 8},  {1, 5, 6, 2, 17, 13, 18, 9},
                              {2, 6, 7, 3, 18, 14, 19, 10}, {3, 7, 4, 0, 19, 15, 16, 11}};
  constexpr int kWedge[5][8] = {{0, 2, 1, 8, 7, 6, -1, -1},
                                {3, 4, 5, 12, 13, 14, -1, -1},
                                {0, 1, 4, 3, 6, 10, 12, 9},
                                {1, 2, 5, 4, 7, 11, 13, 10},
                                {2, 0, 3, 5, 8, 9, 14, 11}};
  if (type == C3D4 || type == C3D10) {
    if (face < 1 || face > 4) return false;
    *nf = type == C3D4 ? 3 : 6;
    *quad = false;
    for (int i = 0; i < *nf; ++i) fn[i] = kTet[face - 1][i];
    return true;
  }
  if (type == C3D8 || type == C3D8R || type == C3D20 || type == C3D20R) {
    if (face < 1 || face > 6) return false;
    *nf = (type == C3D8 || type == C3D8R) ? 4 : 8;
    *quad = true;
    for (int i = 0; i < *nf; ++i) fn[i] = kHex[face - 1][i];
    return true;
  }
  if (type == C3D6 || type == C3D15) {
    if (face < 1 || face > 5) return false;
    *quad = face > 2;
    *nf = face <= 2 ? (type == C3D6 ? 3 : 6) : (type == C3D6 ? 4 : 8);
    for (int i = 0; i < *nf; ++i) fn[i] = kWedge[face - 1][i];
    return true;
  }
  return false;
}

// Face shape functions N and their natural derivatives at (a, b): T3 / T6 in
// barycentric coordinates on the unit triangle (l1 = 1 - a - b, l2 = a, l3 = b), Q4 /
// Q8 (serendipity: corners, then the midsides of edges 0-1, 1-2, 2-3, 3-0) on [-1,1]^2.
__host__ __device__ inline void face_shape(bool quad, int nf, double a, double b, double* N, double* dxi,
                                           double* deta) {
  for (int i = 0; i < 8; ++i) N[i] = dxi[i] = deta[i] = 0.0;
  if (!quad) {
    const double l1 = 1.0 - a - b, l2 = a, l3 = b;
    if (nf == 3) {
      N[0] = l1, N[1] = l2, N[2] = l3;
      dxi[0] = -1, dxi[1] = 1;
      deta[0] = -1, deta[2] = 1;
      return;
    }
    N[0] = l1 * (2 * l1 - 1), N[1] = l2 * (2 * l2 - 1), N[2] = l3 * (2 * l3 - 1);
    N[3] = 4 * l1 * l2, N[4] = 4 * l2 * l3, N[5] = 4 * l3 * l1;
    dxi[0] = -(4 * l1 - 1), dxi[1] = 4 * l2 - 1, dxi[3] = 4 * (l1 - l2), dxi[4] = 4 * l3, dxi[5] = -4 * l3;
    deta[0] = -(4 * l1 - 1), deta[2] = 4 * l3 - 1, deta[3] = -4 * l2, deta[4] = 4 * l2, deta[5] = 4 * (l1 - l3);
    return;
  }
  constexpr int sgn[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
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
  // midsides 4, 6 on the edges b = -1, +1 (a varies); 5, 7 on a = +1, -1 (b varies)
  N[4] = 0.5 * (1.0 - a * a) * (1.0 - b), dxi[4] = -a * (1.0 - b), deta[4] = -0.5 * (1.0 - a * a);
  N[6] = 0.5 * (1.0 - a * a) * (1.0 + b), dxi[6] = -a * (1.0 + b), deta[6] = 0.5 * (1.0 - a * a);
  N[5] = 0.5 * (1.0 + a) * (1.0 - b * b), dxi[5] = 0.5 * (1.0 - b * b), deta[5] = -(1.0 + a) * b;
  N[7] = 0.5 * (1.0 - a) * (1.0 - b * b), dxi[7] = -0.5 * (1.0 - b * b), deta[7] = -(1.0 - a) * b;
}

}  // namespace cxg
