// Host-side geometry of the tensor-product discretisation: the 1-D FE_Q(p)
// basis on Gauss-Lobatto points, its exactly integrated reference matrices, and
// the assembled 1-D operators of one mesh axis.
//
// On an axis-parallel cell the 2-D element matrices of the reference factor
// into 1-D ones (advection.h:6-10, mass.h: M, C_e = int N e.grad N^T,
// K_e = int (e.grad N)(e.grad N^T)), and so do their assembled forms:
//
//   M   = My (x) Mx
//   C_e = ex My (x) Cx + ey Cy (x) Mx
//   K_e = ex^2 My (x) Kx + ey^2 Ky (x) Mx + ex ey (Cy (x) Cx^T + Cy^T (x) Cx)
//
// with, per axis, M = sum_cells h Mhat, C = sum_cells Chat, K = sum_cells Khat / h
// (Mhat_ab = int_0^1 l_a l_b, Chat_ab = int_0^1 l_a l_b', Khat_ab = int_0^1 l_a' l_b',
// exact with the p+1 Gauss points the reference integrates with). Periodic
// axes wrap (the last node is the image of the first).
#pragma once

#include <cstdint>
#include <vector>

namespace lbfem_gpu
{
  constexpr int MAXP = 4;

  struct Basis1D
  {
    int p = 1;
    double xi[MAXP + 1];          // Gauss-Lobatto support points on [0,1]
    double Mh[MAXP + 1][MAXP + 1]; // int l_a l_b
    double Ch[MAXP + 1][MAXP + 1]; // int l_a l_b'
    double Kh[MAXP + 1][MAXP + 1]; // int l_a' l_b'
    double d0[MAXP + 1], d1[MAXP + 1]; // l_a'(0), l_a'(1)
    double gq[MAXP + 1], gw[MAXP + 1];  // the p + 1 Gauss points and weights on [0,1]
    double gS[MAXP + 1][MAXP + 1], gD[MAXP + 1][MAXP + 1]; // [q][a] = l_a(x_q), l_a'(x_q)
    explicit Basis1D(int p);
  };

  // General quadrilaterals: the cells are bilinear images (MappingQ1) of the unit
  // square through the vertices vxy ((ncy+1) x (ncx+1) x 2, vertex (i, j) at
  // 2 (j (ncx+1) + i)). quad_geometry: per cell (cy ncx + cx) and Gauss point
  // (q2 (p+1) + q1), the inverse Jacobian row-major and JxW (5 values).
  std::vector<double> quad_geometry(const Basis1D &b, const double *vxy, int ncx, int ncy);
  // The Jacobi diagonal and the row sums (lumped diagonal) of the assembled mass
  // matrix on the structured nodes; a periodic image node gets 1 in both.
  void quad_diagonals(const Basis1D &b, const std::vector<double> &geo, int ncx, int ncy, bool px, bool py,
                      std::vector<double> &jacobi, std::vector<double> &lumped);

  // The assembled 1-D operators of one axis, as rows of 2p+1 coefficients:
  // row[m][i][k] couples node i to node i+k-p (m: 0 = M, 1 = C, 2 = C^T, 3 = K).
  struct Axis
  {
    int p = 1, n_cells = 0, n_nodes = 0, n_unique = 0;
    bool periodic = false;
    std::vector<double> vertex;
    std::vector<double> rows; // [4][n_nodes][2p+1]
    std::vector<double> diag;    // Jacobi: diagonal of M (images: 1)
    std::vector<double> lump;    // row sums of M (images: 1)
    std::vector<double> invdiag; // 1 / diag
    std::vector<double> invlump; // 1 / lump
    std::vector<double> h, hinv; // cell widths and their inverses
    double h_first = 0, h_last = 0;
  };

  Axis make_axis(const Basis1D &b, const double *vertex, int n_cells, bool periodic);

  // Banded LDL^T factors of the 1-D mass matrix M of an axis restricted to the
  // windows of a tile partition: tile t owns nodes [t T, (t+1) T) and its window
  // is [t T - W, (t+1) T + W). Window position q holds structured node
  // t T - W + q: wrapped on a periodic axis (the window then covers the
  // periodic line, unrolled), an identity row outside a non-periodic axis.
  // Because the rows of M^{-1} decay exponentially, the window solve gives
  // M^{-1} r at the own nodes to about the decay over W nodes (a few 1e-8
  // relative for W = 12, 20, 24, 28 at p = 1..4, a few 1e-6 for W = 8, 12, 16, 20).
  // Layout [tile][q][stride]: l_{q,q-k} for k = 1..p, then 1 / d_q, then zeros
  // up to stride >= p + 1 (a whole vector load per position).
  std::vector<float> window_ldl(const Axis &ax, int T, int W, int n_tiles, int stride);
} // namespace lbfem_gpu
