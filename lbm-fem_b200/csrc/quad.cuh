// General quadrilaterals (the reference's --distort, test_cases.h:52-63): FP64
// cell-based kernels for meshes whose cells are bilinear images of the unit
// square (MappingQ1). The tensor-product factorisation of the other kernels is
// gone on such a mesh, so these follow the reference's cell loop
// (advection.h:93-124, mass.h:105-144): per cell, sum-factorised reference
// gradients at the (p+1)^2 Gauss points, the inverse Jacobian and JxW stored
// per cell and point, the point operation, integration, and the scatter-add.
// The scatter is conflict-free by cell colouring (cells of one colour share no
// node), so the sums are deterministic; one thread takes one cell of one
// population. A correctness path: host-driven steps, plain CG vector kernels.
#pragma once

#include "operators.cuh"

namespace lbfem_gpu
{
  // 1-D FE_Q(p) values and derivatives at the Gauss points: [p-1][q][a] = l_a(x_q), l_a'(x_q).
  __device__ __constant__ double c_gS[MAXPD][MAXPD + 1][MAXPD + 1];
  __device__ __constant__ double c_gD[MAXPD][MAXPD + 1][MAXPD + 1];

  struct QuadGeo
  {
    const double *g;  // per cell, per Gauss point (q2 * n + q1): J^-1 row-major (4) and JxW
    int colour_x, colour_y;
    int ncx, ncy, odd_px, odd_py; // odd periodic cell counts take a third colour (the last cell)
  };

  __device__ __forceinline__ int
  cell_colour(int c, int n, int odd_periodic)
  {
    return (odd_periodic && c == n - 1) ? 2 : (c & 1);
  }

  // Storage index of the master node of structured node (i, j).
  __device__ __forceinline__ long long
  master_index(int i, int j, const Grid &g)
  {
    if (g.px && i == g.nux)
      i = 0;
    if (g.py && j == g.nuy)
      j = 0;
    return (long long)j * g.nfx + i;
  }

  // rhs_al += the cell integrals of the point operation of the advection
  // (TaylorGalerkinAdvection / LeeLinAdvection, advection.h:219-289) over the
  // cells of one colour; thread = (cell of the colour, population).
  template <int P>
  __global__ void
  k_quad_advection(const Geo geo, const QuadGeo qg, const double *__restrict__ f, const double *__restrict__ feq,
                   double *__restrict__ rhs, const AdvCoef ac)
  {
    constexpr int n = P + 1;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int ncx_c = (qg.ncx + 1) / 2 + 1, ncy_c = (qg.ncy + 1) / 2 + 1; // cells per colour and axis, at most
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int al = int(t % NM);
    const long long k = t / NM;
    const int kx = int(k % ncx_c), ky = int(k / ncx_c);
    if (ky >= ncy_c)
      return;
    // the colour's cells: colour 0/1 -> every second cell from 0/1; colour 2 -> the last cell
    const int cx = qg.colour_x == 2 ? (kx == 0 ? qg.ncx - 1 : -1) : qg.colour_x + 2 * kx;
    const int cy = qg.colour_y == 2 ? (ky == 0 ? qg.ncy - 1 : -1) : qg.colour_y + 2 * ky;
    if (cx < 0 || cy < 0 || cx >= qg.ncx || cy >= qg.ncy || cell_colour(cx, qg.ncx, qg.odd_px) != qg.colour_x ||
        cell_colour(cy, qg.ncy, qg.odd_py) != qg.colour_y)
      return;
    long long idx[n][n];
#pragma unroll
    for (int j = 0; j < n; ++j)
#pragma unroll
      for (int i = 0; i < n; ++i)
        idx[j][i] = master_index(cx * P + i, cy * P + j, g);
    const double *cg = qg.g + ((long long)cy * qg.ncx + cx) * n * n * 5;
    const double ex = ac.ex[al], ey = ac.ey[al];
    const bool two = feq != nullptr;
    double gx[2][n][n], gy[2][n][n];
    for (int s = 0; s < (two ? 2 : 1); ++s)
      {
        const double *src = (s == 0 ? f : feq) + (long long)(al + 1) * N;
        double u[n][n];
#pragma unroll
        for (int j = 0; j < n; ++j)
#pragma unroll
          for (int i = 0; i < n; ++i)
            u[j][i] = src[idx[j][i]];
        double tx[n][n], tv[n][n]; // [b][q1]
#pragma unroll
        for (int bb = 0; bb < n; ++bb)
#pragma unroll
          for (int q1 = 0; q1 < n; ++q1)
            {
              double sd = 0, sv = 0;
#pragma unroll
              for (int aa = 0; aa < n; ++aa)
                {
                  sd += c_gD[P - 1][q1][aa] * u[bb][aa];
                  sv += c_gS[P - 1][q1][aa] * u[bb][aa];
                }
              tx[bb][q1] = sd;
              tv[bb][q1] = sv;
            }
#pragma unroll
        for (int q2 = 0; q2 < n; ++q2)
#pragma unroll
          for (int q1 = 0; q1 < n; ++q1)
            {
              double sx = 0, sy = 0;
#pragma unroll
              for (int bb = 0; bb < n; ++bb)
                {
                  sx += c_gS[P - 1][q2][bb] * tx[bb][q1];
                  sy += c_gD[P - 1][q2][bb] * tv[bb][q1];
                }
              const double *Ji = cg + (q2 * n + q1) * 5; // grad = J^-T (d/dxi, d/deta)
              gx[s][q2][q1] = Ji[0] * sx + Ji[2] * sy;
              gy[s][q2][q1] = Ji[1] * sx + Ji[3] * sy;
            }
      }
    double V[n][n], FX[n][n], FY[n][n];
#pragma unroll
    for (int q2 = 0; q2 < n; ++q2)
#pragma unroll
      for (int q1 = 0; q1 < n; ++q1)
        {
          const double *Ji = cg + (q2 * n + q1) * 5;
          const double JxW = Ji[4];
          const double s = ex * gx[0][q2][q1] + ey * gy[0][q2][q1];
          double val = ac.a * s;
          if (two)
            val += ac.b * (ex * gx[1][q2][q1] + ey * gy[1][q2][q1]);
          V[q2][q1] = val * JxW;
          const double fx = (ac.c * ex) * s * JxW, fy = (ac.c * ey) * s * JxW; // flux in reference directions: J^-1 F
          FX[q2][q1] = Ji[0] * fx + Ji[1] * fy;
          FY[q2][q1] = Ji[2] * fx + Ji[3] * fy;
        }
    double A1[n][n], A2[n][n]; // [q1][b]
#pragma unroll
    for (int q1 = 0; q1 < n; ++q1)
#pragma unroll
      for (int bb = 0; bb < n; ++bb)
        {
          double s1 = 0, s2 = 0;
#pragma unroll
          for (int q2 = 0; q2 < n; ++q2)
            {
              s1 += c_gS[P - 1][q2][bb] * V[q2][q1] + c_gD[P - 1][q2][bb] * FY[q2][q1];
              s2 += c_gS[P - 1][q2][bb] * FX[q2][q1];
            }
          A1[q1][bb] = s1;
          A2[q1][bb] = s2;
        }
    double *dst = rhs + (long long)al * N;
#pragma unroll
    for (int bb = 0; bb < n; ++bb)
#pragma unroll
      for (int aa = 0; aa < n; ++aa)
        {
          double s = 0;
#pragma unroll
          for (int q1 = 0; q1 < n; ++q1)
            s += c_gS[P - 1][q1][aa] * A1[q1][bb] + c_gD[P - 1][q1][aa] * A2[q1][bb];
          dst[idx[bb][aa]] += s;
        }
  }

  // y += M x over the cells of one colour (MassOperator::local_apply, mass.h:105-144);
  // thread = (cell of the colour, system), nsys systems of stride N.
  template <int P>
  __global__ void
  k_quad_mass(const Geo geo, const QuadGeo qg, const double *__restrict__ x, double *__restrict__ y, int nsys)
  {
    constexpr int n = P + 1;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int ncx_c = (qg.ncx + 1) / 2 + 1, ncy_c = (qg.ncy + 1) / 2 + 1;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int sys = int(t % nsys);
    const long long k = t / nsys;
    const int kx = int(k % ncx_c), ky = int(k / ncx_c);
    if (ky >= ncy_c)
      return;
    const int cx = qg.colour_x == 2 ? (kx == 0 ? qg.ncx - 1 : -1) : qg.colour_x + 2 * kx;
    const int cy = qg.colour_y == 2 ? (ky == 0 ? qg.ncy - 1 : -1) : qg.colour_y + 2 * ky;
    if (cx < 0 || cy < 0 || cx >= qg.ncx || cy >= qg.ncy || cell_colour(cx, qg.ncx, qg.odd_px) != qg.colour_x ||
        cell_colour(cy, qg.ncy, qg.odd_py) != qg.colour_y)
      return;
    long long idx[n][n];
    double u[n][n];
    const double *xs = x + (long long)sys * N;
#pragma unroll
    for (int j = 0; j < n; ++j)
#pragma unroll
      for (int i = 0; i < n; ++i)
        {
          idx[j][i] = master_index(cx * P + i, cy * P + j, g);
          u[j][i] = xs[idx[j][i]];
        }
    const double *cg = qg.g + ((long long)cy * qg.ncx + cx) * n * n * 5;
    double t1[n][n]; // [b][q1]
#pragma unroll
    for (int bb = 0; bb < n; ++bb)
#pragma unroll
      for (int q1 = 0; q1 < n; ++q1)
        {
          double s = 0;
#pragma unroll
          for (int aa = 0; aa < n; ++aa)
            s += c_gS[P - 1][q1][aa] * u[bb][aa];
          t1[bb][q1] = s;
        }
    double vq[n][n]; // [q2][q1]
#pragma unroll
    for (int q2 = 0; q2 < n; ++q2)
#pragma unroll
      for (int q1 = 0; q1 < n; ++q1)
        {
          double s = 0;
#pragma unroll
          for (int bb = 0; bb < n; ++bb)
            s += c_gS[P - 1][q2][bb] * t1[bb][q1];
          vq[q2][q1] = s * cg[(q2 * n + q1) * 5 + 4];
        }
    double a1[n][n]; // [q1][b]
#pragma unroll
    for (int q1 = 0; q1 < n; ++q1)
#pragma unroll
      for (int bb = 0; bb < n; ++bb)
        {
          double s = 0;
#pragma unroll
          for (int q2 = 0; q2 < n; ++q2)
            s += c_gS[P - 1][q2][bb] * vq[q2][q1];
          a1[q1][bb] = s;
        }
    double *ys = y + (long long)sys * N;
#pragma unroll
    for (int bb = 0; bb < n; ++bb)
#pragma unroll
      for (int aa = 0; aa < n; ++aa)
        {
          double s = 0;
#pragma unroll
          for (int q1 = 0; q1 < n; ++q1)
            s += c_gS[P - 1][q1][aa] * a1[q1][bb];
          ys[idx[bb][aa]] += s;
        }
  }

  // The constrained rows of a vmult are the identity (mass.h:87-88): y = x on the periodic images.
  __global__ void
  k_quad_images(const Geo geo, const double *__restrict__ x, double *__restrict__ y, int nsys)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    LBFEM_GRID_STRIDE(idx, N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      if (is_image(i, j, g))
        for (int s = 0; s < nsys; ++s)
          y[s * N + idx] = x[s * N + idx];
    }
  }

  // The vector operations of Jacobi-PCG in deal.II SolverCG's order
  // (mass.h:204-211), one system: dot products by fixed-order partials.
  __global__ void __launch_bounds__(THREADS)
    k_quad_dot(const Geo geo, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ partials)
  {
    const Grid &g = geo.g;
    double s[1] = {0};
    LBFEM_GRID_STRIDE(idx, g.N)
    s[0] += a[idx] * b[idx];
    block_reduce_store<1>(s, partials, blockIdx.x, gridDim.x);
  }

  // mode 0: y = a x + b y; mode 1: y = x * d (element-wise)
  __global__ void
  k_quad_axpby(long long n, double a, const double *__restrict__ x, double b, double *__restrict__ y,
               const double *__restrict__ d, int mode)
  {
    LBFEM_GRID_STRIDE(i, n)
    y[i] = mode == 1 ? x[i] * d[i] : a * x[i] + b * y[i];
  }
} // namespace lbfem_gpu
