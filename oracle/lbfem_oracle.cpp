// CPU FP64 oracle of the lbm-fem hot path -- TEST INFRASTRUCTURE ONLY.
//
// The checker the CUDA path is compared against (tests/, the smoke check and
// the CPU-baseline leg of bench.py). It restates the reference's matrix-free
// algorithm without deal.II, in the reference's order of operations:
//
//   * FE_Q(p) on Gauss-Lobatto support points, QGauss(p+1) cell and face
//     quadrature, cartesian cells (diagonal Jacobian per cell): deal.II's
//     conventions behind discretization.h:114-121.
//   * Cell loop of weak_form::integrate_cells (advection.h:93-124): gather the
//     8 moving populations (periodic images read their source node, as
//     read_dof_values resolves the constraints), sum-factorised gradients at
//     the Gauss points, the point operation of TaylorGalerkinAdvection
//     (advection.h:228-239) or LeeLinAdvection (advection.h:275-287),
//     integrate values and gradients, scatter-add to the source nodes
//     (distribute_local_to_global).
//   * Wall faces, weak_form::integrate_boundary_faces + wall_surface_term
//     (advection.h:126-146,182-199).
//   * MassOperator vmult with identity rows on constrained DoFs, row-sum lumped
//     diagonal and Jacobi diagonal (discretization.h:123-125).
//   * SolverCG with the Jacobi preconditioner in deal.II's order of updates,
//     absolute tolerance cg_tolerance * |r| (mass.h:204-211).
//   * nodal_map semantics of collision.h:78-102 (wall nodes with the wall
//     velocity imposed on their moments), collide_bgk, compute_equilibrium,
//     predictor_corrector (collision.h:105-168).
//   * TaylorGalerkin::increment / stream with the extrapolated CG start
//     2 x^n - x^{n-1} (streaming.h:66-100) and the two schemes
//     (schemes.h:92-98,118-141); TG3 (A = M + dt^2/6 K_e, StreamingMatrix,
//     mass.h:57-129) and its x / y split sweeps (streaming.h:41-60,102-121).
//
// Cells are processed in four colours (no two cells of a colour share a node)
// so that the OpenMP scatter-add is race-free; dot products use a fixed chunking
// so that every result is independent of the thread count.
#include "lbfem_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#ifdef _OPENMP
#  include <omp.h>
#endif

namespace
{
  constexpr int Q = 9;
  constexpr int NM = 8; // moving populations
  constexpr int MAXP = 4;
  constexpr int MAXN = MAXP + 1;

  // d2q9.h:18-22
  constexpr double EX[Q] = {0, 1, 1, 0, -1, -1, -1, 0, 1};
  constexpr double EY[Q] = {0, 0, 1, 1, 1, 0, -1, -1, -1};
  constexpr double W[Q] = {4. / 9., 1. / 9., 1. / 36., 1. / 9., 1. / 36., 1. / 9., 1. / 36., 1. / 9., 1. / 36.};

  struct Moments
  {
    double rho, ux, uy;
  };

  // D2Q9::moments, d2q9.h:30-41
  inline Moments
  moments(const double *f)
  {
    double rho = 0, mx = 0, my = 0;
    for (int a = 0; a < Q; ++a)
      {
        rho += f[a];
        mx += EX[a] * f[a];
        my += EY[a] * f[a];
      }
    return {rho, mx / rho, my / rho};
  }

  // D2Q9::equilibrium, d2q9.h:44-55
  inline void
  equilibrium(const Moments &m, double *feq)
  {
    const double uu = m.ux * m.ux + m.uy * m.uy;
    for (int a = 0; a < Q; ++a)
      {
        const double eu = EX[a] * m.ux + EY[a] * m.uy;
        feq[a] = W[a] * m.rho * (1. + 3. * eu + 4.5 * eu * eu - 1.5 * uu);
      }
  }

  // ---------------------------------------------------------------- 1-D basis
  long double
  legendre(int n, long double t, long double *dp)
  {
    long double p0 = 1, p1 = t;
    if (n == 0)
      {
        *dp = 0;
        return 1;
      }
    for (int k = 1; k < n; ++k)
      {
        const long double p2 = ((2 * k + 1) * t * p1 - k * p0) / (k + 1);
        p0 = p1;
        p1 = p2;
      }
    *dp = n * (t * p1 - p0) / (t * t - 1);
    return p1;
  }

  struct Basis
  {
    int p = 1;
    double xi[MAXN];            // Gauss-Lobatto support points on [0,1]
    double qx[MAXN], qw[MAXN];  // Gauss points and weights on [0,1]
    double S[MAXN][MAXN];       // S[q][a] = l_a(q)
    double D[MAXN][MAXN];       // D[q][a] = l_a'(q)
    double D0[MAXN], D1[MAXN];  // l_a'(0), l_a'(1)

    explicit Basis(int p_)
      : p(p_)
    {
      const int n = p + 1;
      const long double pi = 3.141592653589793238462643383279502884L;
      // Gauss-Legendre: roots of P_{p+1}
      for (int k = 0; k < n; ++k)
        {
          long double t = -std::cos(pi * (k + 0.75L) / (n + 0.5L));
          for (int it = 0; it < 100; ++it)
            {
              long double dp;
              const long double v = legendre(n, t, &dp);
              const long double dt = v / dp;
              t -= dt;
              if (std::fabs(dt) < 1e-19L)
                break;
            }
          long double dp;
          legendre(n, t, &dp);
          qx[k] = double((t + 1) / 2);
          qw[k] = double(1 / ((1 - t * t) * dp * dp)); // 2/((1-t^2)P'^2) / 2
        }
      // Gauss-Lobatto: endpoints and roots of P_p'
      xi[0] = 0.;
      xi[p] = 1.;
      for (int k = 1; k < p; ++k)
        {
          long double t = -std::cos(pi * k / p);
          for (int it = 0; it < 100; ++it)
            {
              long double dp;
              const long double v = legendre(p, t, &dp);
              const long double d2 = (2 * t * dp - p * (p + 1) * v) / (1 - t * t);
              const long double dt = dp / d2;
              t -= dt;
              if (std::fabs(dt) < 1e-19L)
                break;
            }
          xi[k] = double((t + 1) / 2);
        }
      for (int q = 0; q < n; ++q)
        for (int a = 0; a < n; ++a)
          {
            S[q][a] = lagrange(a, qx[q]);
            D[q][a] = dlagrange(a, qx[q]);
          }
      for (int a = 0; a < n; ++a)
        {
          D0[a] = dlagrange(a, 0.);
          D1[a] = dlagrange(a, 1.);
        }
    }

    double
    lagrange(int a, double x) const
    {
      long double v = 1;
      for (int b = 0; b <= p; ++b)
        if (b != a)
          v *= ((long double)x - xi[b]) / ((long double)xi[a] - xi[b]);
      return double(v);
    }

    double
    dlagrange(int a, double x) const
    {
      long double sum = 0;
      for (int c = 0; c <= p; ++c)
        {
          if (c == a)
            continue;
          long double v = 1 / ((long double)xi[a] - xi[c]);
          for (int b = 0; b <= p; ++b)
            if (b != a && b != c)
              v *= ((long double)x - xi[b]) / ((long double)xi[a] - xi[b]);
          sum += v;
        }
      return double(sum);
    }
  };

  // ------------------------------------------------------------------ oracle
  struct WallU
  {
    bool wall = false;
    double ux = 0, uy = 0;
  };

} // namespace

struct lbfem_oracle
{
  int p = 1, ncx = 0, ncy = 0, px = 0, py = 0, nfx = 0, nfy = 0;
  int64_t N = 0;
  std::vector<double> vx, vy;
  std::unique_ptr<Basis> basis;
  std::vector<WallU> wall;         // per node
  std::vector<int64_t> wall_nodes; // nodes with a wall velocity
  std::vector<uint8_t> constrained; // periodic images
  std::vector<double> lumped, inv_lumped, jacobi, inv_jacobi;
  lbfem_params prm{};
  double dt = 0, lambda = 0;
  bool have_ts = false;
  std::vector<double> f, feq, rhs, x0, x1, cg_r, cg_p, cg_v, cg_z;
  int64_t cg_its = 0;
  // one y-strip of a decomposed mesh (lbfem_oracle_set_strip): owned node rows
  // [oy0, oy1), the rest ghost copies of the neighbours' rows
  bool strip = false;
  int oy0 = 0, oy1 = 0;
  lbfem_strip_desc sd{};
  // general quadrilaterals (lbfem_mesh_desc::vertex_xy): the mapped vertices, (ncy+1) x (ncx+1) x 2
  bool distorted = false;
  std::vector<double> vxy;

  int64_t
  master(int i, int j) const
  {
    if (px && i == p * ncx)
      i = 0;
    if (py && j == p * ncy)
      j = 0;
    return int64_t(j) * nfx + i;
  }
};

namespace
{
  int
  colour_of(int c, int n, bool periodic)
  {
    if (periodic && (n % 2 == 1) && c == n - 1)
      return 2;
    return c % 2;
  }

  template <typename F>
  void
  for_cells_coloured(const lbfem_oracle &o, F &&body)
  {
    for (int colour_y = 0; colour_y < 3; ++colour_y)
      for (int colour_x = 0; colour_x < 3; ++colour_x)
        {
          std::vector<std::pair<int, int>> cells;
          for (int cy = 0; cy < o.ncy; ++cy)
            if (colour_of(cy, o.ncy, o.py) == colour_y)
              for (int cx = 0; cx < o.ncx; ++cx)
                if (colour_of(cx, o.ncx, o.px) == colour_x)
                  cells.push_back({cx, cy});
          const int64_t n = cells.size();
#pragma omp parallel for schedule(static)
          for (int64_t k = 0; k < n; ++k)
            body(cells[k].first, cells[k].second);
        }
  }

  // Fixed-chunk deterministic dot product.
  double
  dot(const double *a, const double *b, int64_t n)
  {
    constexpr int64_t CH = 4096;
    const int64_t nch = (n + CH - 1) / CH;
    std::vector<double> part(nch, 0.);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nch; ++c)
      {
        double s = 0;
        const int64_t e = std::min(n, (c + 1) * CH);
        for (int64_t i = c * CH; i < e; ++i)
          s += a[i] * b[i];
        part[c] = s;
      }
    double s = 0;
    for (double v : part)
      s += v;
    return s;
  }

  // The dot product of the solvers: over the owned rows, summed over the ranks
  // of a strip decomposition (the MPI sum of deal.II's distributed vectors).
  int
  strip_dot(const lbfem_oracle &o, const double *a, const double *b, double *out)
  {
    if (!o.strip)
      {
        *out = dot(a, b, o.N);
        return LBFEM_OK;
      }
    const int64_t off = int64_t(o.oy0) * o.nfx;
    o.sd.sums[0] = dot(a + off, b + off, int64_t(o.oy1 - o.oy0) * o.nfx);
    if (o.sd.comm(o.sd.user, LBFEM_COMM_ALLREDUCE, 1) != 0)
      return LBFEM_ERR_ARG;
    *out = o.sd.sums[0];
    return LBFEM_OK;
  }

  // The ghost rows of one vector of N values <- the neighbours' owned rows
  // (1 row down and `degree` rows up out of the owned rows).
  int
  strip_exchange(const lbfem_oracle &o, double *v)
  {
    if (!o.strip)
      return LBFEM_OK;
    const int64_t row = o.nfx;
    const int P = o.p;
    double *sb = static_cast<double *>(o.sd.send_below), *sa = static_cast<double *>(o.sd.send_above);
    double *rb = static_cast<double *>(o.sd.recv_below), *ra = static_cast<double *>(o.sd.recv_above);
    if (o.sd.ghost_below)
      std::copy(v + o.oy0 * row, v + (o.oy0 + 1) * row, sb);
    if (o.sd.ghost_above)
      std::copy(v + (o.oy1 - P) * row, v + o.oy1 * row, sa);
    if (o.sd.comm(o.sd.user, LBFEM_COMM_EXCHANGE, row * int64_t(sizeof(double))) != 0)
      return LBFEM_ERR_ARG;
    if (o.sd.ghost_below)
      std::copy(rb, rb + P * row, v + (o.oy0 - P) * row);
    if (o.sd.ghost_above)
      std::copy(ra, ra + row, v + o.oy1 * row);
    return LBFEM_OK;
  }

  // MappingQ1 of cell (cx, cy) at the reference point (s, t): the inverse
  // Jacobian, row-major (Ji[0] = (J^-1)_00, Ji[1] = (J^-1)_01, ...), and det J.
  double
  cell_map(const lbfem_oracle &o, int cx, int cy, double s, double t, double (&Ji)[4])
  {
    auto v = [&](int i, int j, int k) { return o.vxy[(size_t(j) * (o.ncx + 1) + i) * 2 + k]; };
    double J[2][2];
    for (int k = 0; k < 2; ++k)
      {
        J[k][0] = (1 - t) * (v(cx + 1, cy, k) - v(cx, cy, k)) + t * (v(cx + 1, cy + 1, k) - v(cx, cy + 1, k));
        J[k][1] = (1 - s) * (v(cx, cy + 1, k) - v(cx, cy, k)) + s * (v(cx + 1, cy + 1, k) - v(cx + 1, cy, k));
      }
    const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    Ji[0] = J[1][1] / det;
    Ji[1] = -J[0][1] / det;
    Ji[2] = -J[1][0] / det;
    Ji[3] = J[0][0] / det;
    return det;
  }

  // ------------------------------------------------------- advection (K1)
  // rhs (8 blocks) <- cell integrals of the point operation over f (and feq)
  // + wall-face integrals of the surface term.
  template <int P>
  void
  advection_impl(const lbfem_oracle &o, const double *f, const double *feq, const double *e, double a, double b,
                 double c, double dt, bool remove_flux, double *rhs)
  {
    constexpr int n = P + 1;
    const Basis &B = *o.basis;
    const int64_t N = o.N;
    std::fill(rhs, rhs + NM * N, 0.);
    const bool two = feq != nullptr;
    double ex[NM], ey[NM];
    for (int al = 0; al < NM; ++al)
      {
        ex[al] = e[2 * (al + 1)];
        ey[al] = e[2 * (al + 1) + 1];
      }

    for_cells_coloured(o, [&](int cx, int cy) {
      const double hx = o.vx[cx + 1] - o.vx[cx], hy = o.vy[cy + 1] - o.vy[cy];
      int64_t idx[n][n];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          idx[j][i] = o.master(cx * P + i, cy * P + j);
      double jinv[n][n][4], jxw[n][n]; // general quadrilaterals: MappingQ1 at the Gauss points
      if (o.distorted)
        for (int q2 = 0; q2 < n; ++q2)
          for (int q1 = 0; q1 < n; ++q1)
            jxw[q2][q1] = B.qw[q1] * B.qw[q2] * cell_map(o, cx, cy, B.qx[q1], B.qx[q2], jinv[q2][q1]);
      double V[NM][n][n], FX[NM][n][n], FY[NM][n][n]; // at Gauss points [q2][q1]
      for (int al = 0; al < NM; ++al)
        {
          double gxf[n][n], gyf[n][n], gxe[n][n], gye[n][n];
          for (int s = 0; s < (two ? 2 : 1); ++s)
            {
              const double *src = (s == 0 ? f : feq) + int64_t(al + 1) * N;
              double u[n][n];
              for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                  u[j][i] = src[idx[j][i]];
              double tx[n][n], tv[n][n]; // [b][q1]
              for (int bb = 0; bb < n; ++bb)
                for (int q1 = 0; q1 < n; ++q1)
                  {
                    double sd = 0, sv = 0;
                    for (int aa = 0; aa < n; ++aa)
                      {
                        sd += B.D[q1][aa] * u[bb][aa];
                        sv += B.S[q1][aa] * u[bb][aa];
                      }
                    tx[bb][q1] = sd;
                    tv[bb][q1] = sv;
                  }
              double(*gx)[n] = s == 0 ? gxf : gxe;
              double(*gy)[n] = s == 0 ? gyf : gye;
              for (int q2 = 0; q2 < n; ++q2)
                for (int q1 = 0; q1 < n; ++q1)
                  {
                    double sx = 0, sy = 0;
                    for (int bb = 0; bb < n; ++bb)
                      {
                        sx += B.S[q2][bb] * tx[bb][q1];
                        sy += B.D[q2][bb] * tv[bb][q1];
                      }
                    if (o.distorted)
                      {
                        // grad = J^-T (d/dxi, d/deta)
                        const double *Ji = jinv[q2][q1];
                        gx[q2][q1] = Ji[0] * sx + Ji[2] * sy;
                        gy[q2][q1] = Ji[1] * sx + Ji[3] * sy;
                      }
                    else
                      {
                        gx[q2][q1] = sx / hx;
                        gy[q2][q1] = sy / hy;
                      }
                  }
            }
          for (int q2 = 0; q2 < n; ++q2)
            for (int q1 = 0; q1 < n; ++q1)
              {
                const double JxW = o.distorted ? jxw[q2][q1] : B.qw[q1] * B.qw[q2] * hx * hy;
                const double s = ex[al] * gxf[q2][q1] + ey[al] * gyf[q2][q1];
                double val = a * s;
                if (two)
                  val += b * (ex[al] * gxe[q2][q1] + ey[al] * gye[q2][q1]);
                V[al][q2][q1] = val * JxW;
                if (o.distorted)
                  {
                    // the flux in reference directions: J^-1 F
                    const double *Ji = jinv[q2][q1];
                    const double fx = (c * ex[al]) * s * JxW, fy = (c * ey[al]) * s * JxW;
                    FX[al][q2][q1] = Ji[0] * fx + Ji[1] * fy;
                    FY[al][q2][q1] = Ji[2] * fx + Ji[3] * fy;
                  }
                else
                  {
                    FX[al][q2][q1] = (c * ex[al]) * s * JxW / hx;
                    FY[al][q2][q1] = (c * ey[al]) * s * JxW / hy;
                  }
              }
        }
      for (int al = 0; al < NM; ++al)
        {
          double A1[n][n], A2[n][n]; // [q1][b]
          for (int q1 = 0; q1 < n; ++q1)
            for (int bb = 0; bb < n; ++bb)
              {
                double s1 = 0, s2 = 0;
                for (int q2 = 0; q2 < n; ++q2)
                  {
                    s1 += B.S[q2][bb] * V[al][q2][q1] + B.D[q2][bb] * FY[al][q2][q1];
                    s2 += B.S[q2][bb] * FX[al][q2][q1];
                  }
                A1[q1][bb] = s1;
                A2[q1][bb] = s2;
              }
          double *dst = rhs + int64_t(al) * N;
          for (int bb = 0; bb < n; ++bb)
            for (int aa = 0; aa < n; ++aa)
              {
                double s = 0;
                for (int q1 = 0; q1 < n; ++q1)
                  s += B.S[q1][aa] * A1[q1][bb] + B.D[q1][aa] * A2[q1][bb];
                dst[idx[bb][aa]] += s;
              }
        }
    });

    // Wall faces (all non-periodic sides of the box), serial: O(sqrt N).
    const double half_dt2 = 0.5 * dt * dt;
    auto face = [&](int cx, int cy, int side) {
      // side: 0 bottom (y=0), 1 top (y=L), 2 left (x=0), 3 right (x=L)
      const double hx = o.vx[cx + 1] - o.vx[cx], hy = o.vy[cy + 1] - o.vy[cy];
      int64_t idx[n][n];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          idx[j][i] = o.master(cx * P + i, cy * P + j);
      const double nx = side == 2 ? -1. : side == 3 ? 1. : 0.;
      const double ny = side == 0 ? -1. : side == 1 ? 1. : 0.;
      const bool horizontal = side < 2; // face along x
      const double hface = horizontal ? hx : hy;
      double val[NM][n];
      for (int al = 0; al < NM; ++al)
        {
          const double *src = f + int64_t(al + 1) * N;
          double u[n][n];
          for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
              u[j][i] = src[idx[j][i]];
          for (int q = 0; q < n; ++q)
            {
              double gx = 0, gy = 0;
              if (horizontal)
                {
                  const int jb = side == 0 ? 0 : P;
                  const double *dn = side == 0 ? B.D0 : B.D1;
                  for (int aa = 0; aa < n; ++aa)
                    {
                      gx += B.D[q][aa] * u[jb][aa];
                      double t = 0;
                      for (int bb = 0; bb < n; ++bb)
                        t += dn[bb] * u[bb][aa];
                      gy += B.S[q][aa] * t;
                    }
                }
              else
                {
                  const int ib = side == 2 ? 0 : P;
                  const double *dn = side == 2 ? B.D0 : B.D1;
                  for (int bb = 0; bb < n; ++bb)
                    {
                      gy += B.D[q][bb] * u[bb][ib];
                      double t = 0;
                      for (int aa = 0; aa < n; ++aa)
                        t += dn[aa] * u[bb][aa];
                      gx += B.S[q][bb] * t;
                    }
                }
              gx /= hx;
              gy /= hy;
              val[al][q] = half_dt2 * (ex[al] * nx + ey[al] * ny) * (ex[al] * gx + ey[al] * gy);
            }
        }
      if (remove_flux)
        for (int q = 0; q < n; ++q)
          {
            double flux = 0;
            for (int al = 0; al < NM; ++al)
              flux += val[al][q];
            for (int al = 0; al < NM; ++al)
              val[al][q] -= (W[al + 1] / (1. - W[0])) * flux;
          }
      for (int al = 0; al < NM; ++al)
        {
          double *dst = rhs + int64_t(al) * N;
          for (int k = 0; k < n; ++k)
            {
              double s = 0;
              for (int q = 0; q < n; ++q)
                s += B.S[q][k] * (val[al][q] * (B.qw[q] * hface));
              if (horizontal)
                dst[idx[side == 0 ? 0 : P][k]] += s;
              else
                dst[idx[k][side == 2 ? 0 : P]] += s;
            }
        }
    };
    if (!o.py)
      for (int cx = 0; cx < o.ncx; ++cx)
        {
          face(cx, 0, 0);
          face(cx, o.ncy - 1, 1);
        }
    if (!o.px)
      for (int cy = 0; cy < o.ncy; ++cy)
        {
          face(0, cy, 2);
          face(o.ncx - 1, cy, 3);
        }
  }

  void
  advection(const lbfem_oracle &o, const double *f, const double *feq, const double *e, double a, double b, double c,
            double dt, bool remove_flux, double *rhs)
  {
    switch (o.p)
      {
        case 1:
          advection_impl<1>(o, f, feq, e, a, b, c, dt, remove_flux, rhs);
          break;
        case 2:
          advection_impl<2>(o, f, feq, e, a, b, c, dt, remove_flux, rhs);
          break;
        case 3:
          advection_impl<3>(o, f, feq, e, a, b, c, dt, remove_flux, rhs);
          break;
        default:
          advection_impl<4>(o, f, feq, e, a, b, c, dt, remove_flux, rhs);
      }
  }

  // ----------------------------------------------------------- mass matrix
  // dst = M src over the cells (no constraint rows); mode 0: the action,
  // mode 1: the diagonal of the cell matrices (src unused).
  template <int P>
  void
  mass_cells(const lbfem_oracle &o, const double *src, double *dst, int mode)
  {
    constexpr int n = P + 1;
    const Basis &B = *o.basis;
    std::fill(dst, dst + o.N, 0.);
    for_cells_coloured(o, [&](int cx, int cy) {
      const double hx = o.vx[cx + 1] - o.vx[cx], hy = o.vy[cy + 1] - o.vy[cy];
      int64_t idx[n][n];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          idx[j][i] = o.master(cx * P + i, cy * P + j);
      auto jxw_at = [&](int q1, int q2) {
        if (!o.distorted)
          return B.qw[q1] * B.qw[q2] * hx * hy;
        double Ji[4];
        return B.qw[q1] * B.qw[q2] * cell_map(o, cx, cy, B.qx[q1], B.qx[q2], Ji);
      };
      if (mode == 1)
        {
          for (int bb = 0; bb < n; ++bb)
            for (int aa = 0; aa < n; ++aa)
              {
                double s = 0;
                for (int q2 = 0; q2 < n; ++q2)
                  for (int q1 = 0; q1 < n; ++q1)
                    {
                      const double phi = B.S[q1][aa] * B.S[q2][bb];
                      s += phi * phi * jxw_at(q1, q2);
                    }
                dst[idx[bb][aa]] += s;
              }
          return;
        }
      double u[n][n];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          u[j][i] = src[idx[j][i]];
      double t[n][n]; // [b][q1]
      for (int bb = 0; bb < n; ++bb)
        for (int q1 = 0; q1 < n; ++q1)
          {
            double s = 0;
            for (int aa = 0; aa < n; ++aa)
              s += B.S[q1][aa] * u[bb][aa];
            t[bb][q1] = s;
          }
      double vq[n][n]; // [q2][q1]
      for (int q2 = 0; q2 < n; ++q2)
        for (int q1 = 0; q1 < n; ++q1)
          {
            double s = 0;
            for (int bb = 0; bb < n; ++bb)
              s += B.S[q2][bb] * t[bb][q1];
            vq[q2][q1] = s * jxw_at(q1, q2);
          }
      double a1[n][n]; // [q1][b]
      for (int q1 = 0; q1 < n; ++q1)
        for (int bb = 0; bb < n; ++bb)
          {
            double s = 0;
            for (int q2 = 0; q2 < n; ++q2)
              s += B.S[q2][bb] * vq[q2][q1];
            a1[q1][bb] = s;
          }
      for (int bb = 0; bb < n; ++bb)
        for (int aa = 0; aa < n; ++aa)
          {
            double s = 0;
            for (int q1 = 0; q1 < n; ++q1)
              s += B.S[q1][aa] * a1[q1][bb];
            dst[idx[bb][aa]] += s;
          }
    });
  }

  void
  mass_cells_dispatch(const lbfem_oracle &o, const double *src, double *dst, int mode)
  {
    switch (o.p)
      {
        case 1:
          mass_cells<1>(o, src, dst, mode);
          break;
        case 2:
          mass_cells<2>(o, src, dst, mode);
          break;
        case 3:
          mass_cells<3>(o, src, dst, mode);
          break;
        default:
          mass_cells<4>(o, src, dst, mode);
      }
  }

  // MassOperator vmult: cell loop, then the identity on constrained rows.
  void
  mass_vmult(const lbfem_oracle &o, double *dst, const double *src)
  {
    mass_cells_dispatch(o, src, dst, 0);
    for (int64_t i = 0; i < o.N; ++i)
      if (o.constrained[i])
        dst[i] = src[i];
  }

  // dst = (M + c K_e) src over the cells, K_e = int (e.grad N)(e.grad N^T):
  // StreamingMatrix::cell_integral (mass.h:107-129) with coef != 0 -- value
  // submitted as is, gradient flux c e (e.grad u). Evaluated point by point
  // (no sum factorisation): the oracle runs it on small meshes only.
  template <int P>
  void
  streaming_cells(const lbfem_oracle &o, const double *src, double *dst, double ex, double ey, double c)
  {
    constexpr int n = P + 1;
    const Basis &B = *o.basis;
    std::fill(dst, dst + o.N, 0.);
    for_cells_coloured(o, [&](int cx, int cy) {
      const double hx = o.vx[cx + 1] - o.vx[cx], hy = o.vy[cy + 1] - o.vy[cy];
      int64_t idx[n][n];
      double u[n][n];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          {
            idx[j][i] = o.master(cx * P + i, cy * P + j);
            u[j][i] = src[idx[j][i]];
          }
      double out[n][n] = {};
      for (int q2 = 0; q2 < n; ++q2)
        for (int q1 = 0; q1 < n; ++q1)
          {
            double v = 0, gx = 0, gy = 0;
            for (int bb = 0; bb < n; ++bb)
              for (int aa = 0; aa < n; ++aa)
                {
                  v += B.S[q2][bb] * B.S[q1][aa] * u[bb][aa];
                  gx += B.S[q2][bb] * B.D[q1][aa] * u[bb][aa];
                  gy += B.D[q2][bb] * B.S[q1][aa] * u[bb][aa];
                }
            gx /= hx;
            gy /= hy;
            const double JxW = B.qw[q1] * B.qw[q2] * hx * hy;
            const double eg = ex * gx + ey * gy;
            const double sv = v * JxW, fx = (c * ex) * eg * JxW, fy = (c * ey) * eg * JxW;
            for (int bb = 0; bb < n; ++bb)
              for (int aa = 0; aa < n; ++aa)
                out[bb][aa] += B.S[q2][bb] * B.S[q1][aa] * sv + B.S[q2][bb] * (B.D[q1][aa] / hx) * fx +
                               (B.D[q2][bb] / hy) * B.S[q1][aa] * fy;
          }
      for (int bb = 0; bb < n; ++bb)
        for (int aa = 0; aa < n; ++aa)
          dst[idx[bb][aa]] += out[bb][aa];
    });
  }

  // The matrix of the streaming step, A = M + c K_e (MassSolver::with_matrix,
  // mass.h:219-231): the mass operator for c = 0; constrained rows identity.
  struct StreamOp
  {
    double ex = 0, ey = 0, c = 0;
  };

  void
  op_vmult(const lbfem_oracle &o, const StreamOp &A, double *dst, const double *src)
  {
    if (A.c == 0.)
      {
        mass_vmult(o, dst, src);
        return;
      }
    switch (o.p)
      {
        case 1:
          streaming_cells<1>(o, src, dst, A.ex, A.ey, A.c);
          break;
        case 2:
          streaming_cells<2>(o, src, dst, A.ex, A.ey, A.c);
          break;
        case 3:
          streaming_cells<3>(o, src, dst, A.ex, A.ey, A.c);
          break;
        default:
          streaming_cells<4>(o, src, dst, A.ex, A.ey, A.c);
      }
    for (int64_t i = 0; i < o.N; ++i)
      if (o.constrained[i])
        dst[i] = src[i];
  }

  // deal.II SolverCG with the Jacobi preconditioner, in its order of updates.
  int
  cg_solve(lbfem_oracle &o, const StreamOp &A, double *x, const double *b, int64_t *its)
  {
    const int64_t N = o.N;
    double *r = o.cg_r.data(), *p = o.cg_p.data(), *v = o.cg_v.data(), *z = o.cg_z.data();
    double bb = 0;
    int sst;
    if ((sst = strip_dot(o, b, b, &bb)))
      return sst;
    const double tol = o.prm.cg_tolerance * std::sqrt(bb);
    *its = 0;
    if (bb == 0.)
      {
        // an exactly zero right-hand side: the solution 0. deal.II's SolverCG would
        // iterate from a nonzero (extrapolated) start toward the tolerance 0 and
        // throw NoConvergence at the cap (the x-axis populations of the start-up
        // Couette flow on 32 x 256 cells meet this after a few steps).
        std::fill(x, x + N, 0.);
        return LBFEM_OK;
      }
    bool zero = true;
    for (int64_t i = 0; i < N && zero; ++i)
      zero = x[i] == 0.;
    if (!zero)
      {
        op_vmult(o, A, r, x);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
          r[i] = -r[i] + b[i];
      }
    else
      std::copy(b, b + N, r);
    double res = 0;
    if ((sst = strip_exchange(o, r)) || (sst = strip_dot(o, r, r, &res)))
      return sst;
    res = std::sqrt(res);
    int64_t it = 0;
    *its = 0;
    if (std::isnan(res))
      return LBFEM_ERR_NONFINITE;
    if (res <= tol)
      return LBFEM_OK;
    double rz = 0;
    while (true)
      {
        ++it;
        const double *inv = o.inv_jacobi.data();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
          z[i] = inv[i] * r[i];
        const double rz_prev = rz;
        if ((sst = strip_dot(o, r, z, &rz)))
          return sst;
        const double beta = it > 1 ? rz / rz_prev : 0.;
        if (it > 1)
          {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i)
              p[i] = beta * p[i] + z[i];
          }
        else
          std::copy(z, z + N, p);
        op_vmult(o, A, v, p);
        double pAp = 0;
        if ((sst = strip_dot(o, p, v, &pAp)))
          return sst;
        const double alpha = rz / pAp;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
          {
            x[i] += alpha * p[i];
            r[i] += -alpha * v[i];
          }
        if ((sst = strip_exchange(o, r)) || (sst = strip_dot(o, r, r, &res)))
          return sst;
        res = std::sqrt(res);
        *its = it;
        if (std::isnan(res))
          return LBFEM_ERR_NONFINITE;
        if (res <= tol)
          return LBFEM_OK;
        if (it >= o.prm.cg_max_iterations)
          return LBFEM_ERR_NO_CONVERGENCE;
      }
  }

  int
  mass_solve(lbfem_oracle &o, double *x, const double *r, const StreamOp &A = {})
  {
    if (o.prm.mass == LBFEM_MASS_LUMPED)
      {
        const double *inv = o.inv_lumped.data();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < o.N; ++i)
          x[i] = inv[i] * r[i];
        return strip_exchange(o, x);
      }
    if (o.prm.mass == LBFEM_MASS_RICHARDSON)
      {
        // x_0 = M_L^{-1} r, x_{j+1} = x_j + M_L^{-1} (r - M x_j) (mass.h:193-202)
        const double *inv = o.inv_lumped.data();
        for (int64_t i = 0; i < o.N; ++i)
          x[i] = inv[i] * r[i];
        int sst = strip_exchange(o, x);
        for (int k = 0; k < o.prm.richardson && !sst; ++k)
          {
            op_vmult(o, A, o.cg_v.data(), x);
            for (int64_t i = 0; i < o.N; ++i)
              x[i] += inv[i] * (r[i] - o.cg_v[i]);
            sst = strip_exchange(o, x);
          }
        return sst;
      }
    int64_t its = 0;
    const int st = cg_solve(o, A, x, r, &its);
    o.cg_its += its;
    return st;
  }

  // ---------------------------------------------------------- nodal maps
  template <typename Op>
  void
  nodal_map(const lbfem_oracle &o, Op &&op)
  {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < o.N; ++i)
      op(i, o.wall[i]);
  }

  inline Moments
  impose(Moments m, const WallU &w)
  {
    if (w.wall)
      {
        m.ux = w.ux;
        m.uy = w.uy;
      }
    return m;
  }

  void
  collide_bgk(const lbfem_oracle &o, double *g, double omega)
  {
    const int64_t N = o.N;
    nodal_map(o, [&](int64_t i, const WallU &w) {
      double gi[Q], geq[Q], geqt[Q];
      for (int a = 0; a < Q; ++a)
        gi[a] = g[a * N + i];
      const Moments m = moments(gi);
      equilibrium(m, geq);
      equilibrium(impose(m, w), geqt);
      for (int a = 0; a < Q; ++a)
        g[a * N + i] = geqt[a] + (1. - omega) * (gi[a] - geq[a]);
    });
  }

  void
  compute_equilibrium(const lbfem_oracle &o, const double *f, double *feq)
  {
    const int64_t N = o.N;
    nodal_map(o, [&](int64_t i, const WallU &w) {
      double fi[Q], fe[Q];
      for (int a = 0; a < Q; ++a)
        fi[a] = f[a * N + i];
      equilibrium(impose(moments(fi), w), fe);
      for (int a = 0; a < Q; ++a)
        feq[a * N + i] = fe[a];
    });
  }

  void
  predictor_corrector(const lbfem_oracle &o, double *f, const double *feq, const double *x, double theta)
  {
    const int64_t N = o.N;
    const double inv = 1. / (1. + theta);
    nodal_map(o, [&](int64_t i, const WallU &w) {
      double fh[Q], eqh[Q];
      fh[0] = inv * (f[i] + theta * feq[i]);
      for (int a = 1; a < Q; ++a)
        fh[a] = inv * (f[a * N + i] + theta * feq[a * N + i] + x[(a - 1) * N + i]);
      equilibrium(impose(moments(fh), w), eqh);
      for (int a = 0; a < Q; ++a)
        f[a * N + i] = fh[a] + theta * (eqh[a] - feq[a * N + i]);
    });
  }

  // The directions of the populations in sweep s of the step: D2Q9::e, or
  // for the split TG3 sweeps D2Q9::e with the other component zeroed
  // (TaylorGalerkin::axis, streaming.h:107-115).
  void
  sweep_directions(const lbfem_oracle &o, int s, double *e)
  {
    const bool split = o.prm.streaming == LBFEM_STREAMING_TG3_SPLIT;
    for (int k = 0; k < Q; ++k)
      {
        e[2 * k] = split && s == 1 ? 0. : EX[k];
        e[2 * k + 1] = split && s == 0 ? 0. : EY[k];
      }
  }

  // TaylorGalerkin::increment (streaming.h:66-85): the right-hand side along
  // the directions of sweep s, then x_a <- A^{-1} r_a for the populations that
  // move in the sweep, A = M + tg3 dt^2 K_e(e_a). The CG start is the
  // extrapolation 2 x^n - x^{n-1} (x0 and x1) unless the step is split, where
  // each sweep starts from its own previous increment (x0: sweep 0, x1: sweep 1).
  int
  increment(lbfem_oracle &o, int s, const double *f, const double *feq, double a, double b, double c,
            bool remove_flux)
  {
    double e[2 * Q];
    sweep_directions(o, s, e);
    advection(o, f, feq, e, a, b, c, o.dt, remove_flux, o.rhs.data());
    const bool split = o.prm.streaming == LBFEM_STREAMING_TG3_SPLIT;
    const bool extrapolate = o.prm.mass == LBFEM_MASS_CG && !split;
    const double tg3 = o.prm.streaming == LBFEM_STREAMING_TG2 ? 0. : 1. / 6.;
    const int64_t N = o.N;
    for (int al = 0; al < NM; ++al)
      {
        const double ex = e[2 * (al + 1)], ey = e[2 * (al + 1) + 1];
        if (ex == 0. && ey == 0.)
          continue;
        double *xa = (s == 0 ? o.x0.data() : o.x1.data()) + al * N, *xb = o.x1.data() + al * N;
        if (extrapolate)
          {
            // x[1].block(a).sadd(-1., 2., xa); xa.swap(x[1].block(a)) (streaming.h:76-80)
            for (int64_t i = 0; i < N; ++i)
              xb[i] = -xb[i] + 2. * xa[i];
            std::swap_ranges(xa, xa + N, xb);
          }
        const int st = mass_solve(o, xa, o.rhs.data() + al * N, StreamOp{ex, ey, tg3 * o.dt * o.dt});
        if (st != LBFEM_OK)
          return st;
      }
    return LBFEM_OK;
  }

  int
  step(lbfem_oracle &o)
  {
    const int64_t N = o.N;
    const bool bardow = o.prm.scheme == LBFEM_SCHEME_BARDOW;
    const int rm = o.prm.remove_wall_mass_flux;
    if (bardow)
      {
        // Bardow::step, schemes.h:118-124, and TaylorGalerkin::stream,
        // streaming.h:88-100: f_a += x_a sweep by sweep.
        collide_bgk(o, o.f.data(), o.dt / (o.lambda + 0.5 * o.dt));
        const int n_sweeps = o.prm.streaming == LBFEM_STREAMING_TG3_SPLIT ? 2 : 1;
        for (int s = 0; s < n_sweeps; ++s)
          {
            const int st =
              increment(o, s, o.f.data(), nullptr, -o.dt, 0., -0.5 * o.dt * o.dt, rm < 0 ? true : rm != 0);
            if (st != LBFEM_OK)
              return st;
            double e[2 * Q];
            sweep_directions(o, s, e);
            for (int al = 0; al < NM; ++al)
              {
                if (e[2 * (al + 1)] == 0. && e[2 * (al + 1) + 1] == 0.)
                  continue;
                double *fa = o.f.data() + (al + 1) * N;
                const double *xa = (s == 0 ? o.x0.data() : o.x1.data()) + al * N;
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < N; ++i)
                  fa[i] += xa[i];
              }
          }
        return LBFEM_OK;
      }
    // LeeLin::step, schemes.h:92-98
    compute_equilibrium(o, o.f.data(), o.feq.data());
    const double bb = -0.5 * o.dt * o.dt / o.lambda;
    const int st =
      increment(o, 0, o.f.data(), o.feq.data(), -o.dt - bb, bb, -0.5 * o.dt * o.dt, rm < 0 ? false : rm != 0);
    if (st != LBFEM_OK)
      return st;
    predictor_corrector(o, o.f.data(), o.feq.data(), o.x0.data(), o.dt / o.lambda);
    return LBFEM_OK;
  }
  // ------------------------------------------------------- stream function
  // compute_stream_function (io.h:31-95): (grad phi, grad psi) = (dphi/dx, v) -
  // (dphi/dy, u) with psi = 0 on every side of the box (make_zero_boundary_
  // constraints covers all boundary faces, periodic ones included, and psi has
  // no periodicity constraint), Jacobi-PCG to 1e-12 |b|, at most 10000
  // iterations. psi's DoFs are all stored nodes, images included; the velocity
  // is read through the periodic images (read_dof_values of index 0).
  inline bool
  psi_fixed(const lbfem_oracle &o, int i, int j)
  {
    return i == 0 || j == 0 || i == o.nfx - 1 || j == o.nfy - 1;
  }

  // mode 0: dst = b(u, v); mode 1: dst = K src (the Laplace cell integrals); mode 2:
  // dst = the diagonal of K. Constrained rows are not treated here.
  template <int P>
  void
  psi_cells(const lbfem_oracle &o, const double *u, const double *v, const double *src, double *dst, int mode)
  {
    constexpr int n = P + 1;
    const Basis &B = *o.basis;
    std::fill(dst, dst + o.N, 0.);
    for_cells_coloured(o, [&](int cx, int cy) {
      const double hx = o.vx[cx + 1] - o.vx[cx], hy = o.vy[cy + 1] - o.vy[cy];
      int64_t own[n][n], src_idx[n][n];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          {
            own[j][i] = int64_t(cy * P + j) * o.nfx + cx * P + i;
            src_idx[j][i] = o.master(cx * P + i, cy * P + j);
          }
      double out[n][n] = {};
      for (int q2 = 0; q2 < n; ++q2)
        for (int q1 = 0; q1 < n; ++q1)
          {
            const double JxW = B.qw[q1] * B.qw[q2] * hx * hy;
            if (mode == 2)
              {
                for (int bb = 0; bb < n; ++bb)
                  for (int aa = 0; aa < n; ++aa)
                    {
                      const double gx = B.S[q2][bb] * B.D[q1][aa] / hx, gy = B.D[q2][bb] * B.S[q1][aa] / hy;
                      out[bb][aa] += (gx * gx + gy * gy) * JxW;
                    }
                continue;
              }
            double fx = 0, fy = 0;
            if (mode == 0)
              {
                double uq = 0, vq = 0;
                for (int bb = 0; bb < n; ++bb)
                  for (int aa = 0; aa < n; ++aa)
                    {
                      const double phi = B.S[q2][bb] * B.S[q1][aa];
                      uq += phi * u[src_idx[bb][aa]];
                      vq += phi * v[src_idx[bb][aa]];
                    }
                fx = vq;
                fy = -uq;
              }
            else
              {
                for (int bb = 0; bb < n; ++bb)
                  for (int aa = 0; aa < n; ++aa)
                    {
                      fx += B.S[q2][bb] * B.D[q1][aa] / hx * src[own[bb][aa]];
                      fy += B.D[q2][bb] * B.S[q1][aa] / hy * src[own[bb][aa]];
                    }
              }
            for (int bb = 0; bb < n; ++bb)
              for (int aa = 0; aa < n; ++aa)
                out[bb][aa] += (B.S[q2][bb] * B.D[q1][aa] / hx * fx + B.D[q2][bb] * B.S[q1][aa] / hy * fy) * JxW;
          }
      for (int bb = 0; bb < n; ++bb)
        for (int aa = 0; aa < n; ++aa)
          dst[own[bb][aa]] += out[bb][aa];
    });
  }

  void
  psi_cells_dispatch(const lbfem_oracle &o, const double *u, const double *v, const double *src, double *dst,
                     int mode)
  {
    switch (o.p)
      {
        case 1:
          psi_cells<1>(o, u, v, src, dst, mode);
          break;
        case 2:
          psi_cells<2>(o, u, v, src, dst, mode);
          break;
        case 3:
          psi_cells<3>(o, u, v, src, dst, mode);
          break;
        default:
          psi_cells<4>(o, u, v, src, dst, mode);
      }
  }

  // The Laplace operator of psi with identity rows on the fixed (boundary) nodes;
  // their entries of src are read as zero (homogeneous constraints).
  void
  laplace_vmult(const lbfem_oracle &o, double *dst, const double *src, std::vector<double> &tmp)
  {
    tmp.assign(src, src + o.N);
    for (int j = 0; j < o.nfy; ++j)
      for (int i = 0; i < o.nfx; ++i)
        if (psi_fixed(o, i, j))
          tmp[int64_t(j) * o.nfx + i] = 0.;
    psi_cells_dispatch(o, nullptr, nullptr, tmp.data(), dst, 1);
    for (int j = 0; j < o.nfy; ++j)
      for (int i = 0; i < o.nfx; ++i)
        if (psi_fixed(o, i, j))
          dst[int64_t(j) * o.nfx + i] = src[int64_t(j) * o.nfx + i];
  }

  int
  stream_function(lbfem_oracle &o, const double *u, const double *v, double *psi, int64_t *its)
  {
    const int64_t N = o.N;
    std::vector<double> b(N), diag(N), r(N), z(N), p(N), w(N), tmp;
    psi_cells_dispatch(o, u, v, nullptr, b.data(), 0);
    psi_cells_dispatch(o, nullptr, nullptr, nullptr, diag.data(), 2);
    for (int j = 0; j < o.nfy; ++j)
      for (int i = 0; i < o.nfx; ++i)
        if (psi_fixed(o, i, j))
          {
            b[int64_t(j) * o.nfx + i] = 0.; // distribute_local_to_global drops constrained rows
            diag[int64_t(j) * o.nfx + i] = 1.;
          }
    std::fill(psi, psi + N, 0.);
    // SolverCG with the Jacobi preconditioner from zero, tolerance 1e-12 |b| (io.h:90-92)
    const double tol = 1e-12 * std::sqrt(dot(b.data(), b.data(), N));
    std::copy(b.begin(), b.end(), r.begin());
    double res = std::sqrt(dot(r.data(), r.data(), N)), rz = 0;
    *its = 0;
    if (res <= tol)
      return LBFEM_OK;
    for (int it = 1;; ++it)
      {
        for (int64_t k = 0; k < N; ++k)
          z[k] = r[k] / diag[k];
        const double rz_prev = rz;
        rz = dot(r.data(), z.data(), N);
        if (it > 1)
          for (int64_t k = 0; k < N; ++k)
            p[k] = (rz / rz_prev) * p[k] + z[k];
        else
          std::copy(z.begin(), z.end(), p.begin());
        laplace_vmult(o, w.data(), p.data(), tmp);
        const double alpha = rz / dot(p.data(), w.data(), N);
        for (int64_t k = 0; k < N; ++k)
          {
            psi[k] += alpha * p[k];
            r[k] += -alpha * w[k];
          }
        res = std::sqrt(dot(r.data(), r.data(), N));
        *its = it;
        if (std::isnan(res))
          return LBFEM_ERR_NONFINITE;
        if (res <= tol)
          break;
        if (it >= 10000)
          return LBFEM_ERR_NO_CONVERGENCE;
      }
    // zero.distribute(psi): the fixed nodes are 0
    for (int j = 0; j < o.nfy; ++j)
      for (int i = 0; i < o.nfx; ++i)
        if (psi_fixed(o, i, j))
          psi[int64_t(j) * o.nfx + i] = 0.;
    return LBFEM_OK;
  }
} // namespace

extern "C" {

int
lbfem_oracle_set_threads(int32_t n)
{
#ifdef _OPENMP
  if (n > 0)
    omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int
lbfem_oracle_basis_1d(int32_t p, double *support, double *gp, double *gw)
{
  if (p < 1 || p > MAXP)
    return LBFEM_ERR_ARG;
  Basis B(p);
  for (int k = 0; k <= p; ++k)
    {
      if (support)
        support[k] = B.xi[k];
      if (gp)
        gp[k] = B.qx[k];
      if (gw)
        gw[k] = B.qw[k];
    }
  return LBFEM_OK;
}

int
lbfem_oracle_create(const lbfem_mesh_desc *m, const lbfem_params *prm, lbfem_oracle **h)
{
  if (!m || !prm || !h)
    return LBFEM_ERR_ARG;
  if (m->degree < 1 || m->degree > MAXP || m->n_cells_x < 1 || m->n_cells_y < 1 || m->dof_index)
    return LBFEM_ERR_ARG;
  if ((m->periodic_x && m->n_cells_x < 2) || (m->periodic_y && m->n_cells_y < 2))
    return LBFEM_ERR_ARG;
  // TG3 needs the consistent mass (streaming.h:51-52); Lee-Lin streams with TG2 only (schemes.h:87).
  if (prm->streaming < LBFEM_STREAMING_TG2 || prm->streaming > LBFEM_STREAMING_TG3_SPLIT)
    return LBFEM_ERR_ARG;
  if (prm->streaming != LBFEM_STREAMING_TG2 && (prm->mass != LBFEM_MASS_CG || prm->scheme != LBFEM_SCHEME_BARDOW))
    return LBFEM_ERR_ARG;
  auto o = std::make_unique<lbfem_oracle>();
  o->p = m->degree;
  o->ncx = m->n_cells_x;
  o->ncy = m->n_cells_y;
  o->px = m->periodic_x != 0;
  o->py = m->periodic_y != 0;
  o->nfx = o->p * o->ncx + 1;
  o->nfy = o->p * o->ncy + 1;
  o->N = int64_t(o->nfx) * o->nfy;
  if (m->n_dofs != o->N)
    return LBFEM_ERR_ARG;
  o->vx.assign(m->vertex_x, m->vertex_x + o->ncx + 1);
  o->vy.assign(m->vertex_y, m->vertex_y + o->ncy + 1);
  if (m->vertex_xy)
    {
      // general quadrilaterals: TG2, no walls (the reference's --distort is a Taylor-Green option)
      if (m->n_walls > 0 || prm->streaming != LBFEM_STREAMING_TG2)
        return LBFEM_ERR_UNSUPPORTED;
      o->distorted = true;
      o->vxy.assign(m->vertex_xy, m->vertex_xy + size_t(o->ncx + 1) * (o->ncy + 1) * 2);
    }
  o->basis = std::make_unique<Basis>(o->p);
  o->prm = *prm;
  const int64_t N = o->N;
  o->wall.assign(N, WallU{});
  for (int64_t k = 0; k < m->n_walls; ++k)
    {
      const int64_t d = m->wall_dof[k];
      if (d < 0 || d >= N)
        return LBFEM_ERR_ARG;
      o->wall[d] = {true, m->wall_velocity[2 * k], m->wall_velocity[2 * k + 1]};
    }
  o->constrained.assign(N, 0);
  for (int j = 0; j < o->nfy; ++j)
    for (int i = 0; i < o->nfx; ++i)
      if (o->master(i, j) != int64_t(j) * o->nfx + i)
        o->constrained[int64_t(j) * o->nfx + i] = 1;
  // lumped diagonal: M applied to ones (constraints resolved), constrained = 1
  std::vector<double> ones(N, 1.);
  o->lumped.assign(N, 0.);
  mass_cells_dispatch(*o, ones.data(), o->lumped.data(), 0);
  o->jacobi.assign(N, 0.);
  mass_cells_dispatch(*o, nullptr, o->jacobi.data(), 1);
  o->inv_lumped.resize(N);
  o->inv_jacobi.resize(N);
  for (int64_t i = 0; i < N; ++i)
    {
      if (o->constrained[i])
        {
          o->lumped[i] = 1.;
          o->jacobi[i] = 1.;
        }
      o->inv_lumped[i] = o->lumped[i] == 0. ? 1. : 1. / o->lumped[i];
      o->inv_jacobi[i] = o->jacobi[i] == 0. ? 1. : 1. / o->jacobi[i];
    }
  o->f.assign(Q * N, 0.);
  o->feq.assign(Q * N, 0.);
  o->rhs.assign(NM * N, 0.);
  o->x0.assign(NM * N, 0.);
  o->x1.assign(NM * N, 0.);
  o->cg_r.assign(N, 0.);
  o->cg_p.assign(N, 0.);
  o->cg_v.assign(N, 0.);
  o->cg_z.assign(N, 0.);
  *h = o.release();
  return LBFEM_OK;
}

int
lbfem_oracle_destroy(lbfem_oracle *h)
{
  delete h;
  return LBFEM_OK;
}

int
lbfem_oracle_set_time_step(lbfem_oracle *h, double dt, double lambda)
{
  if (!h || !(dt > 0) || !(lambda > 0))
    return LBFEM_ERR_ARG;
  h->dt = dt;
  h->lambda = lambda;
  h->have_ts = true;
  return LBFEM_OK;
}

int
lbfem_oracle_set_populations(lbfem_oracle *h, const double *f)
{
  if (!h || !f)
    return LBFEM_ERR_ARG;
  std::copy(f, f + Q * h->N, h->f.begin());
  return LBFEM_OK;
}

int
lbfem_oracle_get_populations(lbfem_oracle *h, double *f)
{
  if (!h || !f)
    return LBFEM_ERR_ARG;
  std::copy(h->f.begin(), h->f.end(), f);
  return LBFEM_OK;
}

// write_checkpoint / read_checkpoint (io.h:137-165): name.rank holds the blocks of
// Scheme::f one after the other (raw FP64), written through name.rank.tmp.
int
lbfem_oracle_write_checkpoint(lbfem_oracle *h, const char *name, int32_t rank)
{
  if (!h || !name || rank < 0)
    return LBFEM_ERR_ARG;
  const std::string file = std::string(name) + "." + std::to_string(rank), tmp = file + ".tmp";
  FILE *out = std::fopen(tmp.c_str(), "wb");
  if (!out)
    return LBFEM_ERR_ARG;
  const bool ok = std::fwrite(h->f.data(), sizeof(double), h->f.size(), out) == h->f.size();
  if (std::fclose(out) != 0 || !ok || std::rename(tmp.c_str(), file.c_str()) != 0)
    return LBFEM_ERR_ARG;
  return LBFEM_OK;
}

int
lbfem_oracle_read_checkpoint(lbfem_oracle *h, const char *name, int32_t rank)
{
  if (!h || !name || rank < 0)
    return LBFEM_ERR_ARG;
  const std::string file = std::string(name) + "." + std::to_string(rank);
  FILE *in = std::fopen(file.c_str(), "rb");
  if (!in)
    return LBFEM_ERR_ARG;
  std::vector<double> f(h->f.size());
  const bool ok = std::fread(f.data(), sizeof(double), f.size(), in) == f.size() && std::fgetc(in) == EOF;
  std::fclose(in);
  if (!ok)
    return LBFEM_ERR_ARG;
  h->f = f;
  return LBFEM_OK;
}

int
lbfem_oracle_set_initial_populations(lbfem_oracle *h, const double *f)
{
  if (!h || !f)
    return LBFEM_ERR_ARG;
  if (!h->have_ts)
    return LBFEM_ERR_STATE;
  const int64_t N = h->N;
  std::copy(f, f + Q * N, h->f.begin());
  std::fill(h->x0.begin(), h->x0.end(), 0.);
  std::fill(h->x1.begin(), h->x1.end(), 0.);
  if (h->prm.scheme == LBFEM_SCHEME_BARDOW)
    {
      // Bardow::set_initial_populations, schemes.h:129-141
      const double scale = 0.5 * h->dt / h->lambda;
      for (int64_t i = 0; i < N; ++i)
        {
          double fi[Q], fe[Q];
          for (int a = 0; a < Q; ++a)
            fi[a] = h->f[a * N + i];
          equilibrium(moments(fi), fe);
          for (int a = 0; a < Q; ++a)
            h->f[a * N + i] = fi[a] + scale * (fi[a] - fe[a]);
        }
    }
  return LBFEM_OK;
}

int
lbfem_oracle_step(lbfem_oracle *h, int32_t n_steps)
{
  if (!h || n_steps < 0)
    return LBFEM_ERR_ARG;
  if (!h->have_ts)
    return LBFEM_ERR_STATE;
  for (int s = 0; s < n_steps; ++s)
    {
      const int st = step(*h);
      if (st != LBFEM_OK)
        return st;
    }
  return LBFEM_OK;
}

int
lbfem_oracle_advection(lbfem_oracle *h, const double *f, const double *feq, const double *e, double dt,
                       double lambda, int32_t kind, int32_t remove, double *rhs)
{
  if (!h || !f || !e || !rhs || !(dt > 0))
    return LBFEM_ERR_ARG;
  if (kind == LBFEM_ADVECTION_LEELIN)
    {
      if (!feq || !(lambda > 0))
        return LBFEM_ERR_ARG;
      const double b = -0.5 * dt * dt / lambda;
      advection(*h, f, feq, e, -dt - b, b, -0.5 * dt * dt, dt, remove < 0 ? false : remove != 0, rhs);
      return LBFEM_OK;
    }
  if (kind != LBFEM_ADVECTION_TAYLOR_GALERKIN)
    return LBFEM_ERR_ARG;
  advection(*h, f, nullptr, e, -dt, 0., -0.5 * dt * dt, dt, remove < 0 ? true : remove != 0, rhs);
  return LBFEM_OK;
}

int
lbfem_oracle_mass_solve(lbfem_oracle *h, double *x, const double *r, const double *e, double tg3)
{
  if (!h || !x || !r)
    return LBFEM_ERR_ARG;
  if (tg3 != 0. && !e)
    return LBFEM_ERR_ARG;
  return mass_solve(*h, x, r, tg3 != 0. ? StreamOp{e[0], e[1], tg3} : StreamOp{});
}

int
lbfem_oracle_mass_vmult(lbfem_oracle *h, double *y, const double *x)
{
  if (!h || !x || !y)
    return LBFEM_ERR_ARG;
  mass_vmult(*h, y, x);
  return LBFEM_OK;
}

int
lbfem_oracle_cg_iterations(const lbfem_oracle *h, int64_t *its)
{
  if (!h || !its)
    return LBFEM_ERR_ARG;
  *its = h->cg_its;
  return LBFEM_OK;
}

int
lbfem_oracle_collide_bgk(lbfem_oracle *h, double *g, double omega)
{
  if (!h || !g)
    return LBFEM_ERR_ARG;
  collide_bgk(*h, g, omega);
  return LBFEM_OK;
}

int
lbfem_oracle_compute_equilibrium(lbfem_oracle *h, const double *f, double *feq)
{
  if (!h || !f || !feq)
    return LBFEM_ERR_ARG;
  compute_equilibrium(*h, f, feq);
  return LBFEM_OK;
}

int
lbfem_oracle_predictor_corrector(lbfem_oracle *h, double *f, const double *feq, const double *incr, double theta)
{
  if (!h || !f || !feq || !incr)
    return LBFEM_ERR_ARG;
  predictor_corrector(*h, f, feq, incr, theta);
  return LBFEM_OK;
}

int
lbfem_oracle_node_weight(lbfem_oracle *h, double *w)
{
  if (!h || !w)
    return LBFEM_ERR_ARG;
  std::copy(h->lumped.begin(), h->lumped.end(), w);
  return LBFEM_OK;
}

int
lbfem_oracle_jacobi_diagonal(lbfem_oracle *h, double *d)
{
  if (!h || !d)
    return LBFEM_ERR_ARG;
  std::copy(h->jacobi.begin(), h->jacobi.end(), d);
  return LBFEM_OK;
}

int
lbfem_oracle_conservation(lbfem_oracle *h, double out[5])
{
  if (!h || !out)
    return LBFEM_ERR_ARG;
  const int64_t N = h->N;
  double s[5] = {0, 0, 0, 0, 0};
  for (int64_t i = 0; i < N; ++i)
    {
      const int64_t row = i / h->nfx;
      if (h->constrained[i] || (h->strip && (row < h->oy0 || row >= h->oy1)))
        continue;
      double fi[Q];
      for (int a = 0; a < Q; ++a)
        fi[a] = h->f[a * N + i];
      const Moments m = moments(fi);
      const double w = h->lumped[i];
      s[0] += w;
      s[1] += w * m.rho;
      s[2] += w * m.rho * m.ux;
      s[3] += w * m.rho * m.uy;
      s[4] += w * (m.ux * m.ux + m.uy * m.uy);
    }
  std::copy(s, s + 5, out);
  return LBFEM_OK;
}


int
lbfem_oracle_strip_buffer_bytes(const lbfem_oracle *h, int64_t *bytes)
{
  if (!h || !bytes)
    return LBFEM_ERR_ARG;
  *bytes = int64_t(Q) * h->p * h->nfx * int64_t(sizeof(double));
  return LBFEM_OK;
}

int
lbfem_oracle_set_strip(lbfem_oracle *h, const lbfem_strip_desc *sd)
{
  if (!h || !sd || !sd->comm || !sd->sums || h->py || h->distorted)
    return LBFEM_ERR_ARG;
  if ((sd->ghost_below != 0 && sd->ghost_below != h->p) || (sd->ghost_above != 0 && sd->ghost_above != 1))
    return LBFEM_ERR_ARG;
  if ((sd->ghost_below && (!sd->send_below || !sd->recv_below)) ||
      (sd->ghost_above && (!sd->send_above || !sd->recv_above)))
    return LBFEM_ERR_ARG;
  const int oy0 = sd->ghost_below, oy1 = h->nfy - sd->ghost_above;
  if (oy1 - oy0 < h->p + 1 || !(sd->cell_below >= 0) || !(sd->cell_above >= 0))
    return LBFEM_ERR_ARG;
  // the neighbours' cell's share of the mass diagonals of the end rows (a vertex
  // row's diagonal and row sum scale with the summed width of its two cells)
  const double fb = (h->vy[1] - h->vy[0] + sd->cell_below) / (h->vy[1] - h->vy[0]);
  const double fa = (h->vy[h->ncy] - h->vy[h->ncy - 1] + sd->cell_above) / (h->vy[h->ncy] - h->vy[h->ncy - 1]);
  for (int i = 0; i < h->nfx; ++i)
    for (const auto &[row, fac] : {std::pair<int, double>{0, fb}, std::pair<int, double>{h->nfy - 1, fa}})
      {
        const int64_t k = int64_t(row) * h->nfx + i;
        if (h->constrained[k])
          continue;
        h->jacobi[k] *= fac;
        h->lumped[k] *= fac;
        h->inv_jacobi[k] = 1. / h->jacobi[k];
        h->inv_lumped[k] = 1. / h->lumped[k];
      }
  h->sd = *sd;
  h->strip = true;
  h->oy0 = oy0;
  h->oy1 = oy1;
  return LBFEM_OK;
}

int
lbfem_oracle_stream_function(lbfem_oracle *h, const double *velocity, double *psi)
{
  if (!h || !velocity || !psi)
    return LBFEM_ERR_ARG;
  if (h->strip || h->distorted)
    return LBFEM_ERR_UNSUPPORTED;
  int64_t its = 0;
  return stream_function(*h, velocity, velocity + h->N, psi, &its);
}
} // extern "C"
