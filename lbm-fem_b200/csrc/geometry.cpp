#include "geometry.h"

#include <cmath>

namespace lbfem_gpu
{
  namespace
  {
    // Legendre P_n(t) and its derivative (three-term recurrence).
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

    struct Lagrange
    {
      int p;
      long double x[MAXP + 1];
      long double
      value(int a, long double t) const
      {
        long double v = 1;
        for (int b = 0; b <= p; ++b)
          if (b != a)
            v *= (t - x[b]) / (x[a] - x[b]);
        return v;
      }
      long double
      deriv(int a, long double t) const
      {
        long double sum = 0;
        for (int c = 0; c <= p; ++c)
          {
            if (c == a)
              continue;
            long double v = 1 / (x[a] - x[c]);
            for (int b = 0; b <= p; ++b)
              if (b != a && b != c)
                v *= (t - x[b]) / (x[a] - x[b]);
            sum += v;
          }
        return sum;
      }
    };
  } // namespace

  Basis1D::Basis1D(int p_)
    : p(p_)
  {
    const long double pi = 3.141592653589793238462643383279502884L;
    Lagrange L{p, {}};
    // support points: 0, 1 and the roots of P_p' (Newton on P_p' with P_p'')
    L.x[0] = 0;
    L.x[p] = 1;
    for (int k = 1; k < p; ++k)
      {
        long double t = -std::cos(pi * k / p);
        for (int it = 0; it < 100; ++it)
          {
            long double dp;
            const long double v = legendre(p, t, &dp);
            const long double d2 = (2 * t * dp - p * (p + 1) * v) / (1 - t * t);
            const long double step = dp / d2;
            t -= step;
            if (std::fabs(step) < 1e-19L)
              break;
          }
        L.x[k] = (t + 1) / 2;
      }
    // Gauss points (roots of P_{p+1}) and weights on [0,1]
    const int nq = p + 1;
    long double qx[MAXP + 1], qw[MAXP + 1];
    for (int k = 0; k < nq; ++k)
      {
        long double t = -std::cos(pi * (k + 0.75L) / (nq + 0.5L));
        for (int it = 0; it < 100; ++it)
          {
            long double dp;
            const long double v = legendre(nq, t, &dp);
            const long double step = v / dp;
            t -= step;
            if (std::fabs(step) < 1e-19L)
              break;
          }
        long double dp;
        legendre(nq, t, &dp);
        qx[k] = (t + 1) / 2;
        qw[k] = 1 / ((1 - t * t) * dp * dp);
      }
    for (int q = 0; q < nq; ++q)
      {
        gq[q] = double(qx[q]);
        gw[q] = double(qw[q]);
        for (int a = 0; a <= p; ++a)
          {
            gS[q][a] = double(L.value(a, qx[q]));
            gD[q][a] = double(L.deriv(a, qx[q]));
          }
      }
    for (int a = 0; a <= p; ++a)
      {
        xi[a] = double(L.x[a]);
        d0[a] = double(L.deriv(a, 0));
        d1[a] = double(L.deriv(a, 1));
        for (int b = 0; b <= p; ++b)
          {
            long double m = 0, c = 0, k = 0;
            for (int q = 0; q < nq; ++q)
              {
                m += qw[q] * L.value(a, qx[q]) * L.value(b, qx[q]);
                c += qw[q] * L.value(a, qx[q]) * L.deriv(b, qx[q]);
                k += qw[q] * L.deriv(a, qx[q]) * L.deriv(b, qx[q]);
              }
            Mh[a][b] = double(m);
            Ch[a][b] = double(c);
            Kh[a][b] = double(k);
          }
      }
  }

  Axis
  make_axis(const Basis1D &b, const double *vertex, int n_cells, bool periodic)
  {
    Axis ax;
    const int p = b.p, K = 2 * p + 1;
    ax.p = p;
    ax.n_cells = n_cells;
    ax.periodic = periodic;
    ax.n_nodes = p * n_cells + 1;
    ax.n_unique = periodic ? p * n_cells : ax.n_nodes;
    ax.vertex.assign(vertex, vertex + n_cells + 1);
    ax.h_first = vertex[1] - vertex[0];
    ax.h_last = vertex[n_cells] - vertex[n_cells - 1];
    std::vector<long double> acc(size_t(4) * ax.n_nodes * K, 0.0L);
    auto at = [&](int m, int i, int k) -> long double & { return acc[(size_t(m) * ax.n_nodes + i) * K + k]; };
    for (int c = 0; c < n_cells; ++c)
      {
        const long double h = (long double)vertex[c + 1] - vertex[c];
        for (int a = 0; a <= p; ++a)
          {
            int i = c * p + a;
            if (periodic && i == ax.n_unique)
              i = 0; // the image row is assembled into its source
            for (int bb = 0; bb <= p; ++bb)
              {
                const int k = bb - a + p;
                at(0, i, k) += h * b.Mh[a][bb];
                at(1, i, k) += b.Ch[a][bb];
                at(2, i, k) += b.Ch[bb][a];
                at(3, i, k) += b.Kh[a][bb] / h;
              }
          }
      }
    ax.rows.resize(acc.size());
    for (size_t t = 0; t < acc.size(); ++t)
      ax.rows[t] = double(acc[t]);
    ax.diag.assign(ax.n_nodes, 1.0);
    ax.lump.assign(ax.n_nodes, 1.0);
    ax.h.resize(n_cells);
    ax.hinv.resize(n_cells);
    for (int c = 0; c < n_cells; ++c)
      {
        ax.h[c] = vertex[c + 1] - vertex[c];
        ax.hinv[c] = 1.0 / ax.h[c];
      }
    for (int i = 0; i < ax.n_unique; ++i)
      {
        long double s = 0;
        for (int k = 0; k < K; ++k)
          s += at(0, i, k);
        ax.diag[i] = double(at(0, i, p));
        ax.lump[i] = double(s);
      }
    ax.invdiag.resize(ax.n_nodes);
    ax.invlump.resize(ax.n_nodes);
    for (int i = 0; i < ax.n_nodes; ++i)
      {
        ax.invdiag[i] = 1.0 / ax.diag[i];
        ax.invlump[i] = 1.0 / ax.lump[i];
      }
    return ax;
  }

  std::vector<float>
  window_ldl(const Axis &ax, int T, int W, int n_tiles, int stride)
  {
    const int p = ax.p, K = 2 * p + 1, n = T + 2 * W;
    std::vector<float> out(size_t(n_tiles) * n * stride, 0.f);
    std::vector<long double> a(size_t(n) * K), d(n), l(size_t(n) * (p + 1));
    auto row = [&](int q) { return &a[size_t(q) * K]; };  // band of row q: [k] couples q to q + k - p
    auto lo = [&](int q, int k) -> long double & { return l[size_t(q) * (p + 1) + k]; }; // l_{q, q-k}
    for (int t = 0; t < n_tiles; ++t)
      {
        // the window's band
        for (int q = 0; q < n; ++q)
          {
            long double *r = row(q);
            for (int k = 0; k < K; ++k)
              r[k] = 0;
            int c = t * T - W + q;
            bool valid = true;
            if (ax.periodic)
              {
                c %= ax.n_unique;
                if (c < 0)
                  c += ax.n_unique;
              }
            else
              valid = c >= 0 && c < ax.n_nodes;
            if (!valid)
              {
                r[p] = 1; // identity row outside the axis
                continue;
              }
            for (int k = 0; k < K; ++k)
              {
                const int q2 = q + k - p;
                if (q2 < 0 || q2 >= n)
                  continue;
                if (!ax.periodic)
                  {
                    const int c2 = t * T - W + q2;
                    if (c2 < 0 || c2 >= ax.n_nodes)
                      continue;
                  }
                r[k] = ax.rows[(size_t(0) * ax.n_nodes + c) * K + k];
              }
          }
        // banded LDL^T (no pivoting: the window matrix is symmetric positive definite)
        for (int q = 0; q < n; ++q)
          {
            for (int k = p; k >= 1; --k) // columns j = q - k in increasing order
              {
                const int j = q - k; // l_{q,j} = (a_{q,j} - sum_{m<j} l_{q,m} l_{j,m} d_m) / d_j
                if (j < 0)
                  {
                    lo(q, k) = 0;
                    continue;
                  }
                long double s = row(q)[p - k];
                for (int m = 1; m <= p - k; ++m)
                  if (j - m >= 0)
                    s -= lo(q, k + m) * lo(j, m) * d[j - m];
                lo(q, k) = s / d[j];
              }
            long double s = row(q)[p];
            for (int k = 1; k <= p; ++k)
              if (q - k >= 0)
                s -= lo(q, k) * lo(q, k) * d[q - k];
            d[q] = s;
          }
        float *o = &out[size_t(t) * n * stride];
        for (int q = 0; q < n; ++q)
          {
            for (int k = 1; k <= p; ++k)
              o[q * stride + k - 1] = float(lo(q, k));
            o[q * stride + p] = float(1.0L / d[q]);
          }
      }
    return out;
  }

  std::vector<double>
  quad_geometry(const Basis1D &b, const double *vxy, int ncx, int ncy)
  {
    const int n = b.p + 1;
    std::vector<double> g(size_t(ncx) * ncy * n * n * 5);
    auto v = [&](int i, int j, int k) { return vxy[(size_t(j) * (ncx + 1) + i) * 2 + k]; };
    for (int cy = 0; cy < ncy; ++cy)
      for (int cx = 0; cx < ncx; ++cx)
        for (int q2 = 0; q2 < n; ++q2)
          for (int q1 = 0; q1 < n; ++q1)
            {
              const double s = b.gq[q1], t = b.gq[q2];
              double J[2][2];
              for (int k = 0; k < 2; ++k)
                {
                  J[k][0] = (1 - t) * (v(cx + 1, cy, k) - v(cx, cy, k)) + t * (v(cx + 1, cy + 1, k) - v(cx, cy + 1, k));
                  J[k][1] = (1 - s) * (v(cx, cy + 1, k) - v(cx, cy, k)) + s * (v(cx + 1, cy + 1, k) - v(cx + 1, cy, k));
                }
              const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
              double *o = &g[((size_t(cy) * ncx + cx) * n * n + q2 * n + q1) * 5];
              o[0] = J[1][1] / det;
              o[1] = -J[0][1] / det;
              o[2] = -J[1][0] / det;
              o[3] = J[0][0] / det;
              o[4] = b.gw[q1] * b.gw[q2] * det;
            }
    return g;
  }

  void
  quad_diagonals(const Basis1D &b, const std::vector<double> &geo, int ncx, int ncy, bool px, bool py,
                 std::vector<double> &jacobi, std::vector<double> &lumped)
  {
    const int p = b.p, n = p + 1, nfx = p * ncx + 1, nfy = p * ncy + 1;
    jacobi.assign(size_t(nfx) * nfy, 0.);
    lumped.assign(size_t(nfx) * nfy, 0.);
    auto master = [&](int i, int j) {
      if (px && i == p * ncx)
        i = 0;
      if (py && j == p * ncy)
        j = 0;
      return size_t(j) * nfx + i;
    };
    for (int cy = 0; cy < ncy; ++cy)
      for (int cx = 0; cx < ncx; ++cx)
        for (int bb = 0; bb < n; ++bb)
          for (int aa = 0; aa < n; ++aa)
            {
              double sj = 0, sl = 0;
              for (int q2 = 0; q2 < n; ++q2)
                for (int q1 = 0; q1 < n; ++q1)
                  {
                    const double phi = b.gS[q1][aa] * b.gS[q2][bb];
                    const double jxw = geo[((size_t(cy) * ncx + cx) * n * n + q2 * n + q1) * 5 + 4];
                    sj += phi * phi * jxw;
                    sl += phi * jxw;
                  }
              const size_t k = master(cx * p + aa, cy * p + bb);
              jacobi[k] += sj;
              lumped[k] += sl;
            }
    for (int j = 0; j < nfy; ++j)
      for (int i = 0; i < nfx; ++i)
        if ((px && i == p * ncx) || (py && j == p * ncy))
          {
            jacobi[size_t(j) * nfx + i] = 1.;
            lumped[size_t(j) * nfx + i] = 1.;
          }
  }
} // namespace lbfem_gpu
