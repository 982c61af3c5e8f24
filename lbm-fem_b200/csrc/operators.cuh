// The hot-path kernels: streaming right-hand side (K1), wall-face surface term,
// mass vmult and the Jacobi-PCG steps (K2/K3), lumped solve (K4) and the nodal
// maps of the schemes (K5/K6). FP64.
#pragma once

#include "kernels.cuh"

namespace lbfem_gpu
{
  // ----------------------------------------------------------- nodal maps
  // collide_bgk (collision.h:152-168): g <- geq(rho, u_imposed) + (1 - omega)(g - geq(rho, u)).
  __device__ __forceinline__ void
  collide_node(double (&g)[Q], long long idx, const Geo &geo, double omega)
  {
    const Mom m = moments(g);
    const Mom mt = impose(m, idx, geo);
#pragma unroll
    for (int a = 0; a < Q; ++a)
      g[a] = feq_a(a, mt) + (1. - omega) * (g[a] - feq_a(a, m));
  }

  __global__ void
  k_collide(const Geo geo, double *__restrict__ g, double omega)
  {
    const long long N = geo.g.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      {
        double v[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a)
          v[a] = g[a * N + i];
        collide_node(v, i, geo, omega);
#pragma unroll
        for (int a = 0; a < Q; ++a)
          g[a * N + i] = v[a];
      }
  }

  // compute_equilibrium (collision.h:105-113)
  __global__ void
  k_equilibrium(const Geo geo, const double *__restrict__ f, double *__restrict__ feq)
  {
    const long long N = geo.g.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      {
        double v[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a)
          v[a] = f[a * N + i];
        const Mom m = impose(moments(v), i, geo);
#pragma unroll
        for (int a = 0; a < Q; ++a)
          feq[a * N + i] = feq_a(a, m);
      }
  }

  // predictor_corrector (collision.h:119-145); feq == nullptr: the equilibria of
  // f^n are recomputed here (the fused Lee-Lin step never stores them).
  __global__ void
  k_predictor_corrector(const Geo geo, double *__restrict__ f, const double *__restrict__ feq,
                        const double *__restrict__ x, double theta)
  {
    const long long N = geo.g.N;
    const double inv = 1. / (1. + theta);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      {
        double fi[Q], fe[Q], fh[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a)
          fi[a] = f[a * N + i];
        if (feq)
          {
#pragma unroll
            for (int a = 0; a < Q; ++a)
              fe[a] = feq[a * N + i];
          }
        else
          {
            const Mom m = impose(moments(fi), i, geo);
#pragma unroll
            for (int a = 0; a < Q; ++a)
              fe[a] = feq_a(a, m);
          }
        fh[0] = inv * (fi[0] + theta * fe[0]);
#pragma unroll
        for (int a = 1; a < Q; ++a)
          fh[a] = inv * (fi[a] + theta * fe[a] + x[(a - 1) * N + i]);
        const Mom mh = impose(moments(fh), i, geo);
#pragma unroll
        for (int a = 0; a < Q; ++a)
          f[a * N + i] = fh[a] + theta * (feq_a(a, mh) - fe[a]);
      }
  }

  // Bardow::set_initial_populations (schemes.h:129-141): g = f + scale (f - feq(f)), no imposition.
  __global__ void
  k_bardow_transform(const Geo geo, double *__restrict__ f, double scale)
  {
    const long long N = geo.g.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      {
        double v[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a)
          v[a] = f[a * N + i];
        const Mom m = moments(v);
#pragma unroll
        for (int a = 0; a < Q; ++a)
          f[a * N + i] = v[a] + scale * (v[a] - feq_a(a, m));
      }
  }

  // TaylorGalerkin::stream (streaming.h:94-98): f_a += x_{a-1}, a = 1..8.
  __global__ void
  k_add_increment(const Geo geo, double *__restrict__ f, const double *__restrict__ x)
  {
    const long long N = geo.g.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      {
#pragma unroll
        for (int a = 1; a < Q; ++a)
          f[a * N + i] += x[(a - 1) * N + i];
      }
  }

  // Lumped solve (mass.h:189-191): x = M_L^{-1} r, for nsys vectors.
  __global__ void
  k_lumped(const Geo geo, const double *__restrict__ r, double *__restrict__ x, int nsys)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x)
      {
        const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
        const double inv = is_image(i, j, g) ? 1.0 : 1.0 / (geo.lumpx[i] * geo.lumpy[j]);
        for (int s = 0; s < nsys; ++s)
          x[s * N + idx] = inv * r[s * N + idx];
      }
  }

  // Node weights: the lumped (which = 0) or Jacobi (which = 1) diagonal, images 1.
  __global__ void
  k_diagonal(const Geo geo, double *__restrict__ w, int which)
  {
    const Grid &g = geo.g;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < g.N;
         idx += (long long)gridDim.x * blockDim.x)
      {
        const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
        w[idx] = is_image(i, j, g) ? 1.0 : which == 0 ? geo.lumpx[i] * geo.lumpy[j] : geo.diagx[i] * geo.diagy[j];
      }
  }

  // Moments at every node; images report their source node (constraints.distribute).
  __global__ void
  k_moments(const Geo geo, const double *__restrict__ f, double *__restrict__ rho, double *__restrict__ ux,
            double *__restrict__ uy)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x)
      {
        const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
        const long long src = (long long)wrap(j, g.py, g.nuy, g.nfy) * g.nfx + wrap(i, g.px, g.nux, g.nfx);
        double v[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a)
          v[a] = f[a * N + src];
        const Mom m = moments(v);
        if (rho)
          rho[idx] = m.rho;
        if (ux)
          ux[idx] = m.ux;
        if (uy)
          uy[idx] = m.uy;
      }
  }

  // FP64 conservation sums over the independent nodes (cgdbe.cc:353-368).
  __global__ void
  k_conservation(const Geo geo, const double *__restrict__ f, double *__restrict__ partials)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    double s[5] = {0, 0, 0, 0, 0};
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x)
      {
        const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
        if (is_image(i, j, g))
          continue;
        double v[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a)
          v[a] = f[a * N + idx];
        const Mom m = moments(v);
        const double w = geo.lumpx[i] * geo.lumpy[j];
        s[0] += w;
        s[1] += w * m.rho;
        s[2] += w * m.rho * m.ux;
        s[3] += w * m.rho * m.uy;
        s[4] += w * (m.ux * m.ux + m.uy * m.uy);
      }
    block_reduce_store<5>(s, 5, partials, blockIdx.x, gridDim.x);
  }

  // Caller numbering <-> structured numbering, nb blocks of a vector.
  __global__ void
  k_gather(const double *__restrict__ src, const long long *__restrict__ dof, double *__restrict__ dst, long long N,
           long long n_dofs, int nb)
  {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x)
      {
        const long long d = dof[s];
        for (int b = 0; b < nb; ++b)
          dst[b * N + s] = src[b * n_dofs + d];
      }
  }

  __global__ void
  k_scatter(const double *__restrict__ src, const long long *__restrict__ dof, double *__restrict__ dst, long long N,
            long long n_dofs, int nb)
  {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x)
      {
        const long long d = dof[s];
        for (int b = 0; b < nb; ++b)
          dst[b * n_dofs + d] = src[b * N + s];
      }
  }

  // ------------------------------------------------- K1: streaming right-hand side
  enum AdvMode
  {
    ADV_TG = 0,          // TaylorGalerkinAdvection on the given populations
    ADV_TG_COLLIDE = 1,  // Bardow step: collide_bgk on the fly, write g*, then TaylorGalerkinAdvection
    ADV_LEELIN_FEQ = 2,  // LeeLinAdvection with the equilibria given as an array
    ADV_LEELIN_FUSED = 3 // Lee-Lin step: the equilibria (wall velocity imposed) computed on the fly
  };

  struct AdvCoef
  {
    double a, b, c;        // point operation: value a e.grad f + b e.grad feq, flux c e (e.grad f)
    double ex[NM], ey[NM]; // directions of the moving populations
    double omega;          // BGK rate (ADV_TG_COLLIDE)
  };

  template <int P, int MODE>
  constexpr size_t
  advection_smem()
  {
    using T = Tile<P>;
    return sizeof(double) * (4 * T::TX * T::K + 4 * T::TY * T::K + 9 * T::HN + T::HN + 3 * T::HN + 4 * T::HY * T::TX);
  }

  // rhs_{a-1} <- r_a for a = 1..8 (advection.h:93-124 with the point operations of
  // advection.h:228-239 / 275-287): cell integrals over the whole mesh, in the
  // assembled tensor-product form
  //   r = My (x) (a ex Cx + c ex^2 Kx) f + Cy (x) (a ey Mx + c ex ey Cx^T) f
  //     + Ky (x) (c ey^2 Mx) f + Cy^T (x) (c ex ey Cx) f  [+ b (ex My (x) Cx + ey Cy (x) Mx) feq].
  // Images get 0 (constrained rows, as distribute_local_to_global leaves them).
  template <int P, int MODE>
  __global__ void __launch_bounds__(THREADS)
    k_advection(const Geo geo, const double *__restrict__ f, const double *__restrict__ feq,
                double *__restrict__ fout, double *__restrict__ rhs, const AdvCoef ac)
  {
    using T = Tile<P>;
    constexpr int TX = T::TX, TY = T::TY, HX = T::HX, HN = T::HN, K = T::K;
    extern __shared__ double sm[];
    double *s_rx = sm;
    double *s_ry = s_rx + 4 * TX * K;
    double *s_f = s_ry + 4 * TY * K; // [9][HN]
    double *s_q = s_f + 9 * HN;      // [HN]: equilibrium of the current population
    double *s_m = s_q + HN;          // [3][HN]: rho, ux, uy (imposed) for ADV_LEELIN_FUSED
    double *s_t = s_m + 3 * HN;      // [4][HY][TX]
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;

    load_rows<P>(s_rx, geo.rowx, gx0, TX, g.nfx);
    load_rows<P>(s_ry, geo.rowy, gy0, TY, g.nfy);
    constexpr bool all9 = MODE == ADV_TG_COLLIDE || MODE == ADV_LEELIN_FUSED;
    for (int a = all9 ? 0 : 1; a < Q; ++a)
      load_tile<P>(s_f + a * HN, f + a * N, g, gx0, gy0);
    __syncthreads();

    if constexpr (all9)
      {
        for (int t = threadIdx.x; t < HN; t += blockDim.x)
          {
            const int ly = t / HX, lx = t - ly * HX;
            const int sx = wrap(gx0 - P + lx, g.px, g.nux, g.nfx), sy = wrap(gy0 - P + ly, g.py, g.nuy, g.nfy);
            if (sx < 0 || sy < 0)
              {
                if constexpr (MODE == ADV_LEELIN_FUSED)
                  s_m[t] = s_m[HN + t] = s_m[2 * HN + t] = 0.0;
                continue;
              }
            const long long idx = (long long)sy * g.nfx + sx;
            double v[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a)
              v[a] = s_f[a * HN + t];
            if constexpr (MODE == ADV_TG_COLLIDE)
              {
                collide_node(v, idx, geo, ac.omega);
#pragma unroll
                for (int a = 0; a < Q; ++a)
                  s_f[a * HN + t] = v[a];
                const int gx = gx0 - P + lx, gy = gy0 - P + ly;
                if (lx >= P && lx < P + TX && ly >= P && ly < P + TY && gx < g.nfx && gy < g.nfy &&
                    !is_image(gx, gy, g))
                  {
#pragma unroll
                    for (int a = 0; a < Q; ++a)
                      fout[a * N + idx] = v[a];
                  }
              }
            else
              {
                const Mom m = impose(moments(v), idx, geo);
                s_m[t] = m.rho;
                s_m[HN + t] = m.ux;
                s_m[2 * HN + t] = m.uy;
              }
          }
        __syncthreads();
      }

    for (int al = 0; al < NM; ++al)
      {
        const int a = al + 1;
        const double ex = ac.ex[al], ey = ac.ey[al];
        const bool hx = ex != 0.0, hy = ey != 0.0;
        constexpr bool two = MODE == ADV_LEELIN_FEQ || MODE == ADV_LEELIN_FUSED;
        if constexpr (MODE == ADV_LEELIN_FEQ)
          {
            load_tile<P>(s_q, feq + a * N, g, gx0, gy0);
            __syncthreads();
          }
        else if constexpr (MODE == ADV_LEELIN_FUSED)
          {
            for (int t = threadIdx.x; t < HN; t += blockDim.x)
              s_q[t] = feq_a(a, Mom{s_m[t], s_m[HN + t], s_m[2 * HN + t]});
            __syncthreads();
          }
        // x pass: the four x-filtered fields of the y operators My, Cy, Ky, Cy^T
        const double *u = s_f + a * HN;
        for (int t = threadIdx.x; t < T::HY * TX; t += blockDim.x)
          {
            const int ly = t / TX, lxo = t - ly * TX;
            const double *rM = s_rx + (0 * TX + lxo) * K, *rC = s_rx + (1 * TX + lxo) * K;
            const double *rT = s_rx + (2 * TX + lxo) * K, *rK = s_rx + (3 * TX + lxo) * K;
            const double *uu = u + ly * HX + lxo;
            double Cu = 0, Mu = 0, Tu = 0, Ku = 0, Ce = 0, Me = 0;
            if (hx)
              {
#pragma unroll
                for (int k = 0; k < K; ++k)
                  {
                    Cu += rC[k] * uu[k];
                    Ku += rK[k] * uu[k];
                  }
                if constexpr (two)
                  {
                    const double *ee = s_q + ly * HX + lxo;
#pragma unroll
                    for (int k = 0; k < K; ++k)
                      Ce += rC[k] * ee[k];
                  }
              }
            if (hy)
              {
#pragma unroll
                for (int k = 0; k < K; ++k)
                  Mu += rM[k] * uu[k];
                if (hx)
                  {
#pragma unroll
                    for (int k = 0; k < K; ++k)
                      Tu += rT[k] * uu[k];
                  }
                if constexpr (two)
                  {
                    const double *ee = s_q + ly * HX + lxo;
#pragma unroll
                    for (int k = 0; k < K; ++k)
                      Me += rM[k] * ee[k];
                  }
              }
            const int nt = T::HY * TX;
            s_t[t] = ac.a * ex * Cu + ac.c * ex * ex * Ku + ac.b * ex * Ce;          // -> My
            s_t[nt + t] = ac.a * ey * Mu + ac.c * ex * ey * Tu + ac.b * ey * Me;     // -> Cy
            s_t[2 * nt + t] = ac.c * ey * ey * Mu;                                  // -> Ky
            s_t[3 * nt + t] = ac.c * ex * ey * Cu;                                  // -> Cy^T
          }
        __syncthreads();
        // y pass and store
        for (int t = threadIdx.x; t < TY * TX; t += blockDim.x)
          {
            const int lyo = t / TX, lxo = t - lyo * TX;
            const int gx = gx0 + lxo, gy = gy0 + lyo;
            if (gx >= g.nfx || gy >= g.nfy)
              continue;
            double r = 0;
            if (!is_image(gx, gy, g))
              {
                const int nt = T::HY * TX;
                const double *yM = s_ry + (0 * TY + lyo) * K, *yC = s_ry + (1 * TY + lyo) * K;
                const double *yT = s_ry + (2 * TY + lyo) * K, *yK = s_ry + (3 * TY + lyo) * K;
#pragma unroll
                for (int k = 0; k < K; ++k)
                  r += yM[k] * s_t[(lyo + k) * TX + lxo];
                if (hy)
                  {
#pragma unroll
                    for (int k = 0; k < K; ++k)
                      r += yC[k] * s_t[nt + (lyo + k) * TX + lxo] + yK[k] * s_t[2 * nt + (lyo + k) * TX + lxo];
                    if (hx)
                      {
#pragma unroll
                        for (int k = 0; k < K; ++k)
                          r += yT[k] * s_t[3 * nt + (lyo + k) * TX + lxo];
                      }
                  }
              }
            rhs[al * N + (long long)gy * g.nfx + gx] = r;
          }
        __syncthreads();
      }

    if constexpr (MODE == ADV_TG_COLLIDE)
      {
        // the images collide their own (stale) populations, as the nodal map does
        for (int t = threadIdx.x; t < TY * TX; t += blockDim.x)
          {
            const int lyo = t / TX, lxo = t - lyo * TX;
            const int gx = gx0 + lxo, gy = gy0 + lyo;
            if (gx >= g.nfx || gy >= g.nfy || !is_image(gx, gy, g))
              continue;
            const long long idx = (long long)gy * g.nfx + gx;
            double v[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a)
              v[a] = f[a * N + idx];
            collide_node(v, idx, geo, ac.omega);
#pragma unroll
            for (int a = 0; a < Q; ++a)
              fout[a * N + idx] = v[a];
          }
      }
  }

  // ----------------------------------------------- wall faces (surface term)
  struct FaceCoef
  {
    double half_dt2;       // dt^2 / 2
    double ex[NM], ey[NM]; // directions
    int remove;            // remove the mass flux isotropically (advection.h:194-196)
    double d0[5], d1[5];   // l_a'(0), l_a'(1) of the 1-D basis
    double hx0, hx1, hy0, hy1; // first and last cell widths per axis
  };

  // rhs += int_wall phi (dt^2/2)(n.e)(e.grad f) (advection.h:126-146,182-199) at the
  // boundary nodes of the non-periodic sides; one thread per boundary node
  // (bnode = (i, j, side mask: 1 bottom, 2 top, 4 left, 8 right)).
  template <int P>
  __global__ void
  k_wall_faces(const Geo geo, const double *__restrict__ f, double *__restrict__ rhs, const int4 *__restrict__ bnode,
               int n_bnodes, const FaceCoef fc)
  {
    constexpr int K = 2 * P + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_bnodes)
      return;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int4 bn = bnode[t];
    const int i = bn.x, j = bn.y, sides = bn.z;
    double R[NM];
#pragma unroll
    for (int al = 0; al < NM; ++al)
      R[al] = 0;
    for (int side = 0; side < 4; ++side)
      {
        if (!(sides & (1 << side)))
          continue;
        const bool horizontal = side < 2;
        const double *rows = horizontal ? geo.rowx : geo.rowy;
        const int n_nodes = horizontal ? g.nfx : g.nfy;
        const int per = horizontal ? g.px : g.py, nu = horizontal ? g.nux : g.nuy;
        const int tpos = horizontal ? i : j;
        const double *dn = (side == 0 || side == 2) ? fc.d0 : fc.d1;
        const double hn = side == 0 ? fc.hy0 : side == 1 ? fc.hy1 : side == 2 ? fc.hx0 : fc.hx1;
        const int base = (side == 0 || side == 2) ? 0 : (horizontal ? g.nfy : g.nfx) - 1 - P; // first normal layer
        const int line = (side == 0) ? 0 : (side == 1) ? g.nfy - 1 : (side == 2) ? 0 : g.nfx - 1;
        for (int al = 0; al < NM; ++al)
          {
            const double ex = fc.ex[al], ey = fc.ey[al];
            const double en = side == 0 ? -ey : side == 1 ? ey : side == 2 ? -ex : ex;
            if (en == 0.0)
              continue;
            const double et = horizontal ? ex : ey; // tangential component
            const double enn = horizontal ? ey : ex; // normal component (derivative direction)
            const double *u = f + (long long)(al + 1) * N;
            double tang = 0, norm = 0;
            for (int k = 0; k < K; ++k)
              {
                const int s = wrap(tpos + k - P, per, nu, n_nodes);
                if (s < 0)
                  continue;
                const double cM = rows[((long long)0 * n_nodes + tpos) * K + k];
                const double cC = rows[((long long)1 * n_nodes + tpos) * K + k];
                double d = 0;
#pragma unroll
                for (int b = 0; b <= P; ++b)
                  {
                    const long long id = horizontal ? (long long)(base + b) * g.nfx + s : (long long)s * g.nfx + base + b;
                    d += dn[b] * u[id];
                  }
                d /= hn;
                const long long il = horizontal ? (long long)line * g.nfx + s : (long long)s * g.nfx + line;
                tang += cC * u[il];
                norm += cM * d;
              }
            R[al] += fc.half_dt2 * en * (et * tang + enn * norm);
          }
      }
    if (fc.remove)
      {
        double flux = 0;
#pragma unroll
        for (int al = 0; al < NM; ++al)
          flux += R[al];
#pragma unroll
        for (int al = 0; al < NM; ++al)
          R[al] -= (c_W[al + 1] / (1. - c_W[0])) * flux;
      }
    const long long idx = (long long)j * g.nfx + i;
#pragma unroll
    for (int al = 0; al < NM; ++al)
      rhs[al * N + idx] += R[al];
  }

  // ------------------------------------------------------ mass matrix (K2)
  template <int P>
  constexpr size_t
  mass_smem()
  {
    using T = Tile<P>;
    return sizeof(double) * (4 * T::TX * T::K + 4 * T::TY * T::K + T::HN + T::HY * T::TX);
  }

  // y = M x for nsys vectors, the identity on images (MassOperator vmult).
  template <int P>
  __global__ void __launch_bounds__(THREADS)
    k_mass_vmult(const Geo geo, const double *__restrict__ x, double *__restrict__ y, int nsys)
  {
    using T = Tile<P>;
    constexpr int TX = T::TX, TY = T::TY, HX = T::HX, K = T::K;
    extern __shared__ double sm[];
    double *s_rx = sm, *s_ry = s_rx + 4 * TX * K, *s_u = s_ry + 4 * TY * K, *s_t = s_u + T::HN;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;
    load_rows<P>(s_rx, geo.rowx, gx0, TX, g.nfx);
    load_rows<P>(s_ry, geo.rowy, gy0, TY, g.nfy);
    for (int s = 0; s < nsys; ++s)
      {
        load_tile<P>(s_u, x + s * N, g, gx0, gy0);
        __syncthreads();
        xpass<P>(s_u, s_rx, s_t);
        __syncthreads();
        for (int t = threadIdx.x; t < TY * TX; t += blockDim.x)
          {
            const int lyo = t / TX, lxo = t - lyo * TX, gx = gx0 + lxo, gy = gy0 + lyo;
            if (gx >= g.nfx || gy >= g.nfy)
              continue;
            const long long idx = (long long)gy * g.nfx + gx;
            y[s * N + idx] = is_image(gx, gy, g) ? x[s * N + idx] : ypass_at<P>(s_t, s_ry, lyo, lxo);
          }
        __syncthreads();
      }
    (void)HX;
  }

  // ------------------------------------------- Jacobi-PCG, 8 systems at once (K3)
  // deal.II SolverCG (mass.h:204-211), one state per system.
  struct CgState
  {
    double tol[NM], rz[NM], rz_prev[NM], beta[NM], alpha[NM], res[NM];
    int it[NM], active[NM];
    int status, n_active;
    unsigned long long total_its;
  };

  // r = b - A xg with xg = extrapolate ? 2 x_cur - x_prev (written to x_new) : x_new;
  // partials per system: b.b, r.r, r.D^{-1}r.
  template <int P>
  __global__ void __launch_bounds__(THREADS)
    k_cg_start(const Geo geo, const double *__restrict__ b, const double *__restrict__ x_cur,
               const double *__restrict__ x_prev, double *__restrict__ x_new, double *__restrict__ r, int extrapolate,
               int nsys, double *__restrict__ partials)
  {
    using T = Tile<P>;
    constexpr int TX = T::TX, TY = T::TY, HX = T::HX, K = T::K;
    extern __shared__ double sm[];
    double *s_rx = sm, *s_ry = s_rx + 4 * TX * K, *s_u = s_ry + 4 * TY * K, *s_t = s_u + T::HN;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;
    load_rows<P>(s_rx, geo.rowx, gx0, TX, g.nfx);
    load_rows<P>(s_ry, geo.rowy, gy0, TY, g.nfy);
    double part[3 * NM];
#pragma unroll
    for (int q = 0; q < 3 * NM; ++q)
      part[q] = 0;
    for (int s = 0; s < nsys; ++s)
      {
        for (int t = threadIdx.x; t < T::HN; t += blockDim.x)
          {
            const int ly = t / HX, lx = t - ly * HX;
            const int sx = wrap(gx0 - P + lx, g.px, g.nux, g.nfx), sy = wrap(gy0 - P + ly, g.py, g.nuy, g.nfy);
            double v = 0;
            if (sx >= 0 && sy >= 0)
              {
                const long long id = s * N + (long long)sy * g.nfx + sx;
                v = extrapolate ? -x_prev[id] + 2. * x_cur[id] : x_new[id];
              }
            s_u[t] = v;
          }
        __syncthreads();
        xpass<P>(s_u, s_rx, s_t);
        __syncthreads();
        for (int t = threadIdx.x; t < TY * TX; t += blockDim.x)
          {
            const int lyo = t / TX, lxo = t - lyo * TX, gx = gx0 + lxo, gy = gy0 + lyo;
            if (gx >= g.nfx || gy >= g.nfy)
              continue;
            const long long id = s * N + (long long)gy * g.nfx + gx;
            double xg, Ax;
            if (is_image(gx, gy, g))
              {
                xg = extrapolate ? -x_prev[id] + 2. * x_cur[id] : x_new[id];
                Ax = xg;
              }
            else
              {
                xg = s_u[(lyo + P) * HX + lxo + P];
                Ax = ypass_at<P>(s_t, s_ry, lyo, lxo);
              }
            if (extrapolate)
              x_new[id] = xg;
            const double bb = b[id];
            const double rr = -Ax + bb;
            r[id] = rr;
            part[s] += bb * bb;
            part[NM + s] += rr * rr;
            part[2 * NM + s] += rr * (inv_jacobi(gx, gy, geo) * rr);
          }
        __syncthreads();
      }
    block_reduce_store<3 * NM>(part, 3 * NM, partials, blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y);
  }

  // p <- D^{-1} r + beta p (p <- D^{-1} r on the first iteration), v = A p; partials p.v.
  template <int P>
  __global__ void __launch_bounds__(THREADS)
    k_cg_pv(const Geo geo, const double *__restrict__ r, const double *__restrict__ p_in, double *__restrict__ p_out,
            double *__restrict__ v, const CgState *__restrict__ st, int nsys, double *__restrict__ partials)
  {
    using T = Tile<P>;
    constexpr int TX = T::TX, TY = T::TY, HX = T::HX, K = T::K;
    extern __shared__ double sm[];
    double *s_rx = sm, *s_ry = s_rx + 4 * TX * K, *s_u = s_ry + 4 * TY * K, *s_t = s_u + T::HN;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;
    load_rows<P>(s_rx, geo.rowx, gx0, TX, g.nfx);
    load_rows<P>(s_ry, geo.rowy, gy0, TY, g.nfy);
    double part[NM];
#pragma unroll
    for (int q = 0; q < NM; ++q)
      part[q] = 0;
    for (int s = 0; s < nsys; ++s)
      {
        if (!st->active[s])
          continue;
        const bool first = st->it[s] == 0;
        const double beta = st->beta[s];
        for (int t = threadIdx.x; t < T::HN; t += blockDim.x)
          {
            const int ly = t / HX, lx = t - ly * HX;
            const int sx = wrap(gx0 - P + lx, g.px, g.nux, g.nfx), sy = wrap(gy0 - P + ly, g.py, g.nuy, g.nfy);
            double val = 0;
            if (sx >= 0 && sy >= 0)
              {
                const long long id = s * N + (long long)sy * g.nfx + sx;
                const double z = inv_jacobi(sx, sy, geo) * r[id];
                val = first ? z : beta * p_in[id] + z;
              }
            s_u[t] = val;
          }
        __syncthreads();
        xpass<P>(s_u, s_rx, s_t);
        __syncthreads();
        for (int t = threadIdx.x; t < TY * TX; t += blockDim.x)
          {
            const int lyo = t / TX, lxo = t - lyo * TX, gx = gx0 + lxo, gy = gy0 + lyo;
            if (gx >= g.nfx || gy >= g.nfy)
              continue;
            const long long id = s * N + (long long)gy * g.nfx + gx;
            double pn, vn;
            if (is_image(gx, gy, g))
              {
                pn = first ? r[id] : beta * p_in[id] + r[id];
                vn = pn;
              }
            else
              {
                pn = s_u[(lyo + P) * HX + lxo + P];
                vn = ypass_at<P>(s_t, s_ry, lyo, lxo);
              }
            p_out[id] = pn;
            v[id] = vn;
            part[s] += pn * vn;
          }
        __syncthreads();
      }
    block_reduce_store<NM>(part, NM, partials, blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y);
  }

  // x += alpha p, r -= alpha v; partials r.r, r.D^{-1}r.
  __global__ void __launch_bounds__(THREADS)
    k_cg_update(const Geo geo, double *__restrict__ x, double *__restrict__ r, const double *__restrict__ p,
                const double *__restrict__ v, const CgState *__restrict__ st, int nsys, double *__restrict__ partials)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    double part[2 * NM];
#pragma unroll
    for (int q = 0; q < 2 * NM; ++q)
      part[q] = 0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x)
      {
        const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
        const double inv = inv_jacobi(i, j, geo);
        for (int s = 0; s < nsys; ++s)
          {
            if (!st->active[s])
              continue;
            const double al = st->alpha[s];
            const long long id = s * N + idx;
            x[id] += al * p[id];
            const double rr = r[id] + -al * v[id];
            r[id] = rr;
            part[s] += rr * rr;
            part[NM + s] += rr * (inv * rr);
          }
      }
    block_reduce_store<2 * NM>(part, 2 * NM, partials, blockIdx.x, gridDim.x);
  }

  // The scalar work of one CG phase, one thread per system, from the reduced sums.
  // phase 0 (after start): sums = [bb, rr, rz]; phase 1 (after pv): [pv];
  // phase 2 (after update): [rr, rz].
  __global__ void
  k_cg_scalars(CgState *st, const double *__restrict__ sums, int nsys, int phase, double cg_tol, int max_its)
  {
    const int s = threadIdx.x;
    if (s < NM)
      {
        if (phase == 0)
          {
            if (s < nsys)
              {
                st->tol[s] = cg_tol * sqrt(sums[s]);
                const double res = sqrt(sums[NM + s]);
                st->res[s] = res;
                st->rz[s] = sums[2 * NM + s];
                st->it[s] = 0;
                st->beta[s] = 0;
                if (isnan(res))
                  {
                    st->active[s] = 0;
                    atomicExch(&st->status, 3); // LBFEM_ERR_NONFINITE
                  }
                else
                  st->active[s] = res <= st->tol[s] ? 0 : 1;
              }
            else
              st->active[s] = 0;
          }
        else if (phase == 1)
          {
            if (s < nsys && st->active[s])
              st->alpha[s] = st->rz[s] / sums[s];
          }
        else if (s < nsys && st->active[s])
          {
            const int it = ++st->it[s];
            atomicAdd(&st->total_its, 1ULL);
            const double res = sqrt(sums[s]);
            st->res[s] = res;
            if (isnan(res))
              {
                st->active[s] = 0;
                atomicExch(&st->status, 3);
              }
            else if (res <= st->tol[s])
              st->active[s] = 0;
            else if (it >= max_its)
              {
                st->active[s] = 0;
                atomicCAS(&st->status, 0, 2); // LBFEM_ERR_NO_CONVERGENCE
              }
            else
              {
                st->rz_prev[s] = st->rz[s];
                st->rz[s] = sums[NM + s];
                st->beta[s] = st->rz[s] / st->rz_prev[s];
              }
          }
      }
    __syncthreads();
    if (threadIdx.x == 0)
      {
        int n = 0;
        for (int k = 0; k < NM; ++k)
          n += st->active[k];
        st->n_active = n;
      }
  }
} // namespace lbfem_gpu
