// The hot-path kernels: streaming right-hand side (K1), wall-face surface term,
// mass vmult and the Jacobi-PCG steps (K2/K3), lumped solve (K4) and the nodal
// maps of the schemes (K5/K6). FP64.
#pragma once

#include "kernels.cuh"

namespace lbfem_gpu
{
#define LBFEM_GRID_STRIDE(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

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
    LBFEM_GRID_STRIDE(i, N)
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
    LBFEM_GRID_STRIDE(i, N)
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
  k_predictor_corrector(const Geo geo, DevStats *__restrict__ ds, double *__restrict__ f, const double *__restrict__ feq,
                        const double *__restrict__ x, double theta)
  {
    if (step_skipped(ds))
      return;
    const long long N = geo.g.N;
    const double inv = 1. / (1. + theta);
    LBFEM_GRID_STRIDE(i, N)
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
    LBFEM_GRID_STRIDE(i, N)
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

  // ----- FP32 deviation forms of the nodal maps (mixed precision) -----
  __device__ __forceinline__ void
  collide_node_dev(float (&d)[Q], long long idx, const Geo &geo, float omega)
  {
    const MomF m = moments_dev(d);
    const MomF mt = impose(m, idx, geo);
#pragma unroll
    for (int a = 0; a < Q; ++a)
      d[a] = feqd_a(a, mt) + (1.f - omega) * (d[a] - feqd_a(a, m));
  }

  // FP64 moments / equilibrium of FP32 deviations (exact forms as above).
  __device__ __forceinline__ Mom
  moments_dev64(const double (&d)[Q], double &drho)
  {
    double dr = 0, mx = 0, my = 0;
#pragma unroll
    for (int a = 0; a < Q; ++a)
      {
        dr += d[a];
        mx += c_EX[a] * d[a];
        my += c_EY[a] * d[a];
      }
    drho = dr;
    const double rho = 1.0 + dr;
    return {rho, mx / rho, my / rho};
  }

  __device__ __forceinline__ double
  feqd64_a(int a, const Mom &m, double drho)
  {
    const double uu = m.ux * m.ux + m.uy * m.uy;
    const double eu = c_EX[a] * m.ux + c_EY[a] * m.uy;
    return c_W[a] * (drho + m.rho * (3. * eu + 4.5 * eu * eu - 1.5 * uu));
  }

  // predictor_corrector on FP32 deviations d = f - w with the FP32 increment x, in
  // FP32 arithmetic. The corrector's theta (feq(fhat) - feq(f)) is formed from the
  // moment changes of the predictor, exact in real arithmetic because feq(f) has
  // the moments of f (and its density at a wall): with inv = 1 / (1 + theta),
  //   rho_hat - rho = inv sum x,   J_hat - J = inv sum e x  (J = rho u; a wall
  //   node keeps its imposed u), so that
  //   feq_a(fhat) - feq_a(f) = w_a (d rho + 3 e.dJ + 4.5 d[(e.J)^2 / rho] - 1.5 d[J.J / rho]),
  // each difference written out in the small changes. No difference of two
  // O(1e-2) equilibria is rounded (the reason the corrector once ran in FP64).
  // Node i of the kernel below (also the body of its batched form).
  __device__ __forceinline__ void
  pc_dev_node(const Geo &geo, float *__restrict__ d, const float *__restrict__ x, float th, float inv, long long i)
  {
    const long long N = geo.g.N;
    {
      float di[Q], xa[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a)
        di[a] = d[a * N + i];
      xa[0] = 0.f;
#pragma unroll
      for (int a = 1; a < Q; ++a)
        xa[a] = x[(a - 1) * N + i];
      const int wk = geo.wall ? geo.wall[i] : 0;
      const MomF m = impose_class(moments_dev(di), wk, geo);
      float sx = 0.f, sjx = 0.f, sjy = 0.f;
#pragma unroll
      for (int a = 1; a < Q; ++a)
        {
          sx += xa[a];
          sjx += float(c_EX[a]) * xa[a];
          sjy += float(c_EY[a]) * xa[a];
        }
      const float dr = inv * sx;
      const float rho = m.rho, rh = rho + dr, den = 1.f / (rho * rh);
      const float Jx = rho * m.ux, Jy = rho * m.uy;
      const float djx = wk ? 0.f : inv * sjx, djy = wk ? 0.f : inv * sjy;
      // d[J.J / rho] and the wall's density-only change
      const float duu = ((2.f * (Jx * djx + Jy * djy) + djx * djx + djy * djy) * rho - (Jx * Jx + Jy * Jy) * dr) * den;
      const float uu = m.ux * m.ux + m.uy * m.uy;
#pragma unroll
      for (int a = 0; a < Q; ++a)
        {
          const float ex = float(c_EX[a]), ey = float(c_EY[a]);
          // fhat - d = inv (theta (feq - d) + x): the update is formed apart from d
          // and added to it once (as the FP64 form rounds once)
          const float up = inv * fmaf(th, feqd_a(a, m) - di[a], xa[a]);
          float dq;
          if (wk)
            {
              const float eu = ex * m.ux + ey * m.uy;
              dq = dr * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * uu);
            }
          else
            {
              const float eJ = ex * Jx + ey * Jy, edJ = ex * djx + ey * djy;
              const float de = (edJ * (2.f * eJ + edJ) * rho - eJ * eJ * dr) * den;
              dq = dr + 3.f * edJ + 4.5f * de - 1.5f * duu;
            }
          d[a * N + i] = di[a] + fmaf(th, wmul(kWf[a], kWlf[a], dq), up);
        }
    }
  }

  __global__ void __launch_bounds__(THREADS, 4)
  k_predictor_corrector_dev(const Geo geo, DevStats *__restrict__ ds, float *__restrict__ d,
                            const float *__restrict__ x, double theta)
  {
    if (step_skipped(ds))
      return;
    const float th = float(theta), inv = float(1. / (1. + theta));
    LBFEM_GRID_STRIDE(i, geo.g.N)
    pc_dev_node(geo, d, x, th, inv, i);
  }

  // Bardow's initial transform on deviations: d + scale (d - (feq - w)).
  __global__ void
  k_bardow_transform_dev(const Geo geo, float *__restrict__ d, float scale)
  {
    const long long N = geo.g.N;
    LBFEM_GRID_STRIDE(i, N)
    {
      float v[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a)
        v[a] = d[a * N + i];
      const MomF m = moments_dev(v);
#pragma unroll
      for (int a = 0; a < Q; ++a)
        d[a * N + i] = v[a] + scale * (v[a] - feqd_a(a, m));
    }
  }

  // FP64 populations <-> FP32 deviations from the rest state.
  __global__ void
  k_to_dev(const double *__restrict__ f, float *__restrict__ d, long long N)
  {
    LBFEM_GRID_STRIDE(i, N)
    {
#pragma unroll
      for (int a = 0; a < Q; ++a)
        d[a * N + i] = float(f[a * N + i] - c_W[a]);
    }
  }

  __global__ void
  k_from_dev(const float *__restrict__ d, double *__restrict__ f, long long N)
  {
    LBFEM_GRID_STRIDE(i, N)
    {
#pragma unroll
      for (int a = 0; a < Q; ++a)
        f[a * N + i] = c_W[a] + double(d[a * N + i]);
    }
  }

  // TaylorGalerkin::stream (streaming.h:94-98): f_a += x_{a-1}, a = 1..8.
  template <typename R>
  __global__ void
  k_add_increment(const Geo geo, DevStats *__restrict__ ds, R *__restrict__ f, const R *__restrict__ x,
                  int count_step)
  {
    if (step_skipped(ds, count_step != 0))
      return;
    const long long N = geo.g.N;
    LBFEM_GRID_STRIDE(i, N)
    {
#pragma unroll
      for (int a = 1; a < Q; ++a)
        f[a * N + i] += x[(a - 1) * N + i];
    }
  }

  // Lumped solve (mass.h:189-191): x = M_L^{-1} r, for nsys vectors.
  template <typename RI, typename RO>
  __global__ void
  k_lumped(const Geo geo, const RI *__restrict__ r, RO *__restrict__ x, int nsys)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    LBFEM_GRID_STRIDE(idx, N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      const RO inv = RO(is_image(i, j, g) ? 1.0 : geo.ilx[i] * geo.ily[j]);
      for (int s = 0; s < nsys; ++s)
        x[s * N + idx] = inv * RO(r[s * N + idx]);
    }
  }

  // Node weights: the lumped (which = 0) or Jacobi (which = 1) diagonal, images 1.
  __global__ void
  k_diagonal(const Geo geo, double *__restrict__ w, int which)
  {
    const Grid &g = geo.g;
    LBFEM_GRID_STRIDE(idx, g.N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      if (geo.lump2)
        w[idx] = which == 0 ? geo.lump2[idx] : 1.0 / geo.ijac2[idx]; // images: 1 in both
      else
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
    LBFEM_GRID_STRIDE(idx, N)
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

  // Moments of FP32 deviations, accumulated in FP64 (images report their source).
  __global__ void
  k_moments_dev(const Geo geo, const float *__restrict__ d, double *__restrict__ rho, double *__restrict__ ux,
                double *__restrict__ uy)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    LBFEM_GRID_STRIDE(idx, N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      const long long src = (long long)wrap(j, g.py, g.nuy, g.nfy) * g.nfx + wrap(i, g.px, g.nux, g.nfx);
      double dr = 0, mx = 0, my = 0;
#pragma unroll
      for (int a = 0; a < Q; ++a)
        {
          const double v = d[a * N + src];
          dr += v;
          mx += c_EX[a] * v;
          my += c_EY[a] * v;
        }
      const double r = 1.0 + dr;
      if (rho)
        rho[idx] = r;
      if (ux)
        ux[idx] = mx / r;
      if (uy)
        uy[idx] = my / r;
    }
  }

  // FP64 conservation sums over the independent nodes of FP32 deviations.
  __global__ void __launch_bounds__(THREADS)
    k_conservation_dev(const Geo geo, const float *__restrict__ d, double *__restrict__ partials)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    double s[5] = {0, 0, 0, 0, 0};
    LBFEM_GRID_STRIDE(idx, N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      if (is_image(i, j, g) || !owned_row(j, g))
        continue;
      double dr = 0, mx = 0, my = 0;
#pragma unroll
      for (int a = 0; a < Q; ++a)
        {
          const double v = d[a * N + idx];
          dr += v;
          mx += c_EX[a] * v;
          my += c_EY[a] * v;
        }
      const double rho = 1.0 + dr, ux = mx / rho, uy = my / rho;
      const double w = geo.lump2 ? geo.lump2[idx] : geo.lumpx[i] * geo.lumpy[j];
      s[0] += w;
      s[1] += w * rho;
      s[2] += w * mx;
      s[3] += w * my;
      s[4] += w * (ux * ux + uy * uy);
    }
    block_reduce_store<5>(s, partials, blockIdx.x, gridDim.x);
  }

  // FP64 conservation sums over the independent nodes (cgdbe.cc:353-368).
  __global__ void __launch_bounds__(THREADS)
    k_conservation(const Geo geo, const double *__restrict__ f, double *__restrict__ partials)
  {
    const Grid &g = geo.g;
    const long long N = g.N;
    double s[5] = {0, 0, 0, 0, 0};
    LBFEM_GRID_STRIDE(idx, N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      if (is_image(i, j, g) || !owned_row(j, g))
        continue;
      double v[Q];
#pragma unroll
      for (int a = 0; a < Q; ++a)
        v[a] = f[a * N + idx];
      const Mom m = moments(v);
      const double w = geo.lump2 ? geo.lump2[idx] : geo.lumpx[i] * geo.lumpy[j];
      s[0] += w;
      s[1] += w * m.rho;
      s[2] += w * m.rho * m.ux;
      s[3] += w * m.rho * m.uy;
      s[4] += w * (m.ux * m.ux + m.uy * m.uy);
    }
    block_reduce_store<5>(s, partials, blockIdx.x, gridDim.x);
  }

  // Caller numbering <-> structured numbering, nb blocks of a vector.
  __global__ void
  k_gather(const double *__restrict__ src, const long long *__restrict__ dof, double *__restrict__ dst, long long N,
           long long n_dofs, int nb)
  {
    LBFEM_GRID_STRIDE(s, N)
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
    LBFEM_GRID_STRIDE(s, N)
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
    // FP32 coefficients of the population pairs (a, a + 4), a = 1..4, rounded
    // once on the host: a, b, ex, c ex^2, ey, -2 c ex ey, c ey^2, c ex ey of
    // population a, and its weight
    float pk[4][8];
    float pw[4], pwl[4]; // and its rounding error (w = pw + pwl)
  };

  template <int MODE>
  __host__ __device__ constexpr bool
  has_moments()
  {
    return MODE == ADV_TG_COLLIDE || MODE == ADV_LEELIN_FUSED;
  }

  // Moment fields staged per footprint node: rho, ux, uy (+ drho for FP32 deviations).
  template <typename R>
  __host__ __device__ constexpr int
  n_moment_fields()
  {
    return sizeof(R) == sizeof(float) ? 4 : 3;
  }

  template <int P, int MODE, typename R = double>
  constexpr size_t
  advection_smem()
  {
    using T = Tile<P>;
    const int fields = (has_moments<MODE>() ? n_moment_fields<R>() : 0) + 1 + (MODE == ADV_LEELIN_FEQ ? 1 : 0);
    return sizeof(R) * (fields * T::NF + 3 * T::NY + 2 * T::TX) +
           (MODE == ADV_TG_COLLIDE ? size_t(T::NF + 15) / 16 * 16 : 0);
  }

  // Per-population scalars of the grouped operator
  //   r = My (x) Y1 + Cy (x) Y2' + Ky (x) Y3 + By (x) Y4, with h = a f + b feq:
  //   Y1 = ex Cx h + c ex^2 Kx f, Y2' = ey Mx h - 2 c ex ey Cx f + c ex ey Bx f,
  //   Y3 = c ey^2 Mx f, Y4 = c ex ey Cx f
  // (C^T = B - C, B the end-point term of the integration by parts).
  template <typename R>
  struct AdvK
  {
    R A, B, k1, k2, k3, k4, k5, k6;
  };

  // The equilibrium of population a at footprint index t from the staged moments.
  template <typename R>
  __device__ __forceinline__ R
  staged_feq(const R *s_m, int nf, int t, int a)
  {
    if constexpr (sizeof(R) == sizeof(float))
      return feqd_a(a, MomF{s_m[t], s_m[nf + t], s_m[2 * nf + t], s_m[3 * nf + t]});
    else
      return feq_a(a, Mom{s_m[t], s_m[nf + t], s_m[2 * nf + t]});
  }

  // Population a at footprint index t: u, and h = A u + B feq.
  template <int HM, typename R>
  __device__ __forceinline__ void
  load_uh(const R *s_u, const R *s_e, const R *s_m, int nf, int t, int a, const AdvK<R> &k, R &u, R &h)
  {
    u = s_u[t];
    if constexpr (HM == 0)
      h = k.A * u;
    else if constexpr (HM == 1)
      h = fma(k.B, staged_feq<R>(s_m, nf, t, a), k.A * u);
    else
      h = fma(k.B, s_e[t], k.A * u);
  }

  // x pass of K1 for one footprint row fy and one x segment. CLS: 0 e = (ex, 0), 1 e = (0, ey), 2 diagonal.
  template <int P, int CLS, int HM, typename R>
  __device__ __forceinline__ void
  adv_xpass(const R *s_u, const R *s_e, const R *s_m, R *s_y, R *s_y4, const TileMaps<P, R> &m, const AdvK<R> &k,
            int a, int fy, int seg, int gx0, int y4_slot, int bx_lo, int bx_hi)
  {
    using T = Tile<P>;
    constexpr bool XC = CLS != 1, YC = CLS != 0, DG = CLS == 2;
    const int base = fy * T::PF;
    const int q0 = seg * T::KX;
    R u[P + 1], h[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      load_uh<HM>(s_u, s_e, s_m, T::NF, base + q0 * P + b, a, k, u[b], h[b]);
    R pCh = 0, pKu = 0, pMh = 0, pCu = 0, pMu = 0;
    if constexpr (XC)
      {
        pCh = m.cx[q0] * elem_last<P, OP_C>(h);
        pKu = m.hxi[q0] * elem_last<P, OP_K>(u);
      }
    if constexpr (YC)
      {
        pMh = m.hx[q0] * elem_last<P, OP_M>(h);
        pMu = m.hx[q0] * elem_last<P, OP_M>(u);
      }
    if constexpr (DG)
      pCu = m.cx[q0] * elem_last<P, OP_C>(u);
    R *y1 = s_y + fy * T::PY, *y2 = y1 + T::NY, *y3 = y2 + T::NY;
#pragma unroll
    for (int q = 1; q <= T::KX; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
        h[0] = h[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          load_uh<HM>(s_u, s_e, s_m, T::NF, base + qc * P + b, a, k, u[b], h[b]);
        R eCh[P + 1], eKu[P + 1], eMh[P + 1], eCu[P + 1], eMu[P + 1];
        if constexpr (XC)
          {
            elem<P, OP_C>(h, eCh);
            elem<P, OP_K>(u, eKu);
          }
        if constexpr (YC)
          {
            elem<P, OP_M>(h, eMh);
            elem<P, OP_M>(u, eMu);
          }
        if constexpr (DG)
          elem<P, OP_C>(u, eCu);
        const R sc = m.cx[qc], sh = m.hx[qc], shi = m.hxi[qc];
        const int j0 = (qc - 1) * P;
#pragma unroll
        for (int aa = 0; aa < P; ++aa)
          {
            const int j = j0 + aa;
            R vCh = 0, vKu = 0, vMh = 0, vCu = 0, vMu = 0;
            if constexpr (XC)
              {
                vCh = sc * eCh[aa];
                vKu = shi * eKu[aa];
              }
            if constexpr (YC)
              {
                vMh = sh * eMh[aa];
                vMu = sh * eMu[aa];
              }
            if constexpr (DG)
              vCu = sc * eCu[aa];
            if (aa == 0)
              {
                vCh += pCh;
                vKu += pKu;
                vMh += pMh;
                vMu += pMu;
                vCu += pCu;
              }
            if constexpr (XC)
              y1[j] = k.k1 * vCh + k.k2 * vKu;
            if constexpr (YC)
              {
                R y = k.k3 * vMh;
                if constexpr (DG)
                  {
                    y = fma(k.k4, vCu, y);
                    if (aa == 0)
                      {
                        // Bx f = -f at the first node, +f at the last node of a non-periodic axis
                        const int gx = gx0 + j;
                        if (gx == bx_lo)
                          y = fma(-k.k6, u[0], y);
                        else if (gx == bx_hi)
                          y = fma(k.k6, u[0], y);
                      }
                  }
                y2[j] = y;
                y3[j] = k.k5 * vMu;
              }
            if constexpr (DG)
              if (y4_slot >= 0)
                s_y4[y4_slot * T::TX + j] = k.k6 * vCu;
          }
        if constexpr (XC)
          {
            pCh = sc * eCh[P];
            pKu = shi * eKu[P];
          }
        if constexpr (YC)
          {
            pMh = sh * eMh[P];
            pMu = sh * eMu[P];
          }
        if constexpr (DG)
          pCu = sc * eCu[P];
      }
  }

  // y pass of K1 on column j and y segment seg: emit(own row i, r).
  template <int P, int CLS, typename R, typename Emit>
  __device__ __forceinline__ void
  adv_ypass(const R *s_y, const R *s_y4, const TileMaps<P, R> &m, int j, int seg, int gy0, int by_lo, int by_hi,
            Emit &&emit)
  {
    using T = Tile<P>;
    constexpr bool XC = CLS != 1, YC = CLS != 0, DG = CLS == 2;
    const R *y1 = s_y, *y2 = s_y + T::NY, *y3 = s_y + 2 * T::NY;
    const int q0 = seg * T::KY;
    R v1[P + 1], v2[P + 1], v3[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      {
        const int t = (q0 * P + b) * T::PY + j;
        if constexpr (XC)
          v1[b] = y1[t];
        if constexpr (YC)
          {
            v2[b] = y2[t];
            v3[b] = y3[t];
          }
      }
    R pend = 0;
    if constexpr (XC)
      pend = m.hy[q0] * elem_last<P, OP_M>(v1);
    if constexpr (YC)
      pend += m.cy[q0] * elem_last<P, OP_C>(v2) + m.hyi[q0] * elem_last<P, OP_K>(v3);
#pragma unroll
    for (int q = 1; q <= T::KY; ++q)
      {
        const int qc = q0 + q;
        v1[0] = v1[P];
        v2[0] = v2[P];
        v3[0] = v3[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          {
            const int t = (qc * P + b) * T::PY + j;
            if constexpr (XC)
              v1[b] = y1[t];
            if constexpr (YC)
              {
                v2[b] = y2[t];
                v3[b] = y3[t];
              }
          }
        R e1[P + 1], e2[P + 1], e3[P + 1];
        if constexpr (XC)
          elem<P, OP_M>(v1, e1);
        if constexpr (YC)
          {
            elem<P, OP_C>(v2, e2);
            elem<P, OP_K>(v3, e3);
          }
        const R sh = m.hy[qc], sc = m.cy[qc], shi = m.hyi[qc];
        const int i0 = (qc - 1) * P;
#pragma unroll
        for (int aa = 0; aa <= P; ++aa)
          {
            R r = 0;
            if constexpr (XC)
              r = sh * e1[aa];
            if constexpr (YC)
              r += sc * e2[aa] + shi * e3[aa];
            if (aa == P)
              {
                pend = r;
                break;
              }
            if (aa == 0)
              r += pend;
            if constexpr (DG)
              {
                const int gy = gy0 + i0 + aa;
                if (gy == by_lo)
                  r -= s_y4[0 * T::TX + j];
                else if (gy == by_hi)
                  r += s_y4[1 * T::TX + j];
              }
            emit(i0 + aa, r);
          }
      }
  }

  // rhs_{a-1} <- r_a for a = 1..8: cell integrals of the point operations of
  // TaylorGalerkinAdvection (advection.h:228-239) / LeeLinAdvection
  // (advection.h:275-287), in the grouped tensor-product form above. Images get
  // 0 (constrained rows, as distribute_local_to_global leaves them).
  // R = double: populations f; R = float: deviations f - w (the operator
  // annihilates constants, and collide / feq are applied in deviation form).
  template <int P, int MODE, typename R>
  __global__ void __launch_bounds__(THREADS, 2)
    k_advection(const Geo geo, const DevStats *__restrict__ ds, const R *__restrict__ f, const R *__restrict__ feq,
                R *__restrict__ fout, R *__restrict__ rhs, const AdvCoef ac)
  {
    if (ds && ds->sticky)
      return; // a step after a failed solve: the populations must stay as they are
    using T = Tile<P>;
    constexpr bool MOM = has_moments<MODE>();
    constexpr bool DEV = sizeof(R) == sizeof(float);
    constexpr int NMF = n_moment_fields<R>();
    constexpr int HM = MODE == ADV_LEELIN_FUSED ? 1 : MODE == ADV_LEELIN_FEQ ? 2 : 0;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R *sm = reinterpret_cast<R *>(sm_raw);
    __shared__ TileMaps<P, R> maps;
    R *s_m = sm;                                                // [NMF][NF] moments (MOM modes)
    R *s_u = s_m + (MOM ? NMF * T::NF : 0);                     // [NF] the current population
    R *s_e = s_u + T::NF;                                       // [NF] its equilibrium (ADV_LEELIN_FEQ)
    R *s_y = s_e + (MODE == ADV_LEELIN_FEQ ? T::NF : 0);        // [3][NY] x-pass outputs
    R *s_y4 = s_y + 3 * T::NY;                                  // [2][TX] Y4 on the first / last domain row
    uint8_t *s_wall = reinterpret_cast<uint8_t *>(s_y4 + 2 * T::TX); // [NF] wall classes (ADV_TG_COLLIDE)
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = blockIdx.x * T::TX, gy0 = blockIdx.y * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    __syncthreads();

    if constexpr (MOM)
      {
        // two footprint nodes per iteration: 18 loads in flight per thread
        constexpr int NT = T::FY * T::FX;
        for (int t0 = threadIdx.x; t0 < NT; t0 += 2 * THREADS)
          {
            R v[2][Q];
            int idx[2];
            int wk[2];
#pragma unroll
            for (int h = 0; h < 2; ++h)
              {
                const int t = t0 + h * THREADS;
                idx[h] = -1;
                wk[h] = 0;
                if (t < NT)
                  {
                    const int fy = t / T::FX, fx = t - fy * T::FX;
                    const int r = maps.row[fy];
                    const int c = maps.col[fx];
                    if (r >= 0 && c >= 0)
                      idx[h] = r + c;
                  }
#pragma unroll
                for (int a = 0; a < Q; ++a)
                  v[h][a] = idx[h] >= 0 ? f[a * N + idx[h]] : R(0);
                if (idx[h] >= 0 && geo.wall)
                  wk[h] = geo.wall[idx[h]];
              }
#pragma unroll
            for (int h = 0; h < 2; ++h)
              {
                const int t = t0 + h * THREADS;
                if (t >= NT)
                  continue;
                const int fy = t / T::FX, fx = t - fy * T::FX, st = fy * T::PF + fx;
                if (idx[h] < 0)
                  {
#pragma unroll
                    for (int q = 0; q < NMF; ++q)
                      s_m[q * T::NF + st] = R(0);
                    if constexpr (MODE == ADV_TG_COLLIDE)
                      s_wall[st] = 0;
                    continue;
                  }
                if constexpr (DEV)
                  {
                    MomF mo = moments_dev(v[h]);
                    if constexpr (MODE == ADV_LEELIN_FUSED)
                      mo = impose_class(mo, wk[h], geo);
                    s_m[st] = mo.rho;
                    s_m[T::NF + st] = mo.ux;
                    s_m[2 * T::NF + st] = mo.uy;
                    s_m[3 * T::NF + st] = mo.drho;
                  }
                else
                  {
                    Mom mo = moments(v[h]);
                    if constexpr (MODE == ADV_LEELIN_FUSED)
                      mo = impose_class(mo, wk[h], geo);
                    s_m[st] = mo.rho;
                    s_m[T::NF + st] = mo.ux;
                    s_m[2 * T::NF + st] = mo.uy;
                  }
                if constexpr (MODE == ADV_TG_COLLIDE)
                  s_wall[st] = uint8_t(wk[h]);
              }
          }
      }

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int bx_lo = g.px ? -1 : 0, bx_hi = g.px ? -1 : g.nfx - 1;
    const int by_lo = g.py ? -1 : 0, by_hi = g.py ? -1 : g.nfy - 1;
    const R omega = R(ac.omega);

    for (int a = (MODE == ADV_TG_COLLIDE ? 0 : 1); a < Q; ++a)
      {
        __syncthreads(); // the previous population's passes are done with s_u / s_y
        stage<P>(s_u, maps, [&](long long idx) { return f[a * N + idx]; });
        if constexpr (MODE == ADV_LEELIN_FEQ)
          stage<P>(s_e, maps, [&](long long idx) { return feq[a * N + idx]; });
        if constexpr (MODE == ADV_TG_COLLIDE)
          {
            __syncthreads();
            for (int t = threadIdx.x; t < T::FY * T::FX; t += blockDim.x)
              {
                const int fy = t / T::FX, fx = t - fy * T::FX, st = fy * T::PF + fx;
                const int r = maps.row[fy];
                const int c = maps.col[fx];
                if (r < 0 || c < 0)
                  continue;
                R gs;
                if constexpr (DEV)
                  {
                    const MomF mo{s_m[st], s_m[T::NF + st], s_m[2 * T::NF + st], s_m[3 * T::NF + st]};
                    const MomF mt = impose_class(mo, s_wall[st], geo);
                    gs = feqd_a(a, mt) + (1.f - omega) * (s_u[st] - feqd_a(a, mo));
                  }
                else
                  {
                    const Mom mo{s_m[st], s_m[T::NF + st], s_m[2 * T::NF + st]};
                    const Mom mt = impose_class(mo, s_wall[st], geo);
                    gs = feq_a(a, mt) + (1. - omega) * (s_u[st] - feq_a(a, mo));
                  }
                s_u[st] = gs;
                const int gx = gx0 - P + fx, gy = gy0 - P + fy;
                if (fx >= P && fx < P + T::TX && fy >= P && fy < P + T::TY && gx < g.nfx && gy < g.nfy &&
                    !is_image(gx, gy, g))
                  fout[a * N + r + c] = gs;
              }
            if (a == 0)
              continue;
          }
        __syncthreads();
        const int al = a - 1;
        const double ex = ac.ex[al], ey = ac.ey[al];
        const int cls = ey == 0.0 ? (ex == 0.0 ? 3 : 0) : (ex == 0.0 ? 1 : 2);
        const AdvK<R> k{R(ac.a),
                        R(ac.b),
                        R(ex),
                        R(ac.c * ex * ex),
                        R(ey),
                        R(-2.0 * ac.c * ex * ey),
                        R(ac.c * ey * ey),
                        R(ac.c * ex * ey)};
        // x pass: lane = footprint row, warp = x segment
        if (warp < T::NSX && lane < T::FY)
          {
            const int gy = gy0 - P + lane;
            const int y4_slot = gy == by_lo ? 0 : gy == by_hi ? 1 : -1;
            if (cls == 0)
              adv_xpass<P, 0, HM>(s_u, s_e, s_m, s_y, s_y4, maps, k, a, lane, warp, gx0, y4_slot, bx_lo, bx_hi);
            else if (cls == 1)
              adv_xpass<P, 1, HM>(s_u, s_e, s_m, s_y, s_y4, maps, k, a, lane, warp, gx0, y4_slot, bx_lo, bx_hi);
            else if (cls == 2)
              adv_xpass<P, 2, HM>(s_u, s_e, s_m, s_y, s_y4, maps, k, a, lane, warp, gx0, y4_slot, bx_lo, bx_hi);
          }
        __syncthreads();
        // y pass: lane group = columns, warp group = y segment
        const int j = threadIdx.x % T::YL, seg = threadIdx.x / T::YL;
        if (j < T::TX && seg < T::NSY)
          {
            const int gx = gx0 + j;
            R *out = rhs + (long long)al * N;
            auto emit = [&](int i, R r) {
              const int gy = gy0 + i;
              if (gx < g.nfx && gy < g.nfy)
                out[(long long)gy * g.nfx + gx] = is_image(gx, gy, g) ? R(0) : r;
            };
            if (cls == 0)
              adv_ypass<P, 0>(s_y, s_y4, maps, j, seg, gy0, by_lo, by_hi, emit);
            else if (cls == 1)
              adv_ypass<P, 1>(s_y, s_y4, maps, j, seg, gy0, by_lo, by_hi, emit);
            else if (cls == 2)
              adv_ypass<P, 2>(s_y, s_y4, maps, j, seg, gy0, by_lo, by_hi, emit);
            else
              for (int i = seg * T::SY; i < (seg + 1) * T::SY; ++i)
                emit(i, R(0));
          }
      }

    if constexpr (MODE == ADV_TG_COLLIDE)
      {
        // the images collide their own (stale) populations, as the nodal map does
        for (int t = threadIdx.x; t < T::TY * T::TX; t += blockDim.x)
          {
            const int i = t / T::TX, j = t - i * T::TX;
            const int gx = gx0 + j, gy = gy0 + i;
            if (gx >= g.nfx || gy >= g.nfy || !is_image(gx, gy, g))
              continue;
            const long long idx = (long long)gy * g.nfx + gx;
            R v[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a)
              v[a] = f[a * N + idx];
            if constexpr (DEV)
              collide_node_dev(v, idx, geo, omega);
            else
              collide_node(v, idx, geo, omega);
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
  // boundary nodes of the non-periodic sides; 8 threads per boundary node, one per
  // moving population (bnode = (i, j, side mask: 1 bottom, 2 top, 4 left, 8 right)).
  template <int P, typename R>
  __global__ void
  k_wall_faces(const Geo geo, const R *__restrict__ f, R *__restrict__ rhs, const int4 *__restrict__ bnode,
               int n_bnodes, const FaceCoef fc);

  // Boundary node t, population al + 1, of the kernel below (also the body of its
  // batched form): 8 consecutive lanes take the 8 moving populations of one node,
  // and every lane of the warp calls it (valid: the lane has a node). Each
  // population's sum over the node's sides is that of the reference's loop; the
  // mass-flux removal sums the 8 populations' terms in the order al = 0..7 on
  // every lane of the group.
  template <int P, typename R>
  __device__ __forceinline__ void
  wall_face_pop(const Geo &geo, const R *__restrict__ f, R *__restrict__ rhs, const int4 *__restrict__ bnode,
                const FaceCoef &fc, int t, int al, bool valid)
  {
    constexpr int K = 2 * P + 1;
    const Grid &g = geo.g;
    const long long N = g.N;
    double Rs = 0;
    int i = 0, j = 0;
    if (valid)
      {
        const int4 bn = bnode[t];
        i = bn.x;
        j = bn.y;
        const int sides = bn.z;
        const double ex = fc.ex[al], ey = fc.ey[al];
        const R *u = f + (long long)(al + 1) * N;
        for (int side = 0; side < 4; ++side)
          {
            if (!(sides & (1 << side)))
              continue;
            const double en = side == 0 ? -ey : side == 1 ? ey : side == 2 ? -ex : ex;
            if (en == 0.0)
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
            const double et = horizontal ? ex : ey;  // tangential component
            const double enn = horizontal ? ey : ex; // normal component (derivative direction)
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
                for (int bb = 0; bb <= P; ++bb)
                  {
                    const long long id =
                      horizontal ? (long long)(base + bb) * g.nfx + s : (long long)s * g.nfx + base + bb;
                    d += dn[bb] * u[id];
                  }
                d /= hn;
                const long long il = horizontal ? (long long)line * g.nfx + s : (long long)s * g.nfx + line;
                tang += cC * u[il];
                norm += cM * d;
              }
            Rs += fc.half_dt2 * en * (et * tang + enn * norm);
          }
      }
    if (fc.remove)
      {
        const int lane0 = (threadIdx.x & 31) & ~7;
        double flux = 0;
#pragma unroll
        for (int a = 0; a < NM; ++a)
          flux += __shfl_sync(0xffffffffu, Rs, lane0 + a);
        Rs -= (c_W[al + 1] / (1. - c_W[0])) * flux;
      }
    if (valid)
      {
        const long long idx = (long long)j * g.nfx + i;
        rhs[al * N + idx] = R(double(rhs[al * N + idx]) + Rs);
      }
  }

  // blockDim a multiple of 32: thread 8 t + al takes node t, population al + 1
  template <int P, typename R>
  __global__ void
  k_wall_faces(const Geo geo, const R *__restrict__ f, R *__restrict__ rhs, const int4 *__restrict__ bnode,
               int n_bnodes, const FaceCoef fc)
  {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    wall_face_pop<P, R>(geo, f, rhs, bnode, fc, q >> 3, q & 7, (q >> 3) < n_bnodes);
  }

  // ------------------------------------------------------ mass matrix (K2)
  // staged footprint + x-pass output + `own` own-node vectors
  template <int P>
  constexpr size_t
  mass_smem(int own = 0)
  {
    using T = Tile<P>;
    return sizeof(double) * (T::NF + T::NY + own * T::TX * T::TY);
  }

  // The mass operator My (x) Mx of the staged field s_u for every own node of the
  // tile: emit(i, j, storage index, image, Au); images get the identity row. The
  // storage index is 32-bit: a population array holds fewer than 2^31 nodes.
  template <int P, typename R, typename Emit>
  __device__ __forceinline__ void
  mass_apply(const R *s_u, R *s_t, const TileMaps<P, R> &m, const Grid &g, int gx0, int gy0, Emit &&emit)
  {
    using T = Tile<P>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < T::NSX && lane < T::FY)
      mass_xpass<P>(s_u, s_t, m, lane, warp);
    __syncthreads();
    const int j = threadIdx.x % T::YL, seg = threadIdx.x / T::YL;
    if (j < T::TX && seg < T::NSY)
      {
        const int gx = gx0 + j;
        mass_ypass<P>(s_t, m, j, seg, [&](int i, R v) {
          const int gy = gy0 + i;
          if (gx < g.nfx && gy < g.nfy)
            emit(i, j, gy * g.nfx + gx, is_image(gx, gy, g), v);
        });
      }
  }

  // y = M x for nsys vectors, the identity on images (MassOperator vmult).
  template <int P>
  __global__ void __launch_bounds__(THREADS)
    k_mass_vmult(const Geo geo, const double *__restrict__ x, double *__restrict__ y, int nsys)
  {
    using T = Tile<P>;
    extern __shared__ double sm[];
    __shared__ TileMaps<P, double> maps;
    double *s_u = sm, *s_t = sm + T::NF;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = blockIdx.x * T::TX, gy0 = blockIdx.y * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    __syncthreads();
    for (int s = 0; s < nsys; ++s)
      {
        const double *xs = x + s * N;
        stage<P>(s_u, maps, [&](long long idx) { return xs[idx]; });
        __syncthreads();
        mass_apply<P>(s_u, s_t, maps, g, gx0, gy0, [&](int, int, int idx, bool image, double v) {
          y[s * N + idx] = image ? xs[idx] : v;
        });
        __syncthreads();
      }
  }

  // ------------------------------------------ TG3 streaming matrix (K2, TG3)
  // The matrix of a TG3 streaming solve, A = M + c K_e with
  // K_e = int (e.grad N)(e.grad N^T) (StreamingMatrix, mass.h:57-129), per
  // system: kxx = c ex^2, kyy = c ey^2, kxy = c ex ey (all 0: A = M). In the
  // grouped tensor-product form of the flux term of the advection operator,
  //   A = My (x) Z1 + Cy (x) Z2 + Ky (x) Z3 + By (x) Z4,
  //   Z1 = Mx + kxx Kx, Z2 = kxy (Bx - 2 Cx), Z3 = kyy Mx, Z4 = kxy Cx
  // (C^T = B - C, B the end-point term). An axis-parallel e (kxy = 0, one of
  // kxx, kyy 0) makes it the product (My + kyy Ky) (x) (Mx + kxx Kx).
  struct StreamCoef
  {
    double kxx[NM], kyy[NM], kxy[NM];
  };

  // Scratch of the TG3 apply beyond the staged field: three x-pass output
  // arrays and Z4 on the first / last domain row (elements of R).
  template <int P>
  __host__ __device__ constexpr int
  tg3_scratch()
  {
    return 3 * Tile<P>::NY + 2 * Tile<P>::TX;
  }

  // x pass of the product form: out = (Mx + kxx Kx) s on one footprint row / x segment.
  template <int P, typename R>
  __device__ __forceinline__ void
  sep_xpass(const R *__restrict__ s, R *__restrict__ out, const TileMaps<P, R> &m, int fy, int seg, R kxx)
  {
    using T = Tile<P>;
    const R *row = s + fy * T::PF;
    R *orow = out + fy * T::PY;
    const int q0 = seg * T::KX;
    R u[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      u[b] = row[q0 * P + b];
    R pend = fma(kxx * m.hxi[q0], elem_last<P, OP_K>(u), m.hx[q0] * elem_last<P, OP_M>(u));
#pragma unroll
    for (int q = 1; q <= T::KX; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          u[b] = row[qc * P + b];
        R yM[P + 1], yK[P + 1];
        elem<P, OP_M>(u, yM);
        elem<P, OP_K>(u, yK);
        const R sm = m.hx[qc], sk = kxx * m.hxi[qc];
        const int j0 = (qc - 1) * P;
        orow[j0] = fma(sk, yK[0], fma(sm, yM[0], pend));
#pragma unroll
        for (int a = 1; a < P; ++a)
          orow[j0 + a] = fma(sk, yK[a], sm * yM[a]);
        pend = fma(sk, yK[P], sm * yM[P]);
      }
  }

  // y pass of the product form: (My + kyy Ky) t on column j / y segment seg, emit(own row i, value).
  template <int P, typename R, typename Emit>
  __device__ __forceinline__ void
  sep_ypass(const R *__restrict__ t, const TileMaps<P, R> &m, int j, int seg, R kyy, Emit &&emit)
  {
    using T = Tile<P>;
    const int q0 = seg * T::KY;
    R u[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      u[b] = t[(q0 * P + b) * T::PY + j];
    R pend = fma(kyy * m.hyi[q0], elem_last<P, OP_K>(u), m.hy[q0] * elem_last<P, OP_M>(u));
#pragma unroll
    for (int q = 1; q <= T::KY; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          u[b] = t[(qc * P + b) * T::PY + j];
        R yM[P + 1], yK[P + 1];
        elem<P, OP_M>(u, yM);
        elem<P, OP_K>(u, yK);
        const R sm = m.hy[qc], sk = kyy * m.hyi[qc];
        const int i0 = (qc - 1) * P;
        emit(i0, fma(sk, yK[0], fma(sm, yM[0], pend)));
#pragma unroll
        for (int a = 1; a < P; ++a)
          emit(i0 + a, fma(sk, yK[a], sm * yM[a]));
        pend = fma(sk, yK[P], sm * yM[P]);
      }
  }

  // x pass of the general form on one footprint row / x segment (Z1 with wm Mx in
  // place of Mx, so that wm = 0 gives the Laplace operator): Z1, Z2, Z3 into
  // s_y (three arrays of NY), Z4 into s_y4[slot] when the row is the first
  // (slot 0) or last (slot 1) row of a non-periodic y axis.
  template <int P, typename R>
  __device__ __forceinline__ void
  full_xpass(const R *__restrict__ s, R *__restrict__ s_y, R *__restrict__ s_y4, const TileMaps<P, R> &m, int fy,
             int seg, R wm, R kxx, R kyy, R kxy, int gx0, int y4_slot, int bx_lo, int bx_hi)
  {
    using T = Tile<P>;
    const R *row = s + fy * T::PF;
    R *y1 = s_y + fy * T::PY, *y2 = y1 + T::NY, *y3 = y2 + T::NY;
    const int q0 = seg * T::KX;
    R u[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      u[b] = row[q0 * P + b];
    R pM = m.hx[q0] * elem_last<P, OP_M>(u), pK = m.hxi[q0] * elem_last<P, OP_K>(u),
      pC = m.cx[q0] * elem_last<P, OP_C>(u);
#pragma unroll
    for (int q = 1; q <= T::KX; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          u[b] = row[qc * P + b];
        R eM[P + 1], eK[P + 1], eC[P + 1];
        elem<P, OP_M>(u, eM);
        elem<P, OP_K>(u, eK);
        elem<P, OP_C>(u, eC);
        const R sh = m.hx[qc], shi = m.hxi[qc], sc = m.cx[qc];
        const int j0 = (qc - 1) * P;
#pragma unroll
        for (int aa = 0; aa < P; ++aa)
          {
            const int j = j0 + aa;
            R vM = sh * eM[aa], vK = shi * eK[aa], vC = sc * eC[aa];
            if (aa == 0)
              {
                vM += pM;
                vK += pK;
                vC += pC;
              }
            R z2 = R(-2) * kxy * vC;
            if (aa == 0)
              {
                // Bx u = -u at the first node, +u at the last node of a non-periodic x axis
                const int gx = gx0 + j;
                if (gx == bx_lo)
                  z2 = fma(-kxy, u[0], z2);
                else if (gx == bx_hi)
                  z2 = fma(kxy, u[0], z2);
              }
            y1[j] = fma(kxx, vK, wm * vM);
            y2[j] = z2;
            y3[j] = kyy * vM;
            if (y4_slot >= 0)
              s_y4[y4_slot * T::TX + j] = kxy * vC;
          }
        pM = sh * eM[P];
        pK = shi * eK[P];
        pC = sc * eC[P];
      }
  }

  // y pass of the general form on column j / y segment seg: emit(own row i, value).
  template <int P, typename R, typename Emit>
  __device__ __forceinline__ void
  full_ypass(const R *__restrict__ s_y, const R *__restrict__ s_y4, const TileMaps<P, R> &m, int j, int seg, int gy0,
             int by_lo, int by_hi, Emit &&emit)
  {
    using T = Tile<P>;
    const R *y1 = s_y, *y2 = s_y + T::NY, *y3 = s_y + 2 * T::NY;
    const int q0 = seg * T::KY;
    R v1[P + 1], v2[P + 1], v3[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      {
        const int t = (q0 * P + b) * T::PY + j;
        v1[b] = y1[t];
        v2[b] = y2[t];
        v3[b] = y3[t];
      }
    R pend = m.hy[q0] * elem_last<P, OP_M>(v1) + m.cy[q0] * elem_last<P, OP_C>(v2) +
             m.hyi[q0] * elem_last<P, OP_K>(v3);
#pragma unroll
    for (int q = 1; q <= T::KY; ++q)
      {
        const int qc = q0 + q;
        v1[0] = v1[P];
        v2[0] = v2[P];
        v3[0] = v3[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          {
            const int t = (qc * P + b) * T::PY + j;
            v1[b] = y1[t];
            v2[b] = y2[t];
            v3[b] = y3[t];
          }
        R e1[P + 1], e2[P + 1], e3[P + 1];
        elem<P, OP_M>(v1, e1);
        elem<P, OP_C>(v2, e2);
        elem<P, OP_K>(v3, e3);
        const R sh = m.hy[qc], sc = m.cy[qc], shi = m.hyi[qc];
        const int i0 = (qc - 1) * P;
#pragma unroll
        for (int aa = 0; aa <= P; ++aa)
          {
            R r = sh * e1[aa] + sc * e2[aa] + shi * e3[aa];
            if (aa == P)
              {
                pend = r;
                break;
              }
            if (aa == 0)
              r += pend;
            const int gy = gy0 + i0 + aa;
            if (gy == by_lo)
              r -= s_y4[j];
            else if (gy == by_hi)
              r += s_y4[T::TX + j];
            emit(i0 + aa, r);
          }
      }
  }

  // Whether node (i, j) lies on a side of the box (psi = 0 there, periodic sides included).
  __device__ __forceinline__ bool
  on_box_side(int i, int j, const Grid &g)
  {
    return i == 0 || j == 0 || i == g.nfx - 1 || j == g.nfy - 1;
  }

  // A u for every own node of the tile, A = wm M + (the K_e part of kxx, kyy, kxy),
  // u staged in s_u; s_t holds tg3_scratch<P>() elements. emit(i, j, storage index,
  // fixed, Au) as mass_apply: a fixed row (a periodic image; with DIRICHLET also a
  // node on a side of the box) is the identity row.
  template <int P, bool DIRICHLET, typename R, typename Emit>
  __device__ __forceinline__ void
  tg3_apply(const R *s_u, R *s_t, const TileMaps<P, R> &m, const Grid &g, int gx0, int gy0, R wm, R kxx, R kyy,
            R kxy, Emit &&emit)
  {
    using T = Tile<P>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the product form needs wm = 1 and an axis-parallel e
    const bool sep = wm == R(1) && kxy == R(0) && (kxx == R(0) || kyy == R(0));
    R *s_y4 = s_t + 3 * T::NY;
    if (warp < T::NSX && lane < T::FY)
      {
        if (sep)
          sep_xpass<P>(s_u, s_t, m, lane, warp, kxx);
        else
          {
            const int gy = gy0 - P + lane;
            const int y4_slot = g.py ? -1 : gy == 0 ? 0 : gy == g.nfy - 1 ? 1 : -1;
            full_xpass<P>(s_u, s_t, s_y4, m, lane, warp, wm, kxx, kyy, kxy, gx0, y4_slot, g.px ? -1 : 0,
                          g.px ? -1 : g.nfx - 1);
          }
      }
    __syncthreads();
    const int j = threadIdx.x % T::YL, seg = threadIdx.x / T::YL;
    if (j < T::TX && seg < T::NSY)
      {
        const int gx = gx0 + j;
        auto out = [&](int i, R v) {
          const int gy = gy0 + i;
          if (gx < g.nfx && gy < g.nfy)
            emit(i, j, gy * g.nfx + gx, DIRICHLET ? on_box_side(gx, gy, g) : is_image(gx, gy, g), v);
        };
        if (sep)
          sep_ypass<P>(s_t, m, j, seg, kyy, out);
        else
          full_ypass<P>(s_t, s_y4, m, j, seg, gy0, g.py ? -1 : 0, g.py ? -1 : g.nfy - 1, out);
      }
  }

  // The operators of the CG kernels.
  enum
  {
    OPK_MASS = 0,   // M (MassOperator)
    OPK_TG3 = 1,    // M + c K_e of system s (StreamingMatrix)
    OPK_LAPLACE = 2 // K with zero rows on the sides of the box (the stream function, io.h:31-95)
  };

  template <int P, int OPK, typename R, typename Emit>
  __device__ __forceinline__ void
  op_apply(const R *s_u, R *s_t, const TileMaps<P, R> &m, const Grid &g, int gx0, int gy0, const StreamCoef &sc,
           int s, Emit &&emit)
  {
    if constexpr (OPK == OPK_TG3)
      tg3_apply<P, false>(s_u, s_t, m, g, gx0, gy0, R(1), R(sc.kxx[s]), R(sc.kyy[s]), R(sc.kxy[s]), emit);
    else if constexpr (OPK == OPK_LAPLACE)
      tg3_apply<P, true>(s_u, s_t, m, g, gx0, gy0, R(0), R(1), R(1), R(0), emit);
    else
      mass_apply<P>(s_u, s_t, m, g, gx0, gy0, emit);
  }

  // Elements of the x-pass scratch of a CG kernel.
  template <int P, int OPK>
  __host__ __device__ constexpr int
  op_scratch()
  {
    return OPK == OPK_MASS ? Tile<P>::NY : tg3_scratch<P>();
  }

  // The inverse Jacobi diagonal of the Laplace operator at storage node (c, r):
  // diag(My (x) Kx + Ky (x) Mx) from the assembled 1-D rows; 1 on the fixed nodes.
  template <int P>
  __device__ __forceinline__ double
  laplace_inv_diag(const Geo &geo, int c, int r)
  {
    constexpr int K = 2 * P + 1;
    const Grid &g = geo.g;
    if (on_box_side(c, r, g))
      return 1.0;
    const long long nx = g.nfx, ny = g.nfy;
    const double mx = geo.rowx[(0 * nx + c) * K + P], kx = geo.rowx[(3 * nx + c) * K + P];
    const double my = geo.rowy[(0 * ny + r) * K + P], ky = geo.rowy[(3 * ny + r) * K + P];
    return 1.0 / (my * kx + ky * mx);
  }

  // The right-hand side of the stream function (io.h:64-88): b = (dphi/dx, v) -
  // (dphi/dy, u) = (My (x) Cx^T) v - (Cy^T (x) Mx) u from the assembled 1-D rows,
  // 0 on the sides of the box. One thread per node.
  template <int P>
  __global__ void
  k_psi_rhs(const Geo geo, const double *__restrict__ u, const double *__restrict__ v, double *__restrict__ b)
  {
    constexpr int K = 2 * P + 1;
    const Grid &g = geo.g;
    const long long nx = g.nfx, ny = g.nfy;
    LBFEM_GRID_STRIDE(idx, g.N)
    {
      const int j = int(idx / g.nfx), i = int(idx - (long long)j * g.nfx);
      double s = 0;
      if (!on_box_side(i, j, g))
        for (int k = 0; k < K; ++k)
          {
            const int r = wrap(j + k - P, g.py, g.nuy, g.nfy);
            if (r < 0)
              continue;
            const double my = geo.rowy[(0 * ny + j) * K + k], cyt = geo.rowy[(2 * ny + j) * K + k];
            double sv = 0, su = 0;
            for (int l = 0; l < K; ++l)
              {
                const int c = wrap(i + l - P, g.px, g.nux, g.nfx);
                if (c < 0)
                  continue;
                const long long id = (long long)r * g.nfx + c;
                sv = fma(geo.rowx[(2 * nx + i) * K + l], v[id], sv);
                su = fma(geo.rowx[(0 * nx + i) * K + l], u[id], su);
              }
            s += my * sv - cyt * su;
          }
      b[idx] = s;
    }
  }

  // ---------------------------------------- iterated lumping (Richardson)
  // One Richardson pass of MassSolver::solve with Mass::richardson (mass.h:193-202):
  // x_out = x_in + M_L^{-1} (b - M x_in) for nsys systems (grid.z), constrained
  // rows the identity. x_in is read with a halo, so x_out is another buffer.
  template <int P, typename R>
  __global__ void __launch_bounds__(THREADS)
    k_richardson_pass(const Geo geo, const R *__restrict__ b, const R *__restrict__ x_in, R *__restrict__ x_out)
  {
    using T = Tile<P>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R *s_u = reinterpret_cast<R *>(sm_raw), *s_t = s_u + T::NF;
    __shared__ TileMaps<P, R> maps;
    const Grid &g = geo.g;
    const long long o = (long long)blockIdx.z * g.N;
    const int gx0 = blockIdx.x * T::TX, gy0 = blockIdx.y * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    __syncthreads();
    const R *xs = x_in + o, *bs = b + o;
    R *xo = x_out + o;
    stage<P>(s_u, maps, [&](long long idx) { return xs[idx]; });
    __syncthreads();
    mass_apply<P>(s_u, s_t, maps, g, gx0, gy0, [&](int i, int j, int idx, bool image, R Ax) {
      const R xv = image ? xs[idx] : s_u[(i + P) * T::PF + j + P];
      if (image)
        Ax = xv;
      const int gx = gx0 + j, gy = gy0 + i;
      const R inv = R(image ? 1.0 : geo.ilx[gx] * geo.ily[gy]);
      xo[idx] = xv + inv * (bs[idx] - Ax);
    });
  }

  // ------------------------------------------- Jacobi-PCG, 8 systems at once (K3)
  // deal.II SolverCG (mass.h:204-211), one state per system. With mixed
  // precision the vectors are FP32, the inner iterations run in FP32 with FP64
  // dot products, and each solve restarts from a true residual computed in
  // FP64 (iterative refinement) until the outer tolerance holds.
  struct CgState
  {
    double tol[NM], rz[NM], rz_prev[NM], beta[NM], alpha[NM], res[NM];
    int it[NM], its_total[NM], active[NM];
    int zero[NM]; // the system's right-hand side is exactly zero: its solution is 0 (k_zero_flagged)
    int status, n_active, iter;
    unsigned long long total_its;
  };

  // x_s <- 0 for the systems whose right-hand side is exactly zero. deal.II's
  // SolverCG would iterate from a nonzero (extrapolated) start toward the
  // tolerance cg_tol |b| = 0, which it cannot meet, and throw NoConvergence at
  // the cap; the exact solution 0 is returned instead, with no iterations.
  template <typename R>
  __global__ void
  k_zero_flagged(R *__restrict__ x, const CgState *__restrict__ st, long long N, int nsys)
  {
    const int s = blockIdx.y;
    if (s >= nsys || !st->zero[s])
      return;
    R *xs = x + s * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      xs[i] = R(0);
  }

  __device__ __forceinline__ double
  inv_jacobi_at(const Geo &geo, int i, int j)
  {
    return is_image(i, j, geo.g) ? 1.0 : geo.ijx[i] * geo.ijy[j];
  }

  // The inverse Jacobi diagonal at own node (i, j) of a tile, from its maps.
  template <int P, typename RM>
  __device__ __forceinline__ double
  own_inv_jacobi(const TileMaps<P, RM> &m, int i, int j, bool image)
  {
    return image ? 1.0 : m.ijx[j + P] * m.ijy[i + P];
  }

  // The same for the operator of a CG kernel: the mass diagonal (M and the TG3
  // matrix, RangeJacobi of mass.h:164-176), or the Laplace diagonal.
  template <int P, int OPK, typename RM>
  __device__ __forceinline__ double
  cg_inv_jacobi(const Geo &geo, const TileMaps<P, RM> &m, int gx0, int gy0, int i, int j, bool fixed)
  {
    if constexpr (OPK == OPK_LAPLACE)
      return fixed ? 1.0 : laplace_inv_diag<P>(geo, gx0 + j, gy0 + i);
    else
      return own_inv_jacobi(m, i, j, fixed);
  }

  // r = b - A xg with xg = extrapolate ? 2 x_cur - x_prev (written to x_new) : x_new;
  // partials per system: b.b, r.r, r.D^{-1}r. Storage R, arithmetic A (A = double:
  // the FP64 residual of the refinement). One system per CTA.
  // TG3: A is the streaming matrix of sc; systems whose bit is set in skip are
  // not solved (zero sums: converged at the start, x untouched). With FP32
  // arithmetic (the start of the mixed solve, whose rounds form their own sums)
  // no partials are written.
  // FP32 storage and the register-bound TG3 / Laplace operators stage b in shared
  // memory (the FP32 start runs 8 CTAs per SM at 32 registers); the FP64 mass start
  // reads it in place, which leaves room for 6 CTAs per SM.
  // Tile (bx, by) of system bz, of an nbx x nby tile grid (the kernel below, and
  // the body of its batched form).
  template <int P, typename R, typename X, typename A, int OPK>
  __device__ __forceinline__ void
  cg_start_tile(const Geo &geo, const R *__restrict__ b, const X *__restrict__ x_cur, const X *__restrict__ x_prev,
                X *__restrict__ x_new, R *__restrict__ r, int extrapolate, double *__restrict__ partials,
                const StreamCoef &sc, int skip, int bx, int by, int bz, int nbx, int nby)
  {
    using T = Tile<P>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    A *s_u = reinterpret_cast<A *>(sm_raw), *s_t = s_u + T::NF;
    R *s_b = reinterpret_cast<R *>(s_t + op_scratch<P, OPK>());
    __shared__ TileMaps<P, A> maps;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int s = bz;
    if ((skip >> s) & 1)
      {
        if (threadIdx.x == 0)
          {
            const int nt = nbx * nby, tile = by * nbx + bx;
            for (int q = 0; q < 3; ++q)
              partials[(long long)(q * NM + s) * nt + tile] = 0.0;
          }
        return;
      }
    const int gx0 = bx * T::TX, gy0 = by * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    __syncthreads();
    const long long o = s * N;
    // the start as stored (rounded to X), so that r is the residual of the stored x
    if (extrapolate)
      stage<P>(s_u, maps, [&](long long idx) -> A { return A(X(-A(x_prev[o + idx]) + A(2) * A(x_cur[o + idx]))); });
    else
      stage<P>(s_u, maps, [&](long long idx) -> A { return A(x_new[o + idx]); });
    constexpr bool STAGE_B = sizeof(R) == sizeof(float) || OPK != OPK_MASS;
    if constexpr (STAGE_B)
      stage_own<P>(s_b, b + o, g, gx0, gy0);
    __syncthreads();
    constexpr bool SUMS = sizeof(A) == sizeof(double);
    double part[3] = {0, 0, 0};
    R *rs = r + o;
    // this system's vectors, indexed by 32-bit node offsets
    X *xns = x_new + o;
    const X *xcs = extrapolate ? x_cur + o : nullptr, *xps = extrapolate ? x_prev + o : nullptr;
    const R *bs = b + o;
    op_apply<P, OPK>(s_u, s_t, maps, g, gx0, gy0, sc, s, [&](int i, int j, int idx, bool image, A Ax) {
      A xg;
      if (image)
        {
          xg = extrapolate ? A(X(-A(xps[idx]) + A(2) * A(xcs[idx]))) : A(xns[idx]);
          Ax = xg;
        }
      else
        xg = s_u[(i + P) * T::PF + j + P];
      if (extrapolate)
        xns[idx] = X(xg);
      const A bb = A(STAGE_B ? s_b[i * T::TX + j] : bs[idx]);
      const A rr = -Ax + bb;
      rs[idx] = R(rr);
      if constexpr (SUMS)
        if (owned_row(gy0 + i, g))
          {
            part[0] += double(bb) * double(bb);
            part[1] += double(rr) * double(rr);
            part[2] += double(rr) * (cg_inv_jacobi<P, OPK>(geo, maps, gx0, gy0, i, j, image) * double(rr));
          }
    });
    if constexpr (SUMS)
      {
        const int nt = nbx * nby, tile = by * nbx + bx;
        // partial (quantity k of system s) at [(k*NM + s) * n_tiles + tile]
        block_reduce_store<3>(part, partials + (long long)s * nt, tile, NM * nt);
      }
  }

  template <int P, typename R, typename X = R, typename A = R, int OPK = OPK_MASS>
  __global__ void __launch_bounds__(THREADS, OPK != OPK_MASS ? 2 : sizeof(R) == sizeof(float) ? 8 : 6)
    k_cg_start(const Geo geo, const R *__restrict__ b, const X *__restrict__ x_cur, const X *__restrict__ x_prev,
               X *__restrict__ x_new, R *__restrict__ r, int extrapolate, double *__restrict__ partials,
               const StreamCoef sc, int skip)
  {
    cg_start_tile<P, R, X, A, OPK>(geo, b, x_cur, x_prev, x_new, r, extrapolate, partials, sc, skip, blockIdx.x,
                                   blockIdx.y, blockIdx.z, gridDim.x, gridDim.y);
  }

  // p <- D^{-1} r + beta p (p <- D^{-1} r on the first iteration); partial p.Ap. One system per CTA.
  template <int P, typename R, int OPK = OPK_MASS>
  __global__ void __launch_bounds__(THREADS, OPK == OPK_MASS ? 8 : 2)
    k_cg_p(const Geo geo, const R *__restrict__ r, const R *__restrict__ p_in, R *__restrict__ p_out,
           const CgState *__restrict__ st, double *__restrict__ partials, const StreamCoef sc)
  {
    using T = Tile<P>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R *s_u = reinterpret_cast<R *>(sm_raw), *s_t = s_u + T::NF;
    __shared__ TileMaps<P, R> maps;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int s = blockIdx.z;
    const int nt = gridDim.x * gridDim.y, tile = blockIdx.y * gridDim.x + blockIdx.x;
    if (!st->active[s])
      return;
    const int gx0 = blockIdx.x * T::TX, gy0 = blockIdx.y * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    const bool first = st->it[s] == 0;
    const R beta = R(st->beta[s]);
    const long long o = s * N;
    __syncthreads();
    const R *rsys = r + o, *psys = p_in + o;
    stage_ij<P>(s_u, maps, [&](long long idx, int c, int rw, int fx, int fy) -> R {
      // the mass Jacobi factors from the tile maps (shared memory), not from global memory
      const R z = R(OPK == OPK_LAPLACE ? laplace_inv_diag<P>(geo, c, rw) : maps.ijx[fx] * maps.ijy[fy]) * rsys[idx];
      return first ? z : fma(beta, psys[idx], z);
    });
    __syncthreads();
    double part[1] = {0};
    R *posys = p_out + o;
    op_apply<P, OPK>(s_u, s_t, maps, g, gx0, gy0, sc, s, [&](int i, int j, int idx, bool image, R Ap) {
      R pn;
      if (image)
        {
          pn = first ? rsys[idx] : fma(beta, psys[idx], rsys[idx]);
          Ap = pn;
        }
      else
        pn = s_u[(i + P) * T::PF + j + P];
      posys[idx] = pn;
      if (owned_row(gy0 + i, g))
        part[0] += double(pn) * double(Ap);
    });
    block_reduce_store<1>(part, partials + (long long)s * nt, tile, NM * nt);
  }

  // v = A p recomputed; x += alpha p, r -= alpha v; partials r.r, r.D^{-1}r. One system per CTA.
  template <int P, typename R, int OPK = OPK_MASS>
  __global__ void __launch_bounds__(THREADS, OPK == OPK_MASS ? 8 : 2)
    k_cg_update(const Geo geo, R *__restrict__ x, R *__restrict__ r, const R *__restrict__ p,
                const CgState *__restrict__ st, double *__restrict__ partials, const StreamCoef sc)
  {
    using T = Tile<P>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R *s_u = reinterpret_cast<R *>(sm_raw), *s_t = s_u + T::NF;
    __shared__ TileMaps<P, R> maps;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int s = blockIdx.z;
    const int nt = gridDim.x * gridDim.y, tile = blockIdx.y * gridDim.x + blockIdx.x;
    if (!st->active[s])
      return;
    const int gx0 = blockIdx.x * T::TX, gy0 = blockIdx.y * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    const R al = R(st->alpha[s]);
    const long long o = s * N;
    const R *ps = p + o;
    R *xs = x + o, *rs = r + o;
    // The mass update reads the own x and r in place (less shared memory: more CTAs
    // per SM); the TG3 and Laplace updates, held at 2 CTAs per SM by their registers,
    // stage them with the footprint so that their loads are in flight together.
    constexpr bool STAGE_XR = OPK != OPK_MASS;
    R *s_x = s_t + op_scratch<P, OPK>(), *s_r = s_x + T::TX * T::TY;
    __syncthreads();
    stage<P>(s_u, maps, [&](long long idx) { return ps[idx]; });
    if constexpr (STAGE_XR)
      {
        stage_own<P>(s_x, xs, g, gx0, gy0);
        stage_own<P>(s_r, rs, g, gx0, gy0);
      }
    __syncthreads();
    double part[2] = {0, 0};
    op_apply<P, OPK>(s_u, s_t, maps, g, gx0, gy0, sc, s, [&](int i, int j, int idx, bool image, R Ap) {
      const R pv = image ? ps[idx] : s_u[(i + P) * T::PF + j + P];
      if (image)
        Ap = pv;
      const int t = i * T::TX + j;
      xs[idx] = (STAGE_XR ? s_x[t] : xs[idx]) + al * pv;
      const R rr = (STAGE_XR ? s_r[t] : rs[idx]) + -al * Ap;
      rs[idx] = rr;
      if (owned_row(gy0 + i, g))
        {
          part[0] += double(rr) * double(rr);
          part[1] += double(rr) * (cg_inv_jacobi<P, OPK>(geo, maps, gx0, gy0, i, j, image) * double(rr));
        }
    });
    block_reduce_store<2>(part, partials + (long long)s * nt, tile, NM * nt);
  }

  // --------------------------- tensor-product window solve (mixed precision)
  // On an axis-parallel tensor-product mesh the consistent mass matrix is
  // M = My (x) Mx, so M^{-1} = My^{-1} (x) Mx^{-1}. The rows of the 1-D inverses
  // decay exponentially, so M^{-1} r at the own nodes of a tile follows from
  // banded LDL^T solves on a window of W nodes around the tile in each direction
  // (factors from window_ldl on the host), to a few 1e-6 of |r|.
  // Tiles of T nodes along an axis of nf stored nodes (nu distinct). On a periodic
  // axis whose distinct nodes fill whole tiles, the image node (the last stored
  // node) gets no tile of its own: the last tile takes it.
  __host__ __device__ constexpr int
  tiles_along(int nf, int nu, int periodic, int T)
  {
    return (periodic && nu % T == 0) ? nu / T : (nf + T - 1) / T;
  }

  // ------------------------------------------------ start of the mixed solve
  // x0 = 2 x_cur - x_prev (the extrapolated start, rounded to FP32 and stored in
  // x_new) and r0 = b - A x0 in FP32 arithmetic, for one tile of TX x TY nodes of
  // one system. A = My (x) Mx on the assembled 1-D rows (rounded to FP32);
  // periodic images have identity rows. x0 is staged with a halo of P nodes; a
  // thread owns one column: the x pass of its column on the tile's rows and halo
  // (kept in registers), then the y pass. r0 only feeds the first FP32
  // correction; the rounds form the residuals in FP64.
  template <int P>
  struct StartShape
  {
    static constexpr int TX = 128, TY = 16, THREADS = 128;
    static constexpr int FX = TX + 2 * P, FY = TY + 2 * P; // staged x0
    static constexpr int K = 2 * P + 1;                   // entries of an assembled 1-D row
  };

  __device__ __forceinline__ float
  extrapolated(const float *__restrict__ x_cur, const float *__restrict__ x_prev, long long idx)
  {
    return fmaf(2.f, x_cur[idx], -x_prev[idx]);
  }

  template <int P>
  __device__ __forceinline__ void
  mixed_start_tile(const Geo &geo, const float *__restrict__ b, const float *__restrict__ x_cur,
                   const float *__restrict__ x_prev, float *__restrict__ x_new, float *__restrict__ r, int bx, int by,
                   int s)
  {
    using S = StartShape<P>;
    constexpr int K = S::K, FX = S::FX, FY = S::FY;
    __shared__ float s_x[FY * FX], s_p[FY * FX]; // x_cur, then x0; x_prev
    __shared__ int s_col[FX], s_rowoff[FY];
    __shared__ float s_my[S::TY][K + 1];
    const Grid &g = geo.g;
    const long long o = (long long)s * g.N;
    const float *xc = x_cur + o, *xp = x_prev + o, *bs = b + o;
    float *xn = x_new + o, *rs = r + o;
    const int gx0 = bx * S::TX, gy0 = by * S::TY, tid = threadIdx.x;
    for (int t = tid; t < FX; t += S::THREADS)
      s_col[t] = wrap(gx0 - P + t, g.px, g.nux, g.nfx);
    for (int t = tid; t < FY; t += S::THREADS)
      {
        const int row = wrap(gy0 - P + t, g.py, g.nuy, g.nfy);
        s_rowoff[t] = row < 0 ? -1 : row * g.nfx;
      }
    for (int t = tid; t < S::TY * (K + 1); t += S::THREADS)
      {
        const int i = t / (K + 1), k = t - i * (K + 1), gy = gy0 + i;
        s_my[i][k] = (k < K && gy < g.nfy && !(g.py && gy == g.nuy)) ? float(geo.rowy[(long long)gy * K + k]) : 0.f;
      }
    __syncthreads();
    // x_cur and x_prev on the tile and its halo: asynchronous copies, all in flight
    // at once (zero outside the grid). A tile whose staged rows and columns neither
    // leave the grid nor cross a periodic seam addresses them directly.
    const bool inner = gx0 - P >= 0 && gx0 - P + FX <= (g.px ? g.nux : g.nfx) && gy0 - P >= 0 &&
                       gy0 - P + FY <= (g.py ? g.nuy : g.nfy);
    if (inner)
      {
        const long long first = (long long)(gy0 - P) * g.nfx + gx0 - P;
        for (int c = tid; c < FX; c += S::THREADS)
          {
            const float *pc = xc + first + c, *pp = xp + first + c;
#pragma unroll 11
            for (int q = 0; q < FY; ++q)
              {
                cp_async4(&s_x[q * FX + c], pc, true);
                cp_async4(&s_p[q * FX + c], pp, true);
                pc += g.nfx;
                pp += g.nfx;
              }
          }
      }
    else
      for (int c = tid; c < FX; c += S::THREADS)
        {
          const int col = s_col[c];
#pragma unroll 8
          for (int q = 0; q < FY; ++q)
            {
              const int ro = s_rowoff[q];
              const bool ok = ro >= 0 && col >= 0;
              const long long at = ok ? ro + col : 0;
              cp_async4(&s_x[q * FX + c], xc + at, ok);
              cp_async4(&s_p[q * FX + c], xp + at, ok);
            }
        }
    const int j = tid, gx = gx0 + j;
    const bool col_in = gx < g.nfx;
    const bool img_col = g.px && gx == g.nux;
    float mx[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
      mx[k] = (col_in && !img_col) ? float(geo.rowx[(long long)gx * K + k]) : 0.f;
    // this column's b, loaded while the copies land
    const int rows_in = g.nfy - gy0;
    float bv[S::TY];
#pragma unroll
    for (int i = 0; i < S::TY; ++i)
      bv[i] = (col_in && i < rows_in) ? bs[(long long)(gy0 + i) * g.nfx + gx] : 0.f;
    cp_async_wait_all();
    __syncthreads();
    for (int t = tid; t < FY * FX; t += S::THREADS)
      s_x[t] = fmaf(2.f, s_x[t], -s_p[t]);
    __syncthreads();
    if (!col_in)
      return; // no barrier follows
    // (Mx x0) of this column on the tile's rows and a halo of P rows
    float t[FY];
#pragma unroll
    for (int q = 0; q < FY; ++q)
      {
        const float *w = &s_x[q * FX + j]; // columns gx - P .. gx + P
        float a0 = mx[0] * w[0], a1 = mx[1] * w[1];
#pragma unroll
        for (int k = 2; k < K; k += 2)
          {
            a0 = fmaf(mx[k], w[k], a0);
            if (k + 1 < K)
              a1 = fmaf(mx[k + 1], w[k + 1], a1);
          }
        t[q] = a0 + a1;
      }
#pragma unroll
    for (int i = 0; i < S::TY; ++i)
      {
        if (i >= rows_in)
          break;
        const int gy = gy0 + i;
        const long long idx = (long long)gy * g.nfx + gx;
        const bool image = img_col || (g.py && gy == g.nuy);
        float x0, ax;
        if (image)
          {
            x0 = extrapolated(xc, xp, idx);
            ax = x0; // identity row
          }
        else
          {
            x0 = s_x[(i + P) * FX + j + P];
            float a0 = s_my[i][0] * t[i], a1 = s_my[i][1] * t[i + 1];
#pragma unroll
            for (int k = 2; k < K; k += 2)
              {
                a0 = fmaf(s_my[i][k], t[i + k], a0);
                if (k + 1 < K)
                  a1 = fmaf(s_my[i][k + 1], t[i + k + 1], a1);
              }
            ax = a0 + a1;
          }
        xn[idx] = x0;
        rs[idx] = bv[i] - ax;
      }
    // a periodic axis's image column (row) beyond the last tile (tiles_along): identity rows
    auto image_start = [&](int x, int y) {
      const long long idx = (long long)y * g.nfx + x;
      const float v = extrapolated(xc, xp, idx);
      xn[idx] = v;
      rs[idx] = bs[idx] - v;
    };
    const int nbx = tiles_along(g.nfx, g.nux, g.px, S::TX), nby = tiles_along(g.nfy, g.nuy, g.py, S::TY);
    const bool ext_x = g.px && g.nux % S::TX == 0 && bx == nbx - 1;
    const bool ext_y = g.py && g.nuy % S::TY == 0 && by == nby - 1;
    if (ext_y)
      image_start(gx, g.nuy);
    if (ext_x && j == 0)
      {
        for (int i = 0; i < S::TY && gy0 + i < g.nfy; ++i)
          image_start(g.nux, gy0 + i);
        if (ext_y)
          image_start(g.nux, g.nuy);
      }
  }

  // grid (x tiles, y tiles, systems)
  template <int P>
  __global__ void __launch_bounds__(StartShape<P>::THREADS)
    k_mixed_start(const Geo geo, const float *__restrict__ b, const float *__restrict__ x_cur,
                  const float *__restrict__ x_prev, float *__restrict__ x_new, float *__restrict__ r)
  {
    mixed_start_tile<P>(geo, b, x_cur, x_prev, x_new, r, blockIdx.x, blockIdx.y, blockIdx.z);
  }

  template <int P>
  struct WinShape
  {
    // window halo: the 1-D inverses decay to a few 1e-6 over W nodes; one round's FP64
    // check then finds the residual at about 1e-5 of the round's start residual
    static constexpr int W = P == 1 ? 8 : P == 2 ? 12 : P == 3 ? 16 : 20;
    static constexpr int TX = 128, TY = 64;                // own nodes
    // CTAs per SM the registers are sized for (shared memory admits 4 / 3 / 3 / 2)
    static constexpr int MIN_CTAS = P == 1 ? 4 : P == 4 ? 2 : 3;
    static constexpr int FX = TX + 2 * W, FY = TY + 2 * W; // window
    // pitch = 4 (mod 8): rows are 16-byte aligned, and eight lanes on eight rows hit
    // distinct bank groups with 16-byte accesses (row sweeps) as with 4-byte ones
    // on consecutive columns (column sweeps)
    static constexpr int PF = FX + 4;
    static constexpr int NC = P == 1 ? 2 : P <= 3 ? 4 : 8; // factor floats per window position (padded)
    static constexpr int K = 2 * P + 1;                    // entries of an assembled 1-D row
    static constexpr int KP = K + 1;                       // row pitch of the My rows (16-byte pairs)
    static constexpr int THREADS = 160;
    static_assert(FY <= THREADS && TX + 2 * P <= THREADS, "one thread per window row and per own-plus-halo column");
    static_assert(TX < THREADS, "a spare thread for an image column");
    static_assert(FX % 8 == 0 && FY % 4 == 0 && W - P >= 3, "whole chunks; the backward sweeps stop at W - P");
  };

  template <int P>
  constexpr size_t
  window_smem()
  {
    using S = WinShape<P>;
    return sizeof(float) * size_t(S::PF) * S::FY + sizeof(double) * S::TY * S::KP;
  }

  // The factor row of window position q: l[k-1] = l_{q,q-k}, l[P] = 1/d_q (one
  // or two vector loads from rows of NC floats, 16-byte aligned).
  template <int P, int NC>
  __device__ __forceinline__ void
  ldl_row(const float *c, int q, float (&l)[P + 1])
  {
    if constexpr (NC == 2)
      {
        const float2 v = *reinterpret_cast<const float2 *>(c + q * NC);
        l[0] = v.x;
        l[1] = v.y;
      }
    else
      {
        float tmp[NC];
#pragma unroll
        for (int h = 0; h < NC; h += 4)
          {
            const float4 v = *reinterpret_cast<const float4 *>(c + q * NC + h);
            tmp[h] = v.x;
            tmp[h + 1] = v.y;
            tmp[h + 2] = v.z;
            tmp[h + 3] = v.w;
          }
#pragma unroll
        for (int k = 0; k <= P; ++k)
          l[k] = tmp[k];
      }
  }

  // Forward and backward substitution of one banded LDL^T system of n
  // unknowns stored at line[q * stride] (in place), with the factor rows of
  // ldl_row; the backward sweep stops at the chunk holding position stop.
  // Chunks of four positions: the loads of a chunk are issued before its
  // dependent chain; with stride 1 a chunk is one 16-byte access.
  template <int P, int NC, int n, int stride, int stop>
  __device__ __forceinline__ void
  ldl_solve(float *line, const float *c)
  {
    static_assert(n % 4 == 0, "whole chunks");
    constexpr int CH = 4;
    auto load4 = [&](int q0, float (&v)[CH]) {
      if constexpr (stride == 1)
        {
          const float4 t = *reinterpret_cast<const float4 *>(line + q0);
          v[0] = t.x;
          v[1] = t.y;
          v[2] = t.z;
          v[3] = t.w;
        }
      else
        {
#pragma unroll
          for (int u = 0; u < CH; ++u)
            v[u] = line[(q0 + u) * stride];
        }
    };
    auto store4 = [&](int q0, const float (&v)[CH]) {
      if constexpr (stride == 1)
        *reinterpret_cast<float4 *>(line + q0) = make_float4(v[0], v[1], v[2], v[3]);
      else
        {
#pragma unroll
          for (int u = 0; u < CH; ++u)
            line[(q0 + u) * stride] = v[u];
        }
    };
    float y[P];
#pragma unroll
    for (int k = 0; k < P; ++k)
      y[k] = 0.f; // y[k]: the value k + 1 positions back
#pragma unroll 2
    for (int q0 = 0; q0 < n; q0 += CH)
      {
        float v[CH], l[CH][P + 1];
        load4(q0, v);
#pragma unroll
        for (int u = 0; u < CH; ++u)
          ldl_row<P, NC>(c, q0 + u, l[u]);
#pragma unroll
        for (int u = 0; u < CH; ++u)
          {
            float t = v[u];
#pragma unroll
            for (int k = P; k >= 1; --k)
              t = fmaf(-l[u][k - 1], y[k - 1], t);
#pragma unroll
            for (int k = P - 1; k >= 1; --k)
              y[k] = y[k - 1];
            y[0] = t;
            v[u] = t * l[u][P];
          }
        store4(q0, v);
      }
#pragma unroll
    for (int k = 0; k < P; ++k)
      y[k] = 0.f; // y[k]: the value k + 1 positions ahead
    // the factor rows of the P positions after the chunk: the first P rows of the
    // previous chunk (none after the last position)
    float lp[P][P + 1];
#pragma unroll
    for (int u = 0; u < P; ++u)
#pragma unroll
      for (int k = 0; k <= P; ++k)
        lp[u][k] = 0.f;
#pragma unroll 2
    for (int q0 = n - CH; q0 + CH > stop; q0 -= CH) // the last chunk may reach below stop
      {
        float v[CH], l[CH + P][P + 1];
        load4(q0, v);
#pragma unroll
        for (int u = 0; u < CH; ++u)
          ldl_row<P, NC>(c, q0 + u, l[u]);
#pragma unroll
        for (int u = 0; u < P; ++u)
#pragma unroll
          for (int k = 0; k <= P; ++k)
            {
              l[CH + u][k] = lp[u][k];
              lp[u][k] = l[u][k];
            }
#pragma unroll
        for (int u = CH - 1; u >= 0; --u)
          {
            float t = v[u];
#pragma unroll
            for (int k = P; k >= 1; --k)
              t = fmaf(-l[u + k][k - 1], y[k - 1], t);
#pragma unroll
            for (int k = P - 1; k >= 1; --k)
              y[k] = y[k - 1];
            y[0] = t;
            v[u] = t;
          }
        store4(q0, v);
      }
  }

  // One refinement round of the mixed-precision mass solve, for the active
  // systems (all of them when all is set):
  //   x_out = x_in + M^{-1} r_in   (FP32 window solves),
  //   r_out = b - A x_out           (FP64 arithmetic on the FP32 values),
  // with the partial sums b.b and r.r of each system. The window
  // solves give the correction on the own nodes and on a halo of P nodes, so
  // that A x_out follows without another pass; the halo's correction is the
  // window solve's own, within a few 1e-8 of the neighbouring tile's. An
  // inactive system is copied (x_out = x_in, r_out = r_in): all systems end a
  // round in the same buffers. x and r are never updated in place (the halos
  // read the inputs). Periodic images have identity rows.
  template <int P>
  __device__ __forceinline__ void
  window_correct_tile(const Geo &geo, const float *__restrict__ lx, const float *__restrict__ ly,
                      const float *__restrict__ r_in, const float *__restrict__ x_in, const float *__restrict__ b,
                      float *__restrict__ x_out, float *__restrict__ r_out, const CgState *__restrict__ st, int all,
                      double *__restrict__ partials, int bx, int by, int bz, int nbx, int nby)
  {
    using S = WinShape<P>;
    constexpr int W = S::W, FX = S::FX, FY = S::FY, PF = S::PF, NC = S::NC, K = S::K, NT = S::THREADS;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    float *s_w = reinterpret_cast<float *>(sm_raw);                  // [FY][PF] the window
    double *s_my = reinterpret_cast<double *>(s_w + PF * FY);       // [TY][KP] My rows of the own rows (zero padded)
    __shared__ __align__(16) float s_lx[FX * NC], s_ly[FY * NC];     // factors (apart from the window: no aliasing)
    __shared__ int s_col[FX], s_row[FY];                             // storage column / row, -1 outside the grid
    __shared__ int s_rowoff[FY];                                     // storage offset of a window row, -1 outside
    const int s = bz;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = bx * S::TX, gy0 = by * S::TY;
    const int tid = threadIdx.x;
    const int n_tiles = nbx * nby, tile = by * nbx + bx;
    const float *rs = r_in + (long long)s * N, *xs = x_in + (long long)s * N, *bs = b + (long long)s * N;
    float *xo = x_out + (long long)s * N, *ro = r_out + (long long)s * N;
    double part[2] = {0, 0};
    // A periodic axis whose distinct nodes fill whole tiles has no tile for its
    // image column (row) alone: the last tile takes it (identity rows).
    const bool ext_x = g.px && g.nux % S::TX == 0 && bx == nbx - 1;
    const bool ext_y = g.py && g.nuy % S::TY == 0 && by == nby - 1;
    if (!all && !st->active[s])
      {
        // converged: carried over to the output buffers
        auto copy = [&](int gx, int gy) {
          const long long idx = (long long)gy * g.nfx + gx;
          xo[idx] = xs[idx];
          ro[idx] = rs[idx];
        };
        for (int t = tid; t < S::TX * S::TY; t += NT)
          {
            const int i = t / S::TX, j = t - i * S::TX;
            const int gx = gx0 + j, gy = gy0 + i;
            if (gx < g.nfx && gy < g.nfy)
              copy(gx, gy);
          }
        if (ext_y)
          for (int j = tid; j < S::TX; j += NT)
            if (gx0 + j < g.nfx)
              copy(gx0 + j, g.nuy);
        if (ext_x)
          for (int i = tid; i < S::TY + (ext_y ? 1 : 0); i += NT)
            if (gy0 + i < g.nfy)
              copy(g.nux, gy0 + i);
        block_reduce_store_n<2, NT>(part, partials + (long long)s * n_tiles, tile, NM * n_tiles);
        return;
      }
    const float *lxt = lx + (size_t)bx * FX * NC, *lyt = ly + (size_t)by * FY * NC;
    for (int t = tid; t < FX * NC; t += NT)
      s_lx[t] = lxt[t];
    for (int t = tid; t < FY * NC; t += NT)
      s_ly[t] = lyt[t];
    for (int t = tid; t < FX; t += NT)
      s_col[t] = wrap(gx0 - W + t, g.px, g.nux, g.nfx);
    for (int t = tid; t < FY; t += NT)
      {
        const int r = wrap(gy0 - W + t, g.py, g.nuy, g.nfy);
        s_row[t] = r;
        s_rowoff[t] = r < 0 ? -1 : r * g.nfx;
      }
    for (int t = tid; t < S::TY * S::KP; t += NT)
      {
        const int i = t / S::KP, k = t - i * S::KP, gy = gy0 + i;
        s_my[t] = (k < K && gy < g.nfy && !(g.py && gy == g.nuy)) ? geo.rowy[(long long)gy * K + k] : 0.0;
      }
    __syncthreads();
    // the window of r_in by asynchronous copies, all in flight at once, a window
    // column per thread (consecutive threads: consecutive addresses); meanwhile
    // this thread's column of x_in (own rows and a halo of P) into registers
    for (int c = tid; c < FX; c += NT)
      {
        const int col = s_col[c];
#pragma unroll 8
        for (int q = 0; q < FY; ++q)
          {
            const int ro = s_rowoff[q];
            const bool ok = ro >= 0 && col >= 0;
            cp_async4(&s_w[q * PF + c], ok ? rs + (ro + col) : rs, ok);
          }
      }
    const int cw = W - P + tid; // window column of this thread's y solve
    float xr[S::TY + 2 * P];
    {
      const int col = tid < S::TX + 2 * P ? s_col[cw] : -1;
#pragma unroll
      for (int q = 0; q < S::TY + 2 * P; ++q)
        {
          const int ro = s_rowoff[W - P + q];
          xr[q] = (ro >= 0 && col >= 0) ? xs[ro + col] : 0.f;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // x solves: one thread per window row (the y solves read the own columns and a halo of P)
    if (tid < FY)
      ldl_solve<P, NC, FX, 1, W - P>(s_w + tid * PF, s_lx);
    __syncthreads();
    // y solves: one thread per own-or-halo column, then x_out = x_in + z on the
    // own rows and a halo of P rows of that column (kept in the window)
    if (tid < S::TX + 2 * P)
      {
        ldl_solve<P, NC, FY, PF, W - P>(s_w + cw, s_ly);
        const int col = s_col[cw];
#pragma unroll
        for (int q = 0; q < S::TY + 2 * P; ++q)
          {
            const int row = s_row[W - P + q];
            float *w = &s_w[(W - P + q) * PF + cw];
            *w = (row >= 0 && col >= 0) ? xr[q] + *w : 0.f;
          }
      }
    __syncthreads();
    // own columns: write x_out, form r_out = b - A x_out in FP64
    if (tid < S::TX)
      {
        const int j = tid, gx = gx0 + j, c = W + j;
        const bool col_ok = gx < g.nfx;
        const bool img_col = g.px && gx == g.nux;
        double mx[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
          mx[k] = (col_ok && !img_col) ? geo.rowx[(long long)gx * K + k] : 0.0;
        // this column of b in batches of BR rows, the next batch in flight while one is used
        constexpr int BR = 16;
        static_assert(S::TY % BR == 0, "whole batches");
        float bn[BR];
        // this column's own nodes, by 32-bit offsets (a population array holds fewer than 2^31 nodes)
        const int col0 = gy0 * g.nfx + gx, pitch = g.nfx;
        const int rows_in = g.nfy - gy0; // own rows inside the grid
        auto load_b = [&](int i0) {
#pragma unroll
          for (int u = 0; u < BR; ++u)
            bn[u] = (col_ok && i0 + u < rows_in) ? bs[col0 + (i0 + u) * pitch] : 0.f;
        };
        load_b(0);
        // t[k] = (Mx x)(row i - P + k) of this column, a sliding window of 2P + 1 rows;
        // each row's sum in two independent halves (shorter FP64 dependency chains)
        double t[K];
        auto xrow = [&](int q) -> double {
          const float *w = &s_w[q * PF + c - P];
          double v0 = mx[0] * double(w[0]), v1 = mx[1] * double(w[1]);
#pragma unroll
          for (int l = 2; l < K; l += 2)
            {
              v0 = fma(mx[l], double(w[l]), v0);
              if (l + 1 < K)
                v1 = fma(mx[l + 1], double(w[l + 1]), v1);
            }
          return v0 + v1;
        };
#pragma unroll
        for (int k = 1; k < K; ++k)
          t[k] = xrow(W - P + k - 1);
#pragma unroll 1
        for (int i0 = 0; i0 < S::TY; i0 += BR)
        {
        float bc[BR];
#pragma unroll
        for (int u = 0; u < BR; ++u)
          bc[u] = bn[u];
        if (i0 + BR < S::TY)
          load_b(i0 + BR);
#pragma unroll
        for (int u = 0; u < BR; ++u)
          {
            const int i = i0 + u;
#pragma unroll
            for (int k = 0; k < K - 1; ++k)
              t[k] = t[k + 1];
            t[K - 1] = xrow(W + i + P);
            const int gy = gy0 + i;
            if (!col_ok || i >= rows_in)
              continue;
            const int idx = col0 + i * pitch;
            const bool image = img_col || (g.py && gy == g.nuy);
            double xv, ax;
            if (image)
              {
                xv = double(xs[idx]) + double(rs[idx]); // identity rows
                ax = xv;
              }
            else
              {
                xv = s_w[(W + i) * PF + c];
                // the row's coefficients in 16-byte pairs (broadcast loads)
                const double2 *my = reinterpret_cast<const double2 *>(s_my + i * S::KP);
                const double2 m0 = my[0];
                double a0 = m0.x * t[0], a1 = m0.y * t[1];
#pragma unroll
                for (int k = 2; k < K; k += 2)
                  {
                    const double2 mk = my[k / 2];
                    a0 = fma(mk.x, t[k], a0);
                    if (k + 1 < K)
                      a1 = fma(mk.y, t[k + 1], a1);
                  }
                ax = a0 + a1;
              }
            const double bb = bc[u], rr = bb - ax;
            xo[idx] = float(xv);
            ro[idx] = float(rr);
            if (owned_row(gy, g))
              {
                part[0] += bb * bb;
                part[1] += rr * rr;
              }
          }
        }
      }
    // the image row and column a tile takes beyond its own nodes (identity rows, as above)
    auto image_node = [&](int gx, int gy) {
      const long long idx = (long long)gy * g.nfx + gx;
      const double xv = double(xs[idx]) + double(rs[idx]);
      const double bb = bs[idx], rr = bb - xv;
      xo[idx] = float(xv);
      ro[idx] = float(rr);
      if (owned_row(gy, g))
        {
          part[0] += bb * bb;
          part[1] += rr * rr;
        }
    };
    if (ext_y && tid < S::TX && gx0 + tid < g.nfx)
      image_node(gx0 + tid, g.nuy);
    if (ext_x && tid == S::TX)
      {
        for (int i = 0; i < S::TY && gy0 + i < g.nfy; ++i)
          image_node(g.nux, gy0 + i);
        if (ext_y)
          image_node(g.nux, g.nuy);
      }
    block_reduce_store_n<2, NT>(part, partials + (long long)s * n_tiles, tile, NM * n_tiles);
  }

  template <int P>
  __global__ void __launch_bounds__(WinShape<P>::THREADS, WinShape<P>::MIN_CTAS)
    k_window_correct(const Geo geo, const float *__restrict__ lx, const float *__restrict__ ly,
                     const float *__restrict__ r_in, const float *__restrict__ x_in, const float *__restrict__ b,
                     float *__restrict__ x_out, float *__restrict__ r_out, const CgState *__restrict__ st, int all,
                     double *__restrict__ partials)
  {
    window_correct_tile<P>(geo, lx, ly, r_in, x_in, b, x_out, r_out, st, all, partials, blockIdx.x, blockIdx.y,
                           blockIdx.z, gridDim.x, gridDim.y);
  }

  // The scalar work of one CG phase, one thread per system, from the reduced sums.
  // phase 0 (after start): sums = [bb, rr, rz]; phase 1 (after p): [pAp];
  // phase 2 (after update): [rr, rz].
  __global__ void
  k_cg_scalars(CgState *st, const double *__restrict__ sums, int nsys, int phase, double cg_tol, int max_its)
  {
    const int s = threadIdx.x;
    if (s < NM)
      {
        if (phase == 0)
          {
            if (s < nsys && st->status == 0 && st->its_total[s] < max_its)
              {
                st->tol[s] = cg_tol * sqrt(sums[s]);
                const double res = sqrt(sums[NM + s]);
                st->res[s] = res;
                st->rz[s] = sums[2 * NM + s];
                st->it[s] = 0;
                st->beta[s] = 0;
                st->zero[s] = sums[s] == 0.0;
                if (isnan(res))
                  {
                    st->active[s] = 0;
                    atomicExch(&st->status, 3); // LBFEM_ERR_NONFINITE
                  }
                else
                  st->active[s] = (res <= st->tol[s] || st->zero[s]) ? 0 : 1;
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
            ++st->it[s];
            const int it = ++st->its_total[s];
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
        if (phase == 2)
          ++st->iter;
      }
  }

  // ------------------------------------------------- device-side step control
  // Graph control after a CG phase: the loop goes on while a system is active
  // and no failure occurred; on exit the solve is folded into the counters.
  __global__ void
  k_cg_control(const CgState *__restrict__ st, DevStats *__restrict__ ds, cudaGraphConditionalHandle h, int in_body)
  {
    if (threadIdx.x != 0)
      return;
    const bool go = st->n_active > 0 && st->status == 0;
    if (in_body)
      ++ds->bodies;
    if (!go)
      {
        ds->its += st->total_its;
        if (st->status != 0 && ds->sticky == 0)
          ds->sticky = st->status;
      }
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }

  // The bookkeeping of one round of the mixed-precision mass solve, after the
  // round's correction kernel and the reduction of its sums [bb, rr]: a
  // corrected system whose residual meets tol stops; a round that halves no
  // active residual means the tolerance lies below the FP32 resolution of the
  // solution (status 4); round max_rounds is the cap (status 2). Corrections
  // are counted; use_h: sets the graph loop condition.
  constexpr double MIXED_SLACK = 64.0;

  __device__ __forceinline__ void
  mixed_round_body(CgState *__restrict__ st, const double *__restrict__ sums, DevStats *__restrict__ ds, int nsys,
                   double tol, int max_rounds)
  {
    __shared__ int corrected[NM], progress[NM];
    const int s = threadIdx.x;
    const int round = st->iter;
    if (s < NM)
      {
        corrected[s] = s < nsys && (round == 0 || st->active[s]);
        progress[s] = 0;
        if (corrected[s] && st->status == 0)
          {
            const double res = sqrt(sums[NM + s]), tv = tol * sqrt(sums[s]);
            st->tol[s] = tv;
            if (sums[s] == 0.0)
              st->zero[s] = 1; // b = 0 exactly: x = 0 (k_zero_flagged), no further rounds
            if (isnan(res))
              {
                st->active[s] = 0;
                atomicExch(&st->status, 3); // LBFEM_ERR_NONFINITE
              }
            else
              {
                int act = (res > tv && !st->zero[s]) ? 1 : 0;
                const bool halved = round == 0 || res <= 0.5 * st->res[s];
                // A correction that no longer halves the residual has reached the FP32
                // resolution of the solution, about 2^-24 cond(M) |b|, which exceeds the
                // default tolerance on strongly stretched meshes. Within MIXED_SLACK of the
                // tolerance that is convergence; beyond it, stagnation (a failure).
                if (act && !halved && res <= MIXED_SLACK * tv)
                  act = 0;
                st->active[s] = act;
                progress[s] = act && halved;
              }
            st->res[s] = res;
          }
        else if (!corrected[s])
          st->active[s] = 0;
      }
    __syncthreads();
    if (threadIdx.x == 0)
      {
        int n = 0, nc = 0, np = 0;
        for (int k = 0; k < NM; ++k)
          {
            n += st->active[k];
            nc += corrected[k];
            np += progress[k];
          }
        st->total_its += nc;
        if (ds)
          ds->its += nc;
        ++st->iter;
        if (st->status == 0 && n > 0 && np == 0)
          st->status = 4; // stagnation
        else if (st->status == 0 && n > 0 && st->iter >= max_rounds)
          st->status = 2; // LBFEM_ERR_NO_CONVERGENCE
        st->n_active = st->status ? 0 : n;
        if (ds)
          {
            if (round > 0 && nc > 0)
              ++ds->bodies;
            if (st->status != 0 && ds->sticky == 0)
              ds->sticky = st->status;
          }
      }
  }

  __global__ void
  k_mixed_round(CgState *__restrict__ st, const double *__restrict__ sums, DevStats *__restrict__ ds, int nsys,
                double tol, int max_rounds, cudaGraphConditionalHandle h, int use_h)
  {
    mixed_round_body(st, sums, ds, nsys, tol, max_rounds);
    if (use_h && threadIdx.x == 0)
      cudaGraphSetConditional(h, st->n_active > 0 ? 1u : 0u);
  }
} // namespace lbfem_gpu
