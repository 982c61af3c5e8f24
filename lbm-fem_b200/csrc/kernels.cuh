// Device kernels of the lbm-fem hot path for sm_100a (FP64 plain path).
//
// Layout in HBM: structure of arrays, one contiguous array per population
// (block a of a population vector at [a*N, (a+1)*N)), node (i, j) of the
// (p*nx+1) x (p*ny+1) structured grid at j*nfx + i. In a periodic direction
// the last column/row holds the periodic images (deal.II's constrained DoFs):
// stencils never read them (they read the source node), nodal maps update
// them from their own values, and the streaming increment there is zero, as
// in the reference.
//
// Operators (see geometry.h): the advection right-hand side and the mass
// vmult are owner-computes tile stencils. A CTA stages one tile of nodes plus a
// halo of p nodes in shared memory, applies the assembled 1-D x operators
// (x pass) and then the y operators (y pass), and writes its own nodes: no
// scatter, no atomics, deterministic. Reductions are fixed-order (per-CTA
// partials, then a one-CTA final sum).
#pragma once

#include <cstdint>

namespace lbfem_gpu
{
  constexpr int Q = 9;
  constexpr int NM = 8;
  constexpr int THREADS = 256;
  constexpr int NPART = 16; // max reduction quantities per kernel

  // Shape of a tile of nodes per CTA.
  template <int P>
  struct Tile
  {
    static constexpr int TX = 32, TY = 16;
    static constexpr int HX = TX + 2 * P, HY = TY + 2 * P, HN = HX * HY;
    static constexpr int K = 2 * P + 1;
  };

  struct Grid
  {
    int nfx, nfy; // nodes per axis, images included
    int nux, nuy; // distinct nodes per axis (the wrap modulus of a periodic axis)
    int px, py;
    long long N;
  };

  // Everything a kernel needs to know about the discretisation.
  struct Geo
  {
    Grid g;
    const double *rowx, *rowy;   // [4][n][2p+1]: M, C, C^T, K
    const double *diagx, *diagy; // Jacobi diagonal per axis
    const double *lumpx, *lumpy; // lumped diagonal per axis
    const uint8_t *wall;         // per node: 0 fluid, k > 0 wall with velocity wall_u[2(k-1)..]; may be null
    const double *wall_u;
  };

  __device__ __constant__ double c_W[Q] = {4. / 9., 1. / 9., 1. / 36., 1. / 9., 1. / 36.,
                                           1. / 9., 1. / 36., 1. / 9., 1. / 36.};
  __device__ __constant__ double c_EX[Q] = {0, 1, 1, 0, -1, -1, -1, 0, 1};
  __device__ __constant__ double c_EY[Q] = {0, 0, 1, 1, 1, 0, -1, -1, -1};

  // Storage index of a (possibly out-of-range) grid coordinate: periodic axes
  // wrap to the distinct nodes (images map to their source), others give -1.
  __device__ __forceinline__ int
  wrap(int i, int periodic, int nu, int nf)
  {
    if (periodic)
      {
        i %= nu;
        return i < 0 ? i + nu : i;
      }
    return (i >= 0 && i < nf) ? i : -1;
  }

  __device__ __forceinline__ bool
  is_image(int i, int j, const Grid &g)
  {
    return (g.px && i == g.nux) || (g.py && j == g.nuy);
  }

  __device__ __forceinline__ double
  inv_jacobi(int i, int j, const Geo &geo)
  {
    if (is_image(i, j, geo.g))
      return 1.0;
    return 1.0 / (geo.diagx[i] * geo.diagy[j]);
  }

  struct Mom
  {
    double rho, ux, uy;
  };

  // D2Q9::moments, d2q9.h:30-41
  __device__ __forceinline__ Mom
  moments(const double (&f)[Q])
  {
    double rho = 0, mx = 0, my = 0;
#pragma unroll
    for (int a = 0; a < Q; ++a)
      {
        rho += f[a];
        mx += c_EX[a] * f[a];
        my += c_EY[a] * f[a];
      }
    return {rho, mx / rho, my / rho};
  }

  // D2Q9::equilibrium, d2q9.h:44-55, population a
  __device__ __forceinline__ double
  feq_a(int a, const Mom &m)
  {
    const double uu = m.ux * m.ux + m.uy * m.uy;
    const double eu = c_EX[a] * m.ux + c_EY[a] * m.uy;
    return c_W[a] * m.rho * (1. + 3. * eu + 4.5 * eu * eu - 1.5 * uu);
  }

  // What a node imposes on its moments (collision.h:53-72).
  __device__ __forceinline__ Mom
  impose(Mom m, long long idx, const Geo &geo)
  {
    if (geo.wall)
      {
        const int k = geo.wall[idx];
        if (k)
          {
            m.ux = geo.wall_u[2 * (k - 1)];
            m.uy = geo.wall_u[2 * (k - 1) + 1];
          }
      }
    return m;
  }

  // ---------------------------------------------------- fixed-order reductions
  // Sums v[0..nq) over the CTA (warp shuffles, then warp 0) and stores the CTA
  // totals at partials[q * gridDim + block].
  template <int NQ>
  __device__ __forceinline__ void
  block_reduce_store(double (&v)[NQ], int nq, double *partials, int block, int n_blocks)
  {
    __shared__ double warp_sum[NQ][THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      {
        if (q >= nq)
          break;
        double s = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0)
          warp_sum[q][warp] = s;
      }
    __syncthreads();
    if (warp == 0)
      {
        for (int q = 0; q < nq; ++q)
          {
            double s = lane < THREADS / 32 ? warp_sum[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
              s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0)
              partials[(long long)q * n_blocks + block] = s;
          }
      }
    __syncthreads();
  }

  // One CTA of 1024 threads: out[q] = sum_b partials[q * n_blocks + b], in a fixed order.
  __global__ void
  k_reduce_partials(const double *__restrict__ partials, int n_blocks, int nq, double *__restrict__ out)
  {
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < nq; ++q)
      {
        double s = 0;
        for (int b = threadIdx.x; b < n_blocks; b += blockDim.x)
          s += partials[(long long)q * n_blocks + b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0)
          red[warp] = s;
        __syncthreads();
        if (warp == 0)
          {
            s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
              s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0)
              out[q] = s;
          }
        __syncthreads();
      }
  }

  // ------------------------------------------------------------ tile helpers
  template <int P>
  __device__ __forceinline__ void
  load_rows(double *s_row, const double *__restrict__ rows, int g0, int n_own, int n_nodes)
  {
    constexpr int K = 2 * P + 1;
    for (int t = threadIdx.x; t < 4 * n_own * K; t += blockDim.x)
      {
        const int m = t / (n_own * K), r = t - m * n_own * K, i = r / K, k = r - i * K;
        const int gi = g0 + i;
        s_row[t] = gi < n_nodes ? rows[((long long)m * n_nodes + gi) * K + k] : 0.0;
      }
  }

  // s[ly][lx] <- src at grid (gx0 - P + lx, gy0 - P + ly), images read their source, outside 0.
  template <int P>
  __device__ __forceinline__ void
  load_tile(double *s, const double *__restrict__ src, const Grid &g, int gx0, int gy0)
  {
    using T = Tile<P>;
    for (int t = threadIdx.x; t < T::HN; t += blockDim.x)
      {
        const int ly = t / T::HX, lx = t - ly * T::HX;
        const int sx = wrap(gx0 - P + lx, g.px, g.nux, g.nfx), sy = wrap(gy0 - P + ly, g.py, g.nuy, g.nfy);
        s[t] = (sx >= 0 && sy >= 0) ? src[(long long)sy * g.nfx + sx] : 0.0;
      }
  }

  // out[lyo][lxo] = sum_k rowy[lyo][k] * (sum_k' rowx[lxo][k'] * s[lyo + k][lxo + k']) : the
  // tensor-product operator My (x) Mx (m = 0) or another (mx, my) pair, for all own nodes.
  // s_t is scratch of HY * TX.
  template <int P>
  __device__ __forceinline__ void
  xpass(const double *s, const double *s_rx, double *s_t)
  {
    using T = Tile<P>;
    for (int t = threadIdx.x; t < T::HY * T::TX; t += blockDim.x)
      {
        const int ly = t / T::TX, lxo = t - ly * T::TX;
        const double *row = s_rx + lxo * T::K;
        const double *u = s + ly * T::HX + lxo;
        double acc = 0;
#pragma unroll
        for (int k = 0; k < T::K; ++k)
          acc += row[k] * u[k];
        s_t[t] = acc;
      }
  }

  template <int P>
  __device__ __forceinline__ double
  ypass_at(const double *s_t, const double *s_ry, int lyo, int lxo)
  {
    using T = Tile<P>;
    const double *row = s_ry + lyo * T::K;
    double acc = 0;
#pragma unroll
    for (int k = 0; k < T::K; ++k)
      acc += row[k] * s_t[(lyo + k) * T::TX + lxo];
    return acc;
  }
} // namespace lbfem_gpu
