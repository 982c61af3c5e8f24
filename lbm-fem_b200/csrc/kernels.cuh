// Device building blocks of the lbm-fem hot path for sm_100a (FP64 plain path).
//
// Layout in HBM: structure of arrays, one contiguous array per population
// (block a of a population vector at [a*N, (a+1)*N)), node (i, j) of the
// (p*nx+1) x (p*ny+1) structured grid at j*nfx + i. In a periodic direction
// the last column/row holds the periodic images (deal.II's constrained DoFs):
// stencils never read them (they read the source node), nodal maps update
// them from their own values, and the streaming increment there is zero, as
// in the reference.
//
// Tensor-product operators (see geometry.h) are applied by owner-computes
// tiles. A CTA owns TX x TY nodes (whole cells: TX = p*CX, TY = p*CY) and
// stages the footprint -- the own nodes, one cell to the left/below and one
// node to the right/above -- in shared memory. The x pass applies the 1-D
// element matrices along x for every footprint row; the y pass applies them
// along y and writes the own nodes. Both passes sweep a run of cells per
// thread with the element matrices of the reference cell as constant-bank
// operands, the per-cell widths as the only geometry, and the shared vertex of
// two cells summed in a register: no scatter, no atomics, deterministic.
// Reductions are fixed-order: per-CTA partials, then one CTA per quantity.
#pragma once

#include <cstdint>

namespace lbfem_gpu
{
  constexpr int Q = 9;
  constexpr int NM = 8;
  constexpr int THREADS = 256;
  constexpr int MAXPD = 4;

  // Reference 1-D element matrices of FE_Q(p) on [0,1] (exact Gauss integration):
  // [p-1][0] = int l_a l_b, [1] = int l_a l_b', [2] = int l_a' l_b'.
  __device__ __constant__ double c_ref[MAXPD][3][MAXPD + 1][MAXPD + 1];
  __device__ __constant__ float c_reff[MAXPD][3][MAXPD + 1][MAXPD + 1]; // the same, rounded to FP32

  // Entry (a, b) of reference matrix OP of degree P in the arithmetic type R.
  template <typename R, int P, int OP>
  __device__ __forceinline__ R
  ref(int a, int b)
  {
    if constexpr (sizeof(R) == sizeof(float))
      return c_reff[P - 1][OP][a][b];
    else
      return c_ref[P - 1][OP][a][b];
  }
  enum
  {
    OP_M = 0,
    OP_C = 1,
    OP_K = 2
  };

  // Tile shapes: CX x CY cells per CTA; x-pass segments of KX cells, y-pass segments of KY cells.
  // Constraints: footprint rows TY + p + 1 <= 32 (one warp lane per row in the x pass).
  template <int P>
  struct TileShape;
  template <>
  struct TileShape<1>
  {
    static constexpr int CX = 64, CY = 24, KX = 8, KY = 6;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };
  template <>
  struct TileShape<2>
  {
    static constexpr int CX = 32, CY = 12, KX = 4, KY = 3;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };
  template <>
  struct TileShape<3>
  {
    static constexpr int CX = 21, CY = 8, KX = 3, KY = 2;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };
  template <>
  struct TileShape<4>
  {
    static constexpr int CX = 15, CY = 6, KX = 3, KY = 2;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };

  // A second shape per degree, for the run-time choice of the streaming kernel's
  // tile (tune_pair): 8 x-pass warps busy at every degree.
  template <int P>
  struct TileShapeAlt;
  template <>
  struct TileShapeAlt<1>
  {
    static constexpr int CX = 48, CY = 24, KX = 6, KY = 6;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };
  template <>
  struct TileShapeAlt<2>
  {
    static constexpr int CX = 24, CY = 12, KX = 3, KY = 3;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };
  template <>
  struct TileShapeAlt<3>
  {
    static constexpr int CX = 16, CY = 8, KX = 2, KY = 2;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };
  template <>
  struct TileShapeAlt<4>
  {
    static constexpr int CX = 16, CY = 6, KX = 2, KY = 2;
    static constexpr int MIN_CTAS = 2; // CTAs per SM the streaming kernel's registers are sized for
  };

  // A third shape: fewer rows, shared memory for 3 CTAs per SM (degrees 1-3)
  // and registers capped to match.
  template <int P>
  struct TileShapeSmall;
  template <>
  struct TileShapeSmall<1>
  {
    static constexpr int CX = 48, CY = 16, KX = 6, KY = 4;
    static constexpr int MIN_CTAS = 3;
  };
  template <>
  struct TileShapeSmall<2>
  {
    static constexpr int CX = 24, CY = 8, KX = 3, KY = 2;
    static constexpr int MIN_CTAS = 3;
  };
  template <>
  struct TileShapeSmall<3>
  {
    static constexpr int CX = 16, CY = 6, KX = 2, KY = 2;
    static constexpr int MIN_CTAS = 3;
  };
  template <>
  struct TileShapeSmall<4>
  {
    static constexpr int CX = 16, CY = 4, KX = 2, KY = 1;
    static constexpr int MIN_CTAS = 2;
  };

  template <int P, typename S = TileShape<P>>
  struct Tile
  {
    static constexpr int CX = S::CX, CY = S::CY;
    static constexpr int KX = S::KX, KY = S::KY;
    static constexpr int TX = P * CX, TY = P * CY;         // own nodes
    static constexpr int FX = TX + P + 1, FY = TY + P + 1; // footprint
    static constexpr int PF = FX | 1;                      // odd row pitch: conflict-free column access
    static constexpr int PY = TX | 1;                      // row pitch of the x-pass outputs
    static constexpr int SX = P * KX, SY = P * KY;         // segment lengths (nodes)
    static constexpr int NSX = TX / SX, NSY = TY / SY;     // segments per row / column
    static constexpr int NF = PF * FY;                     // doubles of one staged field
    static constexpr int NY = PY * FY;                     // doubles of one x-pass output array
    static constexpr int YL = (TX + 31) / 32 * 32;         // y-pass lanes per segment row
    static_assert(FY <= 32, "footprint rows must fit one warp");
    static_assert(TX % SX == 0 && TY % SY == 0, "segments must tile the own nodes");
    static_assert(NSX * 32 <= THREADS && NSY * YL <= THREADS, "one pass round per CTA");
  };

  struct Grid
  {
    int nfx, nfy; // nodes per axis, images included
    int nux, nuy; // distinct nodes per axis (the wrap modulus of a periodic axis)
    int ncx, ncy; // cells per axis
    int px, py;
    long long N;
    // Node rows [oy0, oy1) that this context owns. The whole grid for one
    // context; a y-strip of a mesh split over several contexts owns its strip,
    // and its rows outside are ghost copies of the neighbours' (lbfem_gpu_set_strip).
    // Sums over nodes (CG dot products, conservation) count the owned rows only.
    int oy0, oy1;
  };

  __device__ __forceinline__ bool
  owned_row(int j, const Grid &g)
  {
    return j >= g.oy0 && j < g.oy1;
  }

  // Everything a kernel needs to know about the discretisation.
  struct Geo
  {
    Grid g;
    const double *hx, *hxi, *hy, *hyi;   // cell widths and their inverses
    const double *ijx, *ijy;             // inverse Jacobi diagonal per axis (1 on images)
    const double *ilx, *ily;             // inverse lumped diagonal per axis (1 on images)
    const double *lumpx, *lumpy;         // lumped diagonal per axis (node weights)
    const double *diagx, *diagy;         // Jacobi diagonal per axis
    const double *rowx, *rowy;           // assembled 1-D rows [4][n][2p+1] (M, C, C^T, K), wall faces
    const uint8_t *wall;                 // per node: 0 fluid, k > 0 wall with velocity wall_u[2(k-1)..]; may be null
    const double *wall_u;
    // general quadrilaterals only (else null): per node lumped diagonal and inverse Jacobi diagonal
    const double *lump2, *ijac2;
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

  // FP32 deviation form: d_a = f_a - w_a (rest state rho0 = 1). Exact in real
  // arithmetic: rho = 1 + sum d, momentum = sum e d, and
  // feq_a - w_a = w_a (drho + rho (3 e.u + 4.5 (e.u)^2 - 1.5 u.u)).
  struct MomF
  {
    float rho, ux, uy, drho;
  };

  // The D2Q9 directions and weights as compile-time FP32 values: literal
  // operands in the FP32 kernels instead of constant-bank loads and FP64->FP32
  // conversions (the weights are the FP64 values rounded to FP32, as before).
  __device__ constexpr float kEXf[Q] = {0, 1, 1, 0, -1, -1, -1, 0, 1};
  __device__ constexpr float kEYf[Q] = {0, 0, 1, 1, 1, 0, -1, -1, -1};
  __device__ constexpr float kWf[Q] = {float(4. / 9.),  float(1. / 9.),  float(1. / 36.), float(1. / 9.), float(1. / 36.),
                            float(1. / 9.),  float(1. / 36.), float(1. / 9.),  float(1. / 36.)};
  // The weights' FP32 rounding errors (w - kWf, rounded to FP32). All nine FP32
  // weights are 4 / 9, 1 / 9 and 1 / 36 rounded up by the same relative 7.45e-9, so
  // their sum and their second moments exceed 1 and 1 / 3 by that much. A
  // product w t rounded once from kWf t would give every equilibrium that excess
  // of mass and momentum: a bias that the collisions add up step after step,
  // about 7.5e-9 of the velocity per step. Formed as fma(kWf, t, kWlf t), the
  // product is the exact weight's, rounded once, with no common bias.
  constexpr double kW64[Q] = {4. / 9., 1. / 9., 1. / 36., 1. / 9., 1. / 36., 1. / 9., 1. / 36., 1. / 9., 1. / 36.};
  __device__ constexpr float kWlf[Q] = {
    float(kW64[0] - double(float(kW64[0]))), float(kW64[1] - double(float(kW64[1]))),
    float(kW64[2] - double(float(kW64[2]))), float(kW64[3] - double(float(kW64[3]))),
    float(kW64[4] - double(float(kW64[4]))), float(kW64[5] - double(float(kW64[5]))),
    float(kW64[6] - double(float(kW64[6]))), float(kW64[7] - double(float(kW64[7]))),
    float(kW64[8] - double(float(kW64[8])))};

  // w t for the weight w = wh + wl (wh its FP32 rounding, wl the rest), rounded once
  __device__ __forceinline__ float
  wmul(float wh, float wl, float t)
  {
    return fmaf(wh, t, wl * t);
  }

  // The momentum sums in the order of the loop over a with e_a in {-1, 0, 1}
  // (the zero terms dropped: adding +-0 changes no value).
  __device__ __forceinline__ MomF
  moments_dev(const float (&d)[Q])
  {
    float drho = 0;
#pragma unroll
    for (int a = 0; a < Q; ++a)
      drho += d[a];
    const float mx = ((((d[1] + d[2]) - d[4]) - d[5]) - d[6]) + d[8];
    const float my = ((((d[2] + d[3]) + d[4]) - d[6]) - d[7]) - d[8];
    const float rho = 1.f + drho;
    return {rho, mx / rho, my / rho, drho};
  }

  // feq - w of the direction (ex, ey) with weight w = wh + wl.
  __device__ __forceinline__ float
  feqd(float ex, float ey, float wh, float wl, const MomF &m)
  {
    const float uu = m.ux * m.ux + m.uy * m.uy;
    const float eu = ex * m.ux + ey * m.uy;
    return wmul(wh, wl, m.drho + m.rho * (3.f * eu + 4.5f * eu * eu - 1.5f * uu));
  }

  __device__ __forceinline__ float
  feqd_a(int a, const MomF &m)
  {
    return feqd(kEXf[a], kEYf[a], kWf[a], kWlf[a], m);
  }

  // What a node imposes on its moments (collision.h:53-72).
  __device__ __forceinline__ Mom
  impose_class(Mom m, int k, const Geo &geo)
  {
    if (k)
      {
        m.ux = geo.wall_u[2 * (k - 1)];
        m.uy = geo.wall_u[2 * (k - 1) + 1];
      }
    return m;
  }

  __device__ __forceinline__ Mom
  impose(Mom m, long long idx, const Geo &geo)
  {
    return geo.wall ? impose_class(m, geo.wall[idx], geo) : m;
  }

  __device__ __forceinline__ MomF
  impose_class(MomF m, int k, const Geo &geo)
  {
    if (k)
      {
        m.ux = float(geo.wall_u[2 * (k - 1)]);
        m.uy = float(geo.wall_u[2 * (k - 1) + 1]);
      }
    return m;
  }

  __device__ __forceinline__ MomF
  impose(MomF m, long long idx, const Geo &geo)
  {
    return geo.wall ? impose_class(m, geo.wall[idx], geo) : m;
  }

  // Counters that outlive one solve: the first failure of any solve (sticky:
  // a CgState status, 4 = stagnation), CG iterations / mixed corrections summed
  // over systems and solves, loop-body runs of graph-launched solves, and the
  // steps completed.
  struct DevStats
  {
    int sticky;
    int pad;
    unsigned long long its, bodies, steps_done;
  };

  // The nodal update that completes a step (or a sweep of it): skipped after a
  // failure (the populations stay those before the failing step); with count,
  // block 0 counts the step.
  __device__ __forceinline__ bool
  step_skipped(DevStats *ds, bool count = true)
  {
    if (!ds)
      return false;
    if (ds->sticky)
      return true;
    if (count && blockIdx.x == 0 && threadIdx.x == 0)
      atomicAdd(&ds->steps_done, 1ULL);
    return false;
  }

  // ---------------------------------------------------- fixed-order reductions
  // Sums v[0..NQ) over the CTA (warp shuffles, then warp 0) and stores the CTA
  // totals at partials[q * n_blocks + block].
  template <int NQ>
  __device__ __forceinline__ void
  block_reduce_store(double (&v)[NQ], double *partials, int block, int n_blocks)
  {
    __shared__ double warp_sum[NQ][THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      {
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
#pragma unroll
        for (int q = 0; q < NQ; ++q)
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

  // The same for a CTA of NT threads (NT a multiple of 32, at most 1024).
  template <int NQ, int NT>
  __device__ __forceinline__ void
  block_reduce_store_n(double (&v)[NQ], double *partials, int block, int n_blocks)
  {
    static_assert(NT % 32 == 0 && NT <= 1024, "whole warps");
    __shared__ double warp_sum[NQ][NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      {
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
#pragma unroll
        for (int q = 0; q < NQ; ++q)
          {
            double s = lane < NT / 32 ? warp_sum[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
              s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0)
              partials[(long long)q * n_blocks + block] = s;
          }
      }
    __syncthreads();
  }

  // One CTA per quantity q: out[q] = sum_b partials[q * n_blocks + b], in a fixed order.
  __global__ void
  k_reduce_partials(const double *__restrict__ partials, int n_blocks, double *__restrict__ out);

  // Quantity q of the partials (one CTA; the body of k_reduce_partials and of its batched form).
  __device__ __forceinline__ void
  reduce_partials_q(const double *__restrict__ partials, int n_blocks, double *__restrict__ out, int q)
  {
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
  }

  __global__ void
  k_reduce_partials(const double *__restrict__ partials, int n_blocks, double *__restrict__ out)
  {
    reduce_partials_q(partials, n_blocks, out, blockIdx.x);
  }

  // ------------------------------------------------------ asynchronous copies
  // A 4-byte global -> shared copy that does not hold a register until it
  // lands (cp.async, sm_80+); valid = false writes zero and reads nothing.
  __device__ __forceinline__ void
  cp_async4(void *smem, const void *gmem, bool valid)
  {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0)
                 : "memory");
  }

  __device__ __forceinline__ void
  cp_async_wait_all()
  {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }

  __device__ __forceinline__ void
  cp_async_commit()
  {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }

  // Waits until at most N committed groups of this thread are still in flight.
  template <int N>
  __device__ __forceinline__ void
  cp_async_wait_group()
  {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
  }

  // ------------------------------------------------------------ tile staging
  // Per-CTA tables of the footprint: source column and row offset of every
  // footprint column/row (-1 outside a non-periodic domain), the widths of the
  // CX+1 / CY+1 footprint cells and their inverses (0 outside the domain).
  template <int P, typename R = double, typename S = TileShape<P>>
  struct TileMaps
  {
    int col[Tile<P, S>::FX];
    int rowi[Tile<P, S>::FY];
    int row[Tile<P, S>::FY]; // storage offset of the row (a population array holds fewer than 2^31 nodes)
    R hx[Tile<P, S>::CX + 1], hxi[Tile<P, S>::CX + 1], cx[Tile<P, S>::CX + 1];
    R hy[Tile<P, S>::CY + 1], hyi[Tile<P, S>::CY + 1], cy[Tile<P, S>::CY + 1];
    double ijx[Tile<P, S>::FX], ijy[Tile<P, S>::FY]; // inverse Jacobi diagonal factors of the footprint's storage nodes
  };

  template <int P, typename R, typename S>
  __device__ __forceinline__ void
  build_maps(TileMaps<P, R, S> &m, const Geo &geo, int gx0, int gy0)
  {
    using T = Tile<P, S>;
    const Grid &g = geo.g;
    for (int t = threadIdx.x; t < T::FX; t += blockDim.x)
      {
        const int c = wrap(gx0 - P + t, g.px, g.nux, g.nfx);
        m.col[t] = c;
        m.ijx[t] = c < 0 ? 0.0 : geo.ijx[c];
      }
    for (int t = threadIdx.x; t < T::FY; t += blockDim.x)
      {
        const int r = wrap(gy0 - P + t, g.py, g.nuy, g.nfy);
        m.rowi[t] = r;
        m.row[t] = r < 0 ? -1 : r * g.nfx;
        m.ijy[t] = r < 0 ? 0.0 : geo.ijy[r];
      }
    const int cx0 = gx0 / P - 1, cy0 = gy0 / P - 1;
    for (int t = threadIdx.x; t <= T::CX; t += blockDim.x)
      {
        const int c = wrap(cx0 + t, g.px, g.ncx, g.ncx);
        m.hx[t] = R(c < 0 ? 0.0 : geo.hx[c]);
        m.hxi[t] = R(c < 0 ? 0.0 : geo.hxi[c]);
        m.cx[t] = R(c < 0 ? 0.0 : 1.0);
      }
    for (int t = threadIdx.x; t <= T::CY; t += blockDim.x)
      {
        const int c = wrap(cy0 + t, g.py, g.ncy, g.ncy);
        m.hy[t] = R(c < 0 ? 0.0 : geo.hy[c]);
        m.hyi[t] = R(c < 0 ? 0.0 : geo.hyi[c]);
        m.cy[t] = R(c < 0 ? 0.0 : 1.0);
      }
  }

  // s[fy*PF + fx] <- op(storage index) over the footprint (0 outside the domain).
  template <int P, typename R, typename RM, typename F>
  __device__ __forceinline__ void
  stage(R *s, const TileMaps<P, RM> &m, F &&value_at)
  {
    using T = Tile<P>;
    // all loads of a thread are issued before its first shared store (memory-level parallelism)
    constexpr int NT = T::FY * T::FX, IT = (NT + THREADS - 1) / THREADS;
    R v[IT];
    int si[IT]; // shared-memory index of each element (the division is done once)
#pragma unroll
    for (int k = 0; k < IT; ++k)
      {
        const int t = threadIdx.x + k * THREADS;
        v[k] = R{};
        si[k] = -1;
        if (t < NT)
          {
            const int fy = t / T::FX, fx = t - fy * T::FX;
            si[k] = fy * T::PF + fx;
            const int r = m.row[fy];
            const int c = m.col[fx];
            if (r >= 0 && c >= 0)
              v[k] = R(value_at(r + c));
          }
      }
#pragma unroll
    for (int k = 0; k < IT; ++k)
      if (si[k] >= 0)
        s[si[k]] = v[k];
  }

  // The same with the storage coordinates and the footprint position:
  // value_at(storage index, column, row, footprint column, footprint row).
  template <int P, typename R, typename RM, typename F>
  __device__ __forceinline__ void
  stage_ij(R *s, const TileMaps<P, RM> &m, F &&value_at)
  {
    using T = Tile<P>;
    constexpr int NT = T::FY * T::FX, IT = (NT + THREADS - 1) / THREADS;
    R v[IT];
    int si[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k)
      {
        const int t = threadIdx.x + k * THREADS;
        v[k] = R{};
        si[k] = -1;
        if (t < NT)
          {
            const int fy = t / T::FX, fx = t - fy * T::FX;
            si[k] = fy * T::PF + fx;
            const int r = m.row[fy];
            const int c = m.col[fx];
            if (r >= 0 && c >= 0)
              v[k] = R(value_at(r + c, c, m.rowi[fy], fx, fy));
          }
      }
#pragma unroll
    for (int k = 0; k < IT; ++k)
      if (si[k] >= 0)
        s[si[k]] = v[k];
  }

  // s[i*TX + j] <- src at own node (gx0 + j, gy0 + i) of the tile (0 past the grid).
  template <int P, typename R>
  __device__ __forceinline__ void
  stage_own(R *s, const R *__restrict__ src, const Grid &g, int gx0, int gy0)
  {
    using T = Tile<P>;
    constexpr int NT = T::TY * T::TX, IT = (NT + THREADS - 1) / THREADS;
    R v[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k)
      {
        const int t = threadIdx.x + k * THREADS;
        const int i = t / T::TX, j = t - i * T::TX;
        const int gx = gx0 + j, gy = gy0 + i;
        v[k] = (t < NT && gx < g.nfx && gy < g.nfy) ? src[gy * g.nfx + gx] : R(0); // fewer than 2^31 nodes
      }
#pragma unroll
    for (int k = 0; k < IT; ++k)
      {
        const int t = threadIdx.x + k * THREADS;
        if (t < NT)
          s[t] = v[k];
      }
  }

  // y[a] = sum_b R[a][b] u[b] for the reference element matrix OP.
  template <int P, int OP, typename R>
  __device__ __forceinline__ void
  elem(const R (&u)[P + 1], R (&y)[P + 1])
  {
#pragma unroll
    for (int a = 0; a <= P; ++a)
      {
        R s = ref<R, P, OP>(a, 0) * u[0];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          s = fma(ref<R, P, OP>(a, b), u[b], s);
        y[a] = s;
      }
  }

  // The last row (right vertex) only.
  template <int P, int OP, typename R>
  __device__ __forceinline__ R
  elem_last(const R (&u)[P + 1])
  {
    R s = ref<R, P, OP>(P, 0) * u[0];
#pragma unroll
    for (int b = 1; b <= P; ++b)
      s = fma(ref<R, P, OP>(P, b), u[b], s);
    return s;
  }

  // The x pass of a mass-type operator (OP_M with the cell width as scale) on one
  // footprint row and one x segment: out[fy*PY + j] for the segment's own columns j.
  template <int P, typename R>
  __device__ __forceinline__ void
  mass_xpass(const R *__restrict__ s, R *__restrict__ out, const TileMaps<P, R> &m, int fy, int seg)
  {
    using T = Tile<P>;
    const R *row = s + fy * T::PF;
    R *orow = out + fy * T::PY;
    const int q0 = seg * T::KX; // halo cell (footprint cell index)
    R u[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      u[b] = row[q0 * P + b];
    R pend = m.hx[q0] * elem_last<P, OP_M>(u);
#pragma unroll
    for (int q = 1; q <= T::KX; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          u[b] = row[qc * P + b];
        R y[P + 1];
        elem<P, OP_M>(u, y);
        const R sc = m.hx[qc];
        const int j0 = (qc - 1) * P;
        orow[j0] = fma(sc, y[0], pend);
#pragma unroll
        for (int a = 1; a < P; ++a)
          orow[j0 + a] = sc * y[a];
        pend = sc * y[P];
      }
  }

  // The y pass of a mass-type operator on column j and y segment seg: calls
  // emit(own row i, value) for the segment's SY own rows.
  template <int P, typename R, typename Emit>
  __device__ __forceinline__ void
  mass_ypass(const R *__restrict__ t, const TileMaps<P, R> &m, int j, int seg, Emit &&emit)
  {
    using T = Tile<P>;
    const int q0 = seg * T::KY;
    R u[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      u[b] = t[(q0 * P + b) * T::PY + j];
    R pend = m.hy[q0] * elem_last<P, OP_M>(u);
#pragma unroll
    for (int q = 1; q <= T::KY; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          u[b] = t[(qc * P + b) * T::PY + j];
        R y[P + 1];
        elem<P, OP_M>(u, y);
        const R sc = m.hy[qc];
        const int i0 = (qc - 1) * P;
        emit(i0, fma(sc, y[0], pend));
#pragma unroll
        for (int a = 1; a < P; ++a)
          emit(i0 + a, sc * y[a]);
        pend = sc * y[P];
      }
  }
} // namespace lbfem_gpu
