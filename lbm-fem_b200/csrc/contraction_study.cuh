// The sum-factorisation contraction of the streaming right-hand side's x pass,
// on CUDA cores and on tensor cores, for the design decision between the two
// (measured by bench.py --contraction-study and ncu; no step uses these
// kernels).
//
// The contraction: along every node row, for every cell, the four element
// operators of the x pass applied to the cell's p+1 values of two fields,
//   Ch = Chat h, Mh = Mhat h, Ku = Khat u, Mu = Mhat u,
// summed into the assembled rows y1 = Ch + Ku and y2 = Mh + Mu (the shared
// vertex of two cells takes both cells' contributions). A CTA owns 32 node rows
// and 64 cells; it stages one cell more on the left (the contributions to its
// first vertex) and rounds the cells up to 72, a multiple of the 8 cells one
// tensor-core tile takes.
//
// Tensor-core forms:
//  - FP32: mma.sync m16n8k8 TF32 with a three-term split (a = a_hi + a_lo in
//    TF32; D = A_hi B_hi + A_hi B_lo + A_lo B_hi), which keeps FP32 accuracy.
//    A (16 x 8) stacks [Chat 0; Mhat 0; 0 Khat; 0 Mhat] (rows: the four
//    operators' outputs, columns: the cell's h then u nodes); B (8 x 8) holds
//    8 cells' h and u (p = 3: all 8 rows of K used; p = 2: 6);
//  - FP64: mma.sync m8n8k4 (DMMA) twice, [Chat; Mhat] on h and [Khat; Mhat]
//    on u, K = 4 = the p + 1 nodes of a cell at p = 3 (p = 2: 3 of 4 used).
#pragma once

#include <cstdint>

namespace lbfem_gpu
{
  namespace study
  {
    constexpr int ROWS = 32, NT = 256;

    // cells a CTA owns and the cells it stages (one more on the left, rounded up
    // to tiles of 8): fewer in FP64, whose tiles fill shared memory twice as fast
    template <typename R>
    __host__ __device__ constexpr int
    cells_of()
    {
      return sizeof(R) == sizeof(float) ? 64 : 32;
    }

    template <typename R>
    struct Mats
    {
      R M[5][5], C[5][5], K[5][5];
    };

    template <typename R>
    __host__ __device__ constexpr int
    cpad()
    {
      return cells_of<R>() + 8;
    }

    template <int P, typename R>
    __host__ __device__ constexpr int
    pitch()
    {
      return (P * cpad<R>() + 1) | 1; // odd: conflict-free column walks
    }

    template <int P, typename R>
    __host__ __device__ constexpr size_t
    smem()
    {
      // u, h, y1, y2 tiles and the right-vertex partials of y1, y2
      return sizeof(R) * (4 * ROWS * pitch<P, R>() + 2 * ROWS * cpad<R>());
    }

    // In both forms the right-vertex partial of cell n goes to side[n] and the
    // other p nodes to their own positions; after a barrier the kernel folds the
    // partials into the next cell's first node.

    // CUDA cores: thread (row = tid / 8, part = tid % 8) takes 9 cells of its row.
    template <int P, typename R>
    __device__ __forceinline__ void
    contract_cuda(const R *s_u, const R *s_h, R *s_y1, R *s_y2, R *s_s1, R *s_s2, const Mats<R> &m)
    {
      const int row = threadIdx.x / 8, part = threadIdx.x % 8;
      for (int n = part * (cpad<R>() / 8); n < (part + 1) * (cpad<R>() / 8); ++n)
        {
          R u[P + 1], h[P + 1];
#pragma unroll
          for (int b = 0; b <= P; ++b)
            {
              u[b] = s_u[row * pitch<P, R>() + P * n + b];
              h[b] = s_h[row * pitch<P, R>() + P * n + b];
            }
#pragma unroll
          for (int a = 0; a <= P; ++a)
            {
              R ch = 0, mh = 0, ku = 0, mu = 0;
#pragma unroll
              for (int b = 0; b <= P; ++b)
                {
                  ch = fma(m.C[a][b], h[b], ch);
                  mh = fma(m.M[a][b], h[b], mh);
                  ku = fma(m.K[a][b], u[b], ku);
                  mu = fma(m.M[a][b], u[b], mu);
                }
              if (a < P)
                {
                  s_y1[row * pitch<P, R>() + P * n + a] = ch + ku;
                  s_y2[row * pitch<P, R>() + P * n + a] = mh + mu;
                }
              else
                {
                  s_s1[row * cpad<R>() + n] = ch + ku;
                  s_s2[row * cpad<R>() + n] = mh + mu;
                }
            }
        }
    }

    __device__ __forceinline__ uint32_t
    tf32(float x)
    {
      uint32_t r;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
      return r;
    }

    // x = hi + lo, both TF32 (the three-term split keeps FP32 accuracy)
    __device__ __forceinline__ void
    split(float x, uint32_t &hi, uint32_t &lo)
    {
      hi = tf32(x);
      lo = tf32(x - __uint_as_float(hi));
    }

    __device__ __forceinline__ void
    mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
    {
      asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                   "{%0,%1,%2,%3};"
                   : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                   : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }

    __device__ __forceinline__ void
    mma_f64(double (&d)[2], double a, double b)
    {
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(d[0]), "+d"(d[1])
                   : "d"(a), "d"(b));
    }

    // Entry (r, k) of the stacked 16 x 8 operator of the TF32 form.
    template <int P>
    __device__ __forceinline__ float
    stacked(const Mats<float> &m, int r, int k)
    {
      const int op = r / 4, a = r % 4, b = k % 4;
      if (a > P || b > P || (op < 2) != (k < 4))
        return 0.f;
      return op == 0 ? m.C[a][b] : op == 2 ? m.K[a][b] : m.M[a][b];
    }

    // The D fragment of 8 cells of one row into y (nodes a < p) and the sides (a = p).
    template <int P, typename R>
    __device__ __forceinline__ void
    store_fragment(R *s_y1, R *s_y2, R *s_s1, R *s_s2, int row, int n0, int g, int t, R v0, R v1)
    {
      const int a = g % 4;
      if (a > P)
        return;
      R *y = g < 4 ? s_y1 : s_y2, *side = g < 4 ? s_s1 : s_s2;
      const int n = n0 + 2 * t;
      if (a < P)
        {
          y[row * pitch<P, R>() + P * n + a] = v0;
          y[row * pitch<P, R>() + P * (n + 1) + a] = v1;
        }
      else
        {
          side[row * cpad<R>() + n] = v0;
          side[row * cpad<R>() + n + 1] = v1;
        }
    }

    // Tensor cores: warp w takes rows 4w .. 4w + 3, 8 cells per tile.
    template <int P>
    __device__ __forceinline__ void
    contract_tc(const float *s_u, const float *s_h, float *s_y1, float *s_y2, float *s_s1, float *s_s2,
                const Mats<float> &m)
    {
      using R = float;
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
      uint32_t ahi[4], alo[4];
      const float av[4] = {stacked<P>(m, g, t), stacked<P>(m, g + 8, t), stacked<P>(m, g, t + 4),
                           stacked<P>(m, g + 8, t + 4)};
#pragma unroll
      for (int q = 0; q < 4; ++q)
        split(av[q], ahi[q], alo[q]);
      for (int row = 4 * warp; row < 4 * warp + 4; ++row)
        for (int n0 = 0; n0 < cpad<R>(); n0 += 8)
          {
            const int base = row * pitch<P, R>() + P * (n0 + g) + t;
            const float hv = t <= P ? s_h[base] : 0.f, uv = t <= P ? s_u[base] : 0.f;
            uint32_t bh_hi, bh_lo, bu_hi, bu_lo;
            split(hv, bh_hi, bh_lo);
            split(uv, bu_hi, bu_lo);
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            mma_tf32(d, alo, bh_hi, bu_hi);
            mma_tf32(d, ahi, bh_lo, bu_lo);
            mma_tf32(d, ahi, bh_hi, bu_hi);
            // rows g (Ch or Mh) and g + 8 (Ku or Mu) of the same node and cells
            store_fragment<P, float>(s_y1, s_y2, s_s1, s_s2, row, n0, g, t, d[0] + d[2], d[1] + d[3]);
          }
    }

    template <int P>
    __device__ __forceinline__ void
    contract_tc(const double *s_u, const double *s_h, double *s_y1, double *s_y2, double *s_s1, double *s_s2,
                const Mats<double> &m)
    {
      using R = double;
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
      const int a = g % 4;
      // [Chat; Mhat] on h and [Khat; Mhat] on u, row g of each
      const double ah = (a > P || t > P) ? 0.0 : (g < 4 ? m.C[a][t] : m.M[a][t]);
      const double au = (a > P || t > P) ? 0.0 : (g < 4 ? m.K[a][t] : m.M[a][t]);
      for (int row = 4 * warp; row < 4 * warp + 4; ++row)
        for (int n0 = 0; n0 < cpad<R>(); n0 += 8)
          {
            const int base = row * pitch<P, R>() + P * (n0 + g) + t;
            const double hv = t <= P ? s_h[base] : 0.0, uv = t <= P ? s_u[base] : 0.0;
            double d[2] = {0.0, 0.0};
            mma_f64(d, ah, hv);
            mma_f64(d, au, uv);
            store_fragment<P, double>(s_y1, s_y2, s_s1, s_s2, row, n0, g, t, d[0], d[1]);
          }
    }

    // One CTA: 32 node rows and 64 cells of an nrow x (p ncell + 1) grid of two
    // fields; y1, y2 receive the CTA's own nodes.
    template <int P, typename R, bool TC>
    __global__ void __launch_bounds__(NT)
      k_xpass_study(const R *__restrict__ u, const R *__restrict__ h, R *__restrict__ y1, R *__restrict__ y2,
                    int nrow, int ncell, const Mats<R> m)
    {
      extern __shared__ __align__(16) unsigned char raw[];
      constexpr int PF = pitch<P, R>();
      R *s_u = reinterpret_cast<R *>(raw), *s_h = s_u + ROWS * PF, *s_y1 = s_h + ROWS * PF, *s_y2 = s_y1 + ROWS * PF;
      R *s_s1 = s_y2 + ROWS * PF, *s_s2 = s_s1 + ROWS * cpad<R>();
      const int ncol = P * ncell + 1;
      const int r0 = blockIdx.y * ROWS, col0 = P * (int(blockIdx.x) * cells_of<R>() - 1); // local cell 0: one cell left
      for (int e = threadIdx.x; e < ROWS * (P * cpad<R>() + 1); e += NT)
        {
          const int row = e / (P * cpad<R>() + 1), j = e - row * (P * cpad<R>() + 1);
          const int gr = r0 + row, gc = col0 + j;
          const bool ok = gr < nrow && gc >= 0 && gc < ncol;
          const long long gi = ok ? (long long)gr * ncol + gc : 0;
          s_u[row * PF + j] = ok ? u[gi] : R(0);
          s_h[row * PF + j] = ok ? h[gi] : R(0);
        }
      __syncthreads();
      if constexpr (TC)
        contract_tc<P>(s_u, s_h, s_y1, s_y2, s_s1, s_s2, m);
      else
        contract_cuda<P, R>(s_u, s_h, s_y1, s_y2, s_s1, s_s2, m);
      __syncthreads();
      for (int e = threadIdx.x; e < ROWS * (cpad<R>() - 1); e += NT)
        {
          const int row = e / (cpad<R>() - 1), n = e - row * (cpad<R>() - 1);
          s_y1[row * PF + P * (n + 1)] += s_s1[row * cpad<R>() + n];
          s_y2[row * PF + P * (n + 1)] += s_s2[row * cpad<R>() + n];
        }
      __syncthreads();
      // own nodes: local [P, P + P cells_of<R>())
      for (int e = threadIdx.x; e < ROWS * P * cells_of<R>(); e += NT)
        {
          const int row = e / (P * cells_of<R>()), j = P + (e - row * (P * cells_of<R>()));
          const int gr = r0 + row, gc = col0 + j;
          if (gr < nrow && gc < ncol)
            {
              const long long gi = (long long)gr * ncol + gc;
              y1[gi] = s_y1[row * PF + j];
              y2[gi] = s_y2[row * PF + j];
            }
        }
    }

    // A deterministic smooth pattern on the grid (no host copy).
    template <typename R>
    __global__ void
    k_study_fill(R *u, R *h, long long n)
    {
      for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
          u[i] = R(sin(1e-3 * double(i)));
          h[i] = R(cos(7e-4 * double(i)) * 0.5);
        }
    }
  } // namespace study
} // namespace lbfem_gpu
