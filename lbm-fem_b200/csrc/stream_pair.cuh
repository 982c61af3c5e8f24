// The FP32 streaming right-hand side (K1) of the mixed-precision path, on
// pairs of opposite populations.
//
// D2Q9 population a and its opposite abar = a + 4 (a = 1..4) have opposite
// lattice velocities, so every operator of the grouped tensor-product form
// (see k_advection) applies to both with the same matrices, and the
// coefficients differ at most in sign:
//   k1 = ex, k3 = ey flip sign; c ex^2, -2 c ex ey, c ey^2, c ex ey do not.
// The kernel stages each pair as float2 {u_a, u_abar} and runs the x and y
// passes with packed FP32 arithmetic (fma.rn.f32x2, sm_100): one instruction,
// one shared-memory access and one barrier serve two populations (the
// element-matrix products of degree 3 and 4 excepted, see elem2_row). In the
// Lee-Lin right-hand side the equilibria of a pair share their even part:
//   feq_a - w = E + O, feq_abar - w = E - O,
//   E = w (drho + rho (4.5 (e.u)^2 - 1.5 u.u)), O = 3 w rho e.u;
// the Bardow collision, which writes the state, takes each population's own.
// Storage is the FP32 deviation d = f - w (advection annihilates constants).
#pragma once

#include "operators.cuh"

namespace lbfem_gpu
{
  // ----------------------------------------------------- packed FP32 arithmetic
  __device__ __forceinline__ unsigned long long
  pk(float2 v)
  {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
    return r;
  }

  __device__ __forceinline__ float2
  upk(unsigned long long r)
  {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
  }

  // a * b + c, both lanes, one rounding each
  __device__ __forceinline__ float2
  fma2(float2 a, float2 b, float2 c)
  {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
    return upk(d);
  }

  __device__ __forceinline__ float2
  mul2(float2 a, float2 b)
  {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
  }

  __device__ __forceinline__ float2
  add2(float2 a, float2 b)
  {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
    return upk(d);
  }

  __device__ __forceinline__ float2
  bc(float s)
  {
    return make_float2(s, s);
  }

  // Reference element matrices in FP32, each entry duplicated into both lanes.
  __device__ __constant__ float2 c_ref2[MAXPD][3][MAXPD + 1][MAXPD + 1];

  template <int P, int OP>
  __device__ __forceinline__ float2
  ref2(int a, int b)
  {
    return c_ref2[P - 1][OP][a][b];
  }

  // Row a of reference matrix OP applied to u, both lanes. The matrix entries
  // are uniform constants. From degree 3 on they enter as scalar FMA operands
  // read from constant memory (two FP32 FMAs per entry): the packed form
  // needs each entry as a lane-duplicated register pair, and at p = 4 those
  // pairs spill (p = 4 K1 1.3x faster scalar, p = 3 even). Below degree 3 the
  // packed form is kept (about 1% faster there).
  template <int P, int OP>
  __device__ __forceinline__ float2
  elem2_row(int a, const float2 (&u)[P + 1])
  {
    if constexpr (P >= 3)
      {
        float c = ref<float, P, OP>(a, 0);
        float sx = c * u[0].x, sy = c * u[0].y;
#pragma unroll
        for (int b = 1; b <= P; ++b)
          {
            c = ref<float, P, OP>(a, b);
            sx = fmaf(c, u[b].x, sx);
            sy = fmaf(c, u[b].y, sy);
          }
        return make_float2(sx, sy);
      }
    else
      {
        float2 s = mul2(ref2<P, OP>(a, 0), u[0]);
#pragma unroll
        for (int b = 1; b <= P; ++b)
          s = fma2(ref2<P, OP>(a, b), u[b], s);
        return s;
      }
  }

  template <int P, int OP>
  __device__ __forceinline__ void
  elem2(const float2 (&u)[P + 1], float2 (&y)[P + 1])
  {
#pragma unroll
    for (int a = 0; a <= P; ++a)
      y[a] = elem2_row<P, OP>(a, u);
  }

  template <int P, int OP>
  __device__ __forceinline__ float2
  elem2_last(const float2 (&u)[P + 1])
  {
    return elem2_row<P, OP>(P, u);
  }

  // Per-cell scales of the footprint, lane-duplicated: width, 1 / width, and 1 / 0 for
  // a cell inside / outside the domain.
  template <int P, typename S = TileShape<P>>
  struct PairScales
  {
    float2 hx[Tile<P, S>::CX + 1], hxi[Tile<P, S>::CX + 1], cx[Tile<P, S>::CX + 1];
    float2 hy[Tile<P, S>::CY + 1], hyi[Tile<P, S>::CY + 1], cy[Tile<P, S>::CY + 1];
  };

  // The pair's coefficients: h = A u + B feq; k1..k6 of the grouped operator.
  struct PairK
  {
    float2 A, B, k1, k2, k3, k4, k5, k6;
  };

  enum
  {
    PAIR_LEELIN = 0, // Lee-Lin step: r of f with the equilibria (wall velocity imposed) computed on the fly
    PAIR_BARDOW = 1  // Bardow step: collide_bgk on the fly, write g*, then r of g*
  };

  template <int P, int MODE, typename S = TileShape<P>>
  constexpr size_t
  pair_smem()
  {
    using T = Tile<P, S>;
    // moments [4][NF] float, pair [2][NF] float2 (double-buffered), x-pass outputs [3][NY] float2,
    // Y4 [2][TX] float2, walls [NF] bytes
    return sizeof(float) * 4 * T::NF + sizeof(float2) * (2 * T::NF + 3 * T::NY + 2 * T::TX) +
           (MODE == PAIR_BARDOW ? size_t(T::NF + 15) / 16 * 16 : 0);
  }

  // u and h = A u + B feq of the pair at footprint index t (Lee-Lin), or u and A u.
  template <int MODE>
  __device__ __forceinline__ void
  pair_uh(const float2 *s_u, const float *s_m, int nf, int t, float w, float wl, float ex, float ey, const PairK &k,
          float2 &u, float2 &h)
  {
    u = s_u[t];
    if constexpr (MODE == PAIR_LEELIN)
      {
        // staged: rho, ux, uy, base = drho - 1.5 rho u.u (wall velocity imposed)
        const float rho = s_m[t], ux = s_m[nf + t], uy = s_m[2 * nf + t], base = s_m[3 * nf + t];
        const float eu = fmaf(ey, uy, ex * ux), reu = rho * eu;
        const float E = wmul(w, wl, fmaf(4.5f * reu, eu, base)), O = 3.f * wmul(w, wl, reu);
        h = fma2(k.B, make_float2(E + O, E - O), mul2(k.A, u));
      }
    else
      h = mul2(k.A, u);
  }

  // x pass of one footprint row fy and one x segment. CLS: 0 e = (ex, 0), 1 e = (0, ey), 2 diagonal.
  // Each output node's operator rows are formed as they are stored (few live registers).
  template <int P, int CLS, int MODE, typename S>
  __device__ __forceinline__ void
  pair_xpass(const float2 *s_u, const float *s_m, float2 *s_y, float2 *s_y4, const PairScales<P, S> &m,
             const PairK &k, float w, float wl, float ex, float ey, int fy, int seg, int gx0, int y4_slot,
             int bx_lo, int bx_hi)
  {
    using T = Tile<P, S>;
    constexpr bool XC = CLS != 1, YC = CLS != 0, DG = CLS == 2;
    const int base = fy * T::PF;
    const int q0 = seg * T::KX;
    float2 u[P + 1], h[P + 1];
#pragma unroll
    for (int b = 0; b <= P; ++b)
      pair_uh<MODE>(s_u, s_m, T::NF, base + q0 * P + b, w, wl, ex, ey, k, u[b], h[b]);
    // pending right-vertex contributions of the previous cell
    float2 pCh{}, pKu{}, pMh{}, pCu{}, pMu{};
    if constexpr (XC)
      {
        pCh = mul2(m.cx[q0], elem2_row<P, OP_C>(P, h));
        pKu = mul2(m.hxi[q0], elem2_row<P, OP_K>(P, u));
      }
    if constexpr (YC)
      {
        pMh = mul2(m.hx[q0], elem2_row<P, OP_M>(P, h));
        pMu = mul2(m.hx[q0], elem2_row<P, OP_M>(P, u));
      }
    if constexpr (DG)
      pCu = mul2(m.cx[q0], elem2_row<P, OP_C>(P, u));
    float2 *y1 = s_y + fy * T::PY, *y2 = y1 + T::NY, *y3 = y2 + T::NY;
    // unrolled up to p = 3 (K1 3-5% faster); at p = 4 the unrolled loop spills
#pragma unroll(P >= 4 ? 1 : T::KX)
    for (int q = 1; q <= T::KX; ++q)
      {
        const int qc = q0 + q;
        u[0] = u[P];
        h[0] = h[P];
#pragma unroll
        for (int b = 1; b <= P; ++b)
          pair_uh<MODE>(s_u, s_m, T::NF, base + qc * P + b, w, wl, ex, ey, k, u[b], h[b]);
        const float2 sc = m.cx[qc], sh = m.hx[qc], shi = m.hxi[qc];
        const int j0 = (qc - 1) * P;
#pragma unroll
        for (int aa = 0; aa <= P; ++aa)
          {
            float2 vCh{}, vKu{}, vMh{}, vCu{}, vMu{};
            if constexpr (XC)
              {
                vCh = mul2(sc, elem2_row<P, OP_C>(aa, h));
                vKu = mul2(shi, elem2_row<P, OP_K>(aa, u));
              }
            if constexpr (YC)
              {
                vMh = mul2(sh, elem2_row<P, OP_M>(aa, h));
                vMu = mul2(sh, elem2_row<P, OP_M>(aa, u));
              }
            if constexpr (DG)
              vCu = mul2(sc, elem2_row<P, OP_C>(aa, u));
            if (aa == P)
              {
                // the right vertex: pending for the next cell
                pCh = vCh;
                pKu = vKu;
                pMh = vMh;
                pMu = vMu;
                pCu = vCu;
                break;
              }
            if (aa == 0)
              {
                if constexpr (XC)
                  {
                    vCh = add2(vCh, pCh);
                    vKu = add2(vKu, pKu);
                  }
                if constexpr (YC)
                  {
                    vMh = add2(vMh, pMh);
                    vMu = add2(vMu, pMu);
                  }
                if constexpr (DG)
                  vCu = add2(vCu, pCu);
              }
            const int j = j0 + aa;
            if constexpr (XC)
              y1[j] = fma2(k.k1, vCh, mul2(k.k2, vKu));
            if constexpr (YC)
              {
                float2 y = mul2(k.k3, vMh);
                if constexpr (DG)
                  {
                    y = fma2(k.k4, vCu, y);
                    if (aa == 0)
                      {
                        // Bx f = -f at the first node, +f at the last node of a non-periodic axis
                        const int gx = gx0 + j;
                        if (gx == bx_lo)
                          y = fma2(make_float2(-k.k6.x, -k.k6.y), u[0], y);
                        else if (gx == bx_hi)
                          y = fma2(k.k6, u[0], y);
                      }
                  }
                y2[j] = y;
                y3[j] = mul2(k.k5, vMu);
              }
            if constexpr (DG)
              if (y4_slot >= 0)
                s_y4[y4_slot * T::TX + j] = mul2(k.k6, vCu);
          }
      }
  }

  // y pass on column j and y segment seg: emit(own row i, r of the pair).
  template <int P, int CLS, typename S, typename Emit>
  __device__ __forceinline__ void
  pair_ypass(const float2 *s_y, const float2 *s_y4, const PairScales<P, S> &m, int j, int seg, int gy0, int by_lo,
             int by_hi, Emit &&emit)
  {
    using T = Tile<P, S>;
    constexpr bool XC = CLS != 1, YC = CLS != 0, DG = CLS == 2;
    const float2 *y1 = s_y, *y2 = s_y + T::NY, *y3 = s_y + 2 * T::NY;
    const int q0 = seg * T::KY;
    float2 v1[P + 1], v2[P + 1], v3[P + 1];
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
    float2 pend{};
    if constexpr (XC)
      pend = mul2(m.hy[q0], elem2_last<P, OP_M>(v1));
    if constexpr (YC)
      {
        const float2 t = fma2(m.cy[q0], elem2_last<P, OP_C>(v2), mul2(m.hyi[q0], elem2_last<P, OP_K>(v3)));
        pend = XC ? add2(pend, t) : t;
      }
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
        float2 e1[P + 1], e2[P + 1], e3[P + 1];
        if constexpr (XC)
          elem2<P, OP_M>(v1, e1);
        if constexpr (YC)
          {
            elem2<P, OP_C>(v2, e2);
            elem2<P, OP_K>(v3, e3);
          }
        const float2 sh = m.hy[qc], sc = m.cy[qc], shi = m.hyi[qc];
        const int i0 = (qc - 1) * P;
#pragma unroll
        for (int aa = 0; aa <= P; ++aa)
          {
            float2 r{};
            if constexpr (XC && YC)
              r = fma2(sh, e1[aa], fma2(sc, e2[aa], mul2(shi, e3[aa])));
            else if constexpr (XC)
              r = mul2(sh, e1[aa]);
            else
              r = fma2(sc, e2[aa], mul2(shi, e3[aa]));
            if (aa == P)
              {
                pend = r;
                break;
              }
            if (aa == 0)
              r = add2(r, pend);
            if constexpr (DG)
              {
                const int gy = gy0 + i0 + aa;
                if (gy == by_lo)
                  r = add2(r, make_float2(-s_y4[0 * T::TX + j].x, -s_y4[0 * T::TX + j].y));
                else if (gy == by_hi)
                  r = add2(r, s_y4[1 * T::TX + j]);
              }
            emit(i0 + aa, r);
          }
      }
  }

  // rhs_{a-1} <- r_a (a = 1..8) of the scheme's step on FP32 deviations d,
  // pair by pair; PAIR_BARDOW also writes the collided deviations g* to dout.
  // Images get r = 0 (constrained rows).
  // The tile (bx, by) of the kernel below (also the body of its batched form, one
  // launch over the tiles of many instances).
  template <int P, int MODE, typename S>
  __device__ __forceinline__ void
  stream_pair_tile(const Geo &geo, const DevStats *__restrict__ ds, const float *__restrict__ d,
                   float *__restrict__ dout, float *__restrict__ rhs, const AdvCoef &ac, int bx, int by)
  {
    if (ds && ds->sticky)
      return; // a step after a failed solve: the populations must stay as they are
    using T = Tile<P, S>;
    constexpr bool BARDOW = MODE == PAIR_BARDOW;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    float2 *s_pb = reinterpret_cast<float2 *>(sm_raw);        // [2][NF] the pair, double-buffered
    float2 *s_y = s_pb + 2 * T::NF;                           // [3][NY] x-pass outputs
    float2 *s_y4 = s_y + 3 * T::NY;                           // [2][TX] Y4 on the first / last domain row
    float *s_m = reinterpret_cast<float *>(s_y4 + 2 * T::TX); // [4][NF] moments
    uint8_t *s_wall = reinterpret_cast<uint8_t *>(s_m + 4 * T::NF); // [NF] wall classes (Bardow)
    __shared__ TileMaps<P, float, S> maps;
    __shared__ PairScales<P, S> sc;
    const Grid &g = geo.g;
    const long long N = g.N;
    const int gx0 = bx * T::TX, gy0 = by * T::TY;
    build_maps<P>(maps, geo, gx0, gy0);
    __syncthreads();
    for (int t = threadIdx.x; t <= T::CX; t += blockDim.x)
      {
        sc.hx[t] = bc(maps.hx[t]);
        sc.hxi[t] = bc(maps.hxi[t]);
        sc.cx[t] = bc(maps.cx[t]);
      }
    for (int t = threadIdx.x; t <= T::CY; t += blockDim.x)
      {
        sc.hy[t] = bc(maps.hy[t]);
        sc.hyi[t] = bc(maps.hyi[t]);
        sc.cy[t] = bc(maps.cy[t]);
      }

    // Staging walks the footprint a row per warp: a lane's footprint columns
    // (fx = lane + 32 k) and their source columns are the same for every row
    // and every population, so they are looked up once; a row's storage offset
    // is one broadcast load.
    const int slane = threadIdx.x & 31, swarp = threadIdx.x >> 5;
    constexpr int NCOL = (T::FX + 31) / 32;
    int scol[NCOL];
#pragma unroll
    for (int k = 0; k < NCOL; ++k)
      {
        const int fx = slane + 32 * k;
        scol[k] = fx < T::FX ? maps.col[fx] : -1;
      }

    // Pair pr of the footprint into buffer pr & 1 by asynchronous copies (one
    // commit group per pair): pair pr + 1 is in flight while pair pr computes.
    auto issue_pair = [&](int pr) {
      const float *da = d + (pr + 1) * N, *db = d + (pr + 5) * N;
      float2 *buf = s_pb + (pr & 1) * T::NF;
      for (int fy = swarp; fy < T::FY; fy += THREADS / 32)
        {
          const int r = maps.row[fy];
          float2 *brow = buf + fy * T::PF + slane;
#pragma unroll
          for (int k = 0; k < NCOL; ++k)
            if (slane + 32 * k < T::FX)
              {
                const bool ok = r >= 0 && scol[k] >= 0;
                const int idx = ok ? r + scol[k] : 0;
                cp_async4(&brow[32 * k].x, da + idx, ok);
                cp_async4(&brow[32 * k].y, db + idx, ok);
              }
        }
      cp_async_commit();
    };
    issue_pair(0);

    // moments of every footprint node (Lee-Lin: wall velocity imposed, and the
    // even equilibrium base drho - 1.5 rho u.u; Bardow: the node's own moments
    // and its wall class)
    // (row per warp as the staging; a lane's loads of all its columns in a row
    // are issued before the first moment is formed)
    for (int fy = swarp; fy < T::FY; fy += THREADS / 32)
      {
        const int r = maps.row[fy];
        float v[NCOL][Q];
        int wk[NCOL];
        bool ok[NCOL];
#pragma unroll
        for (int k = 0; k < NCOL; ++k)
          {
            ok[k] = r >= 0 && scol[k] >= 0;
            const int idx = ok[k] ? r + scol[k] : 0;
            const float *p = d + idx;
#pragma unroll
            for (int a = 0; a < Q; ++a)
              v[k][a] = ok[k] ? p[a * N] : 0.f;
            wk[k] = ok[k] && geo.wall ? geo.wall[idx] : 0;
          }
        float *mrow = s_m + fy * T::PF + slane;
#pragma unroll
        for (int k = 0; k < NCOL; ++k)
          {
            if (slane + 32 * k >= T::FX)
              continue;
            float *m = mrow + 32 * k;
            if (!ok[k])
              {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                  m[q * T::NF] = 0.f;
                if constexpr (BARDOW)
                  s_wall[fy * T::PF + slane + 32 * k] = 0;
                continue;
              }
            MomF mo = moments_dev(v[k]);
            if constexpr (BARDOW)
              {
                m[0] = mo.rho;
                m[T::NF] = mo.ux;
                m[2 * T::NF] = mo.uy;
                m[3 * T::NF] = mo.drho;
                s_wall[fy * T::PF + slane + 32 * k] = uint8_t(wk[k]);
              }
            else
              {
                mo = impose_class(mo, wk[k], geo);
                m[0] = mo.rho;
                m[T::NF] = mo.ux;
                m[2 * T::NF] = mo.uy;
                m[3 * T::NF] = mo.drho - 1.5f * mo.rho * (mo.ux * mo.ux + mo.uy * mo.uy);
              }
          }
      }

    // a tile of distinct nodes only (no image row or column, nothing past the grid)
    // writes its results without per-node checks
    const bool interior =
      gx0 + T::TX <= (g.px ? g.nux : g.nfx) && gy0 + T::TY <= (g.py ? g.nuy : g.nfy);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int bx_lo = g.px ? -1 : 0, bx_hi = g.px ? -1 : g.nfx - 1;
    const int by_lo = g.py ? -1 : 0, by_hi = g.py ? -1 : g.nfy - 1;
    const float omega = float(ac.omega);

    if constexpr (BARDOW)
      {
        // the rest population: collide only (no streaming)
        __syncthreads();
        for (int t = threadIdx.x; t < T::TY * T::TX; t += blockDim.x)
          {
            const int i = t / T::TX, j = t - i * T::TX;
            const int gx = gx0 + j, gy = gy0 + i;
            if (gx >= g.nfx || gy >= g.nfy || is_image(gx, gy, g))
              continue;
            const int st = (i + P) * T::PF + j + P;
            const MomF mo{s_m[st], s_m[T::NF + st], s_m[2 * T::NF + st], s_m[3 * T::NF + st]};
            const MomF mt = impose_class(mo, s_wall[st], geo);
            const long long idx = (long long)gy * g.nfx + gx;
            dout[idx] = feqd_a(0, mt) + (1.f - omega) * (d[idx] - feqd_a(0, mo));
          }
      }

    for (int pr = 0; pr < 4; ++pr)
      {
        const int a = pr + 1, ab = pr + 5; // opposite populations
        const float *pk = ac.pk[pr];
        const float ex = pk[2], ey = pk[4], w = ac.pw[pr], wl = ac.pwl[pr];
        float2 *s_u = s_pb + (pr & 1) * T::NF;
        if (pr < 3)
          {
            issue_pair(pr + 1); // its buffer was last read by the x pass of pair pr - 1
            cp_async_wait_group<1>();
          }
        else
          cp_async_wait_group<0>();
        __syncthreads(); // pair pr has landed; the previous pair's y pass is done with s_y
        if constexpr (BARDOW)
          {
            // g* = feq(rho, u imposed) + (1 - omega) (g - feq(rho, u)) for both, staged and written
            for (int t = threadIdx.x; t < T::FY * T::FX; t += blockDim.x)
              {
                const int fy = t / T::FX, fx = t - fy * T::FX, st = fy * T::PF + fx;
                const int r = maps.row[fy];
                const int c = maps.col[fx];
                float2 gs = make_float2(0.f, 0.f);
                if (r >= 0 && c >= 0)
                  {
                    const long long idx = r + c;
                    const float2 gv = s_u[st];
                    const MomF mo{s_m[st], s_m[T::NF + st], s_m[2 * T::NF + st], s_m[3 * T::NF + st]};
                    const MomF mt = impose_class(mo, s_wall[st], geo);
                    // each population's own equilibrium: the collision writes the state, and the
                    // rounding of the even +- odd form accumulates there from step to step
                    gs.x = feqd(ex, ey, w, wl, mt) + (1.f - omega) * (gv.x - feqd(ex, ey, w, wl, mo));
                    gs.y = feqd(-ex, -ey, w, wl, mt) + (1.f - omega) * (gv.y - feqd(-ex, -ey, w, wl, mo));
                    const int gx = gx0 - P + fx, gy = gy0 - P + fy;
                    if (fx >= P && fx < P + T::TX && fy >= P && fy < P + T::TY && gx < g.nfx && gy < g.nfy &&
                        !is_image(gx, gy, g))
                      {
                        dout[a * N + idx] = gs.x;
                        dout[ab * N + idx] = gs.y;
                      }
                  }
                s_u[st] = gs;
              }
          }
        __syncthreads();
        const int cls = ey == 0.f ? 0 : (ex == 0.f ? 1 : 2);
        PairK k;
        k.A = bc(pk[0]);
        k.B = bc(pk[1]);
        k.k1 = make_float2(pk[2], -pk[2]);
        k.k2 = bc(pk[3]);
        k.k3 = make_float2(pk[4], -pk[4]);
        k.k4 = bc(pk[5]);
        k.k5 = bc(pk[6]);
        k.k6 = bc(pk[7]);
        // x pass: lane = footprint row, warp = x segment
        if (warp < T::NSX && lane < T::FY)
          {
            const int gy = gy0 - P + lane;
            const int y4_slot = gy == by_lo ? 0 : gy == by_hi ? 1 : -1;
            if (cls == 0)
              pair_xpass<P, 0, MODE, S>(s_u, s_m, s_y, s_y4, sc, k, w, wl, ex, ey, lane, warp, gx0, y4_slot, bx_lo, bx_hi);
            else if (cls == 1)
              pair_xpass<P, 1, MODE, S>(s_u, s_m, s_y, s_y4, sc, k, w, wl, ex, ey, lane, warp, gx0, y4_slot, bx_lo, bx_hi);
            else
              pair_xpass<P, 2, MODE, S>(s_u, s_m, s_y, s_y4, sc, k, w, wl, ex, ey, lane, warp, gx0, y4_slot, bx_lo, bx_hi);
          }
        __syncthreads();
        // y pass: lane group = columns, warp group = y segment
        const int j = threadIdx.x % T::YL, seg = threadIdx.x / T::YL;
        if (j < T::TX && seg < T::NSY)
          {
            const int gx = gx0 + j;
            float *oa = rhs + (long long)(a - 1) * N, *ob = rhs + (long long)(ab - 1) * N;
            float *oac = oa + gx, *obc = ob + gx;
            auto emit = [&](int i, float2 r) {
              const int gy = gy0 + i;
              const int off = gy * g.nfx; // a population array holds fewer than 2^31 nodes
              if (interior)
                {
                  oac[off] = r.x;
                  obc[off] = r.y;
                }
              else if (gx < g.nfx && gy < g.nfy)
                {
                  const bool img = is_image(gx, gy, g);
                  oac[off] = img ? 0.f : r.x;
                  obc[off] = img ? 0.f : r.y;
                }
            };
            if (cls == 0)
              pair_ypass<P, 0, S>(s_y, s_y4, sc, j, seg, gy0, by_lo, by_hi, emit);
            else if (cls == 1)
              pair_ypass<P, 1, S>(s_y, s_y4, sc, j, seg, gy0, by_lo, by_hi, emit);
            else
              pair_ypass<P, 2, S>(s_y, s_y4, sc, j, seg, gy0, by_lo, by_hi, emit);
          }
      }

    if constexpr (BARDOW)
      {
        // the images collide their own (stale) populations, as the nodal map does
        for (int t = threadIdx.x; t < T::TY * T::TX; t += blockDim.x)
          {
            const int i = t / T::TX, j = t - i * T::TX;
            const int gx = gx0 + j, gy = gy0 + i;
            if (gx >= g.nfx || gy >= g.nfy || !is_image(gx, gy, g))
              continue;
            const long long idx = (long long)gy * g.nfx + gx;
            float v[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q)
              v[q] = d[q * N + idx];
            collide_node_dev(v, idx, geo, omega);
#pragma unroll
            for (int q = 0; q < Q; ++q)
              dout[q * N + idx] = v[q];
          }
      }
  }

  template <int P, int MODE, typename S = TileShape<P>>
  __global__ void __launch_bounds__(THREADS, S::MIN_CTAS)
    k_stream_pair(const Geo geo, const DevStats *__restrict__ ds, const float *__restrict__ d,
                  float *__restrict__ dout, float *__restrict__ rhs, const AdvCoef ac)
  {
    stream_pair_tile<P, MODE, S>(geo, ds, d, dout, rhs, ac, blockIdx.x, blockIdx.y);
  }
} // namespace lbfem_gpu
