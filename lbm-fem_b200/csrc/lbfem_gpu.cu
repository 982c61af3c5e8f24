// C ABI of the B200 hot path of lbm-fem (include/lbfem_gpu.h): the context,
// its device buffers, and the launch sequences of Scheme::step and of the
// operator entry points.
#include "lbfem_gpu.h"

#include "geometry.h"
#include "operators.cuh"
#include "stream_pair.cuh"
#include "contraction_study.cuh"
#include "quad.cuh"
#include "batch_group.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <tuple>
#include <memory>
#include <string>
#include <utility>
#include <vector>

using namespace lbfem_gpu;

struct lbfem_gpu_ctx
{
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[16] = {};
  cudaEvent_t ev_join[2] = {}; // orders the context's stream with a caller's stream (no timing)
  lbfem_params prm{};
  int P = 1;
  Grid grid{};
  int64_t n_dofs = 0;
  bool identity = true;
  std::unique_ptr<Basis1D> basis;
  Axis ax, ay;
  // discretisation on the device
  double *d_rowx = nullptr, *d_rowy = nullptr, *d_diagx = nullptr, *d_diagy = nullptr, *d_lumpx = nullptr,
         *d_lumpy = nullptr;
  double *d_hx = nullptr, *d_hxi = nullptr, *d_hy = nullptr, *d_hyi = nullptr, *d_ijx = nullptr, *d_ijy = nullptr,
         *d_ilx = nullptr, *d_ily = nullptr;
  uint8_t *d_wall = nullptr;
  double *d_wall_u = nullptr;
  long long *d_dof = nullptr; // structured node -> caller DoF
  int4 *d_bnode = nullptr;
  int n_bnodes = 0;
  // state
  double *d_f[2] = {nullptr, nullptr};
  int cur = 0;
  double *d_rhs = nullptr, *d_x[3] = {nullptr, nullptr, nullptr};
  int x_cur = 0, x_prev = 1, x_new = 2;
  double *d_r = nullptr, *d_p[2] = {nullptr, nullptr}, *d_v = nullptr;
  double *d_feq = nullptr, *d_stage = nullptr;
  // mixed precision: FP32 deviations f - w and FP32 streaming / CG vectors
  bool mixed = false;
  float *d_fs[2] = {nullptr, nullptr}, *d_rhs_s = nullptr, *d_x_s[3] = {nullptr, nullptr, nullptr};
  float *d_r_s = nullptr, *d_p_s[2] = {nullptr, nullptr};
  float *d_winx = nullptr, *d_winy = nullptr; // window LDL^T factors of Mx, My (mixed consistent mass)
  double *d_partials = nullptr, *d_sums = nullptr;
  size_t partial_cap = 0;
  CgState *d_cg = nullptr;
  CgState *h_cg = nullptr; // pinned mirror
  double dt = 0, lambda = 0;
  bool have_ts = false;
  int64_t cg_its = 0;
  double last_its_per_solve = 0;
  int64_t launches = 0, last_launches = 0;
  bool trace = false; // LBFEM_TRACE set: host-driven steps whose CG rounds print their residuals to stderr
  // graph-launched steps: one instantiated graph per state of the buffer rotation
  struct StepGraph
  {
    cudaGraphExec_t exec = nullptr;
    int64_t fixed = 0, body = 0; // kernels outside the solver loop, kernels per loop body
  };
  std::map<int, StepGraph> graphs;
  int64_t graph_epoch = 0; // counts the invalidations of the step graphs (batch graphs embed them)
  cudaStream_t cap = nullptr;     // captures the loop bodies
  DevStats *d_stats = nullptr, *h_stats = nullptr;
  // the tuned tile shape of the FP32 streaming kernel (tune_pair) and the times it was chosen by
  int pair_shape = 0;
  bool pair_tuned = false;
  float tune_ms[3] = {0.f, 0.f, 0.f};
  // general quadrilaterals (lbfem_mesh_desc::vertex_xy): per cell and Gauss point J^-1 and
  // JxW, and the per-node mass diagonals (inverse Jacobi, lumped and its inverse)
  bool distorted = false;
  double *d_qgeo = nullptr, *d_qijac = nullptr, *d_qlump = nullptr, *d_qilump = nullptr;
  // one y-strip of a decomposed mesh (lbfem_gpu_set_strip): ghost rows and the caller's collectives
  bool strip = false;
  lbfem_strip_desc sd{};
  std::string err;
};

namespace
{
  int
  fail(lbfem_gpu_ctx *c, int status, const char *fmt, ...)
  {
    if (c)
      {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
      }
    return status;
  }

#define CK(call)                                                                                          \
  do                                                                                                      \
    {                                                                                                     \
      const cudaError_t e_ = (call);                                                                      \
      if (e_ != cudaSuccess)                                                                              \
        return fail(ctx, LBFEM_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                                     \
  while (0)

#define LAUNCHED()                                                                                        \
  do                                                                                                      \
    {                                                                                                     \
      ++ctx->launches;                                                                                    \
      CK(cudaGetLastError());                                                                             \
    }                                                                                                     \
  while (0)

  Geo
  geo_of(const lbfem_gpu_ctx *ctx)
  {
    Geo g{};
    g.g = ctx->grid;
    g.hx = ctx->d_hx;
    g.hxi = ctx->d_hxi;
    g.hy = ctx->d_hy;
    g.hyi = ctx->d_hyi;
    g.ijx = ctx->d_ijx;
    g.ijy = ctx->d_ijy;
    g.ilx = ctx->d_ilx;
    g.ily = ctx->d_ily;
    g.lumpx = ctx->d_lumpx;
    g.lumpy = ctx->d_lumpy;
    g.diagx = ctx->d_diagx;
    g.diagy = ctx->d_diagy;
    g.rowx = ctx->d_rowx;
    g.rowy = ctx->d_rowy;
    g.wall = ctx->d_wall;
    g.lump2 = ctx->d_qlump;
    g.ijac2 = ctx->d_qijac;
    g.wall_u = ctx->d_wall_u;
    return g;
  }

  int
  n_pointwise_blocks(long long N)
  {
    const long long b = (N + THREADS - 1) / THREADS;
    return int(std::max(1LL, std::min(b, 148LL * 8)));
  }

  template <int P>
  dim3
  tile_grid(const Grid &g)
  {
    return dim3((g.nfx + Tile<P>::TX - 1) / Tile<P>::TX, (g.nfy + Tile<P>::TY - 1) / Tile<P>::TY);
  }

  // the tiles of the mixed solve's start for nsys systems
  template <int P>
  dim3
  start_grid(const Grid &g, int nsys)
  {
    using S = StartShape<P>;
    return dim3(tiles_along(g.nfx, g.nux, g.px, S::TX), tiles_along(g.nfy, g.nuy, g.py, S::TY), nsys);
  }

  template <typename F>
  int
  with_degree(int P, F &&f)
  {
    switch (P)
      {
        case 1:
          return f(std::integral_constant<int, 1>());
        case 2:
          return f(std::integral_constant<int, 2>());
        case 3:
          return f(std::integral_constant<int, 3>());
        default:
          return f(std::integral_constant<int, 4>());
      }
  }

  template <int P, typename R, int OPK = OPK_MASS>
  constexpr size_t
  cg_smem(int own, bool fp64_arith = false)
  {
    using T = Tile<P>;
    return (fp64_arith ? sizeof(double) : sizeof(R)) * (T::NF + op_scratch<P, OPK>()) +
           sizeof(R) * own * T::TX * T::TY;
  }

  // The reference element matrices of every degree (FE_Q(p) on [0, 1]) in FP64,
  // and the FP32 copies the FP32 kernels use. The rows of the derivative and
  // stiffness matrices sum to zero: they annihilate constants. Their FP32
  // roundings do not (row sums up to 1.5e-7 at p = 2..4), and the streaming
  // kernel would then give the slowly varying part of the deviations a small
  // coherent source every step. Each row's entries, largest first, take up the
  // FP32 row sum until it is exactly zero (entries move by at most 7e-8 of the
  // row's largest).
  void
  reference_matrices(double (&ref)[MAXPD][3][MAXPD + 1][MAXPD + 1], float (&reff)[MAXPD][3][MAXPD + 1][MAXPD + 1])
  {
    std::memset(ref, 0, sizeof ref);
    for (int q = 1; q <= MAXPD; ++q)
      {
        const Basis1D b(q);
        for (int a = 0; a <= q; ++a)
          for (int c = 0; c <= q; ++c)
            {
              ref[q - 1][OP_M][a][c] = b.Mh[a][c];
              ref[q - 1][OP_C][a][c] = b.Ch[a][c];
              ref[q - 1][OP_K][a][c] = b.Kh[a][c];
            }
      }
    for (int q = 0; q < MAXPD; ++q)
      for (int o = 0; o < 3; ++o)
        for (int a = 0; a <= MAXPD; ++a)
          {
            double big = 0;
            for (int c = 0; c <= MAXPD; ++c)
              big = std::max(big, std::fabs(ref[q][o][a][c]));
            // entries that are zero but for the quadrature's rounding (1e-20 beside
            // O(1)) become zero, so that the FP64 sums of a row's FP32 entries below
            // are exact
            for (int c = 0; c <= MAXPD; ++c)
              reff[q][o][a][c] = std::fabs(ref[q][o][a][c]) <= 1e-14 * big ? 0.f : float(ref[q][o][a][c]);
          }
    for (int q = 0; q < MAXPD; ++q)
      for (int o : {int(OP_C), int(OP_K)})
        for (int a = 0; a <= q + 1; ++a)
          {
            float *row = reff[q][o][a];
            int order[MAXPD + 1];
            for (int c = 0; c <= q + 1; ++c)
              order[c] = c;
            std::stable_sort(order, order + q + 2,
                             [&](int x, int y) { return std::fabs(row[x]) > std::fabs(row[y]); });
            for (int k = 0; k <= q + 1; ++k)
              {
                double sum = 0; // exact: a few FP32 values
                for (int c = 0; c <= q + 1; ++c)
                  sum += double(row[c]);
                if (sum == 0.0)
                  break;
                row[order[k]] = float(double(row[order[k]]) - sum);
              }
          }
  }

  template <typename K>
  int
  set_smem(lbfem_gpu_ctx *ctx, K kernel, size_t bytes)
  {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    return LBFEM_OK;
  }

  template <int P>
  int
  set_smem_attributes(lbfem_gpu_ctx *ctx)
  {
    int st;
    if ((st = set_smem(ctx, k_advection<P, ADV_TG, double>, advection_smem<P, ADV_TG, double>())) ||
        (st = set_smem(ctx, k_advection<P, ADV_TG_COLLIDE, double>, advection_smem<P, ADV_TG_COLLIDE, double>())) ||
        (st = set_smem(ctx, k_advection<P, ADV_LEELIN_FEQ, double>, advection_smem<P, ADV_LEELIN_FEQ, double>())) ||
        (st = set_smem(ctx, k_advection<P, ADV_LEELIN_FUSED, double>, advection_smem<P, ADV_LEELIN_FUSED, double>())) ||
        (st = set_smem(ctx, k_stream_pair<P, PAIR_LEELIN>, pair_smem<P, PAIR_LEELIN>())) ||
        (st = set_smem(ctx, k_stream_pair<P, PAIR_BARDOW>, pair_smem<P, PAIR_BARDOW>())) ||
        (st = set_smem(ctx, k_stream_pair<P, PAIR_LEELIN, TileShapeAlt<P>>,
                       pair_smem<P, PAIR_LEELIN, TileShapeAlt<P>>())) ||
        (st = set_smem(ctx, k_stream_pair<P, PAIR_BARDOW, TileShapeAlt<P>>,
                       pair_smem<P, PAIR_BARDOW, TileShapeAlt<P>>())) ||
        (st = set_smem(ctx, k_stream_pair<P, PAIR_LEELIN, TileShapeSmall<P>>,
                       pair_smem<P, PAIR_LEELIN, TileShapeSmall<P>>())) ||
        (st = set_smem(ctx, k_stream_pair<P, PAIR_BARDOW, TileShapeSmall<P>>,
                       pair_smem<P, PAIR_BARDOW, TileShapeSmall<P>>())) ||
        (st = set_smem(ctx, k_mass_vmult<P>, cg_smem<P, double>(0))) ||
        (st = set_smem(ctx, k_cg_start<P, double, double, double>, cg_smem<P, double>(1))) ||
        (st = set_smem(ctx, k_cg_p<P, double>, cg_smem<P, double>(0))) ||
        (st = set_smem(ctx, k_cg_update<P, double>, cg_smem<P, double>(0))) ||
        (st = set_smem(ctx, k_cg_start<P, double, double, double, OPK_TG3>, cg_smem<P, double, OPK_TG3>(1))) ||
        (st = set_smem(ctx, k_cg_p<P, double, OPK_TG3>, cg_smem<P, double, OPK_TG3>(0))) ||
        (st = set_smem(ctx, k_cg_update<P, double, OPK_TG3>, cg_smem<P, double, OPK_TG3>(2))) ||
        (st = set_smem(ctx, k_cg_start<P, double, double, double, OPK_LAPLACE>,
                       cg_smem<P, double, OPK_LAPLACE>(1))) ||
        (st = set_smem(ctx, k_cg_p<P, double, OPK_LAPLACE>, cg_smem<P, double, OPK_LAPLACE>(0))) ||
        (st = set_smem(ctx, k_cg_update<P, double, OPK_LAPLACE>, cg_smem<P, double, OPK_LAPLACE>(2))) ||
        (st = set_smem(ctx, k_cg_start<P, float, float, double>, cg_smem<P, float>(1, true))) ||
        (st = set_smem(ctx, k_window_correct<P>, window_smem<P>())) ||
        (st = set_smem(ctx, kg_stream_pair<P, PAIR_LEELIN>, pair_smem<P, PAIR_LEELIN>())) ||
        (st = set_smem(ctx, kg_stream_pair<P, PAIR_BARDOW>, pair_smem<P, PAIR_BARDOW>())) ||
        (st = set_smem(ctx, kg_window<P>, window_smem<P>())) ||
        (st = set_smem(ctx, k_richardson_pass<P, double>, cg_smem<P, double>(0))) ||
        (st = set_smem(ctx, k_richardson_pass<P, float>, cg_smem<P, float>(0))))
      return st;
    return LBFEM_OK;
  }

  int
  reduce(lbfem_gpu_ctx *ctx, int n_blocks, int nq)
  {
    k_reduce_partials<<<nq, 256, 0, ctx->stream>>>(ctx->d_partials, n_blocks, ctx->d_sums);
    LAUNCHED();
    return LBFEM_OK;
  }

  // --------------------------------------------------- streaming RHS (K1)
  AdvCoef
  adv_coef(double a, double b, double c, const double *e, double omega)
  {
    AdvCoef ac{};
    ac.a = a;
    ac.b = b;
    ac.c = c;
    for (int al = 0; al < NM; ++al)
      {
        ac.ex[al] = e[2 * (al + 1)];
        ac.ey[al] = e[2 * (al + 1) + 1];
      }
    ac.omega = omega;
    static const double w[5] = {0., 1. / 9., 1. / 36., 1. / 9., 1. / 36.};
    for (int pr = 0; pr < 4; ++pr)
      {
        const double exd = ac.ex[pr], eyd = ac.ey[pr];
        const double v[8] = {a, b, exd, c * exd * exd, eyd, -2.0 * c * exd * eyd, c * eyd * eyd, c * exd * eyd};
        for (int k = 0; k < 8; ++k)
          ac.pk[pr][k] = float(v[k]);
        ac.pw[pr] = float(w[pr + 1]);
        ac.pwl[pr] = float(w[pr + 1] - double(ac.pw[pr]));
      }
    return ac;
  }

  const double *
  d2q9_e()
  {
    static const double e[18] = {0, 0, 1, 0, 1, 1, 0, 1, -1, 1, -1, 0, -1, -1, 0, -1, 1, -1};
    return e;
  }

  int quad_advection(lbfem_gpu_ctx *ctx, const double *f, const double *feq, double *rhs, const AdvCoef &ac);
  int quad_solve(lbfem_gpu_ctx *ctx, const double *b, double *x, int nsys, int64_t *its);
  int quad_vmult(lbfem_gpu_ctx *ctx, const double *x, double *y, int nsys);

  // ds: the step counters of a step (its kernel does nothing after a failure), null otherwise.
  template <typename R>
  int
  launch_advection(lbfem_gpu_ctx *ctx, int mode, const R *f, const R *feq, R *fout, R *rhs, const AdvCoef &ac,
                   const DevStats *ds = nullptr)
  {
    if (ctx->distorted)
      {
        if constexpr (sizeof(R) == sizeof(double))
          if (mode == ADV_TG || mode == ADV_LEELIN_FEQ)
            return quad_advection(ctx, f, mode == ADV_LEELIN_FEQ ? feq : nullptr, rhs, ac);
        return fail(ctx, LBFEM_ERR_UNSUPPORTED, "general quadrilaterals: the advection of given populations only");
      }
    const Geo geo = geo_of(ctx);
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      const dim3 grid = tile_grid<P>(ctx->grid);
      switch (mode)
        {
          case ADV_TG:
            if constexpr (sizeof(R) == sizeof(double))
              k_advection<P, ADV_TG, R>
                <<<grid, THREADS, advection_smem<P, ADV_TG, R>(), ctx->stream>>>(geo, ds, f, feq, fout, rhs, ac);
            break;
          case ADV_TG_COLLIDE:
            k_advection<P, ADV_TG_COLLIDE, R>
              <<<grid, THREADS, advection_smem<P, ADV_TG_COLLIDE, R>(), ctx->stream>>>(geo, ds, f, feq, fout, rhs, ac);
            break;
          case ADV_LEELIN_FEQ:
            if constexpr (sizeof(R) == sizeof(double))
              k_advection<P, ADV_LEELIN_FEQ, R>
                <<<grid, THREADS, advection_smem<P, ADV_LEELIN_FEQ, R>(), ctx->stream>>>(geo, ds, f, feq, fout, rhs, ac);
            break;
          default:
            k_advection<P, ADV_LEELIN_FUSED, R>
              <<<grid, THREADS, advection_smem<P, ADV_LEELIN_FUSED, R>(), ctx->stream>>>(geo, ds, f, feq, fout, rhs, ac);
        }
      LAUNCHED();
      return LBFEM_OK;
    });
  }

  // The FP32 streaming kernel of the mixed-precision step (pairs of opposite
  // populations), in tile shape `shape` (0: TileShape, 1: TileShapeAlt,
  // 2: TileShapeSmall; -1: the context's tuned choice).
  int
  launch_pair(lbfem_gpu_ctx *ctx, int mode, const float *d, float *dout, float *rhs, const AdvCoef &ac,
              const DevStats *ds = nullptr, int shape = -1)
  {
    const Geo geo = geo_of(ctx);
    if (shape < 0)
      shape = ctx->pair_shape;
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      auto go = [&](auto SS) {
        using S = decltype(SS);
        using T = Tile<P, S>;
        const dim3 grid((ctx->grid.nfx + T::TX - 1) / T::TX, (ctx->grid.nfy + T::TY - 1) / T::TY);
        if (mode == PAIR_BARDOW)
          k_stream_pair<P, PAIR_BARDOW, S><<<grid, THREADS, pair_smem<P, PAIR_BARDOW, S>(), ctx->stream>>>(
            geo, ds, d, dout, rhs, ac);
        else
          k_stream_pair<P, PAIR_LEELIN, S><<<grid, THREADS, pair_smem<P, PAIR_LEELIN, S>(), ctx->stream>>>(
            geo, ds, d, dout, rhs, ac);
      };
      if (shape == 1)
        go(TileShapeAlt<P>{});
      else if (shape == 2)
        go(TileShapeSmall<P>{});
      else
        go(TileShape<P>{});
      LAUNCHED();
      return LBFEM_OK;
    });
  }

  // The run-time choice of the FP32 streaming kernel's tile (cells per CTA and
  // per x / y segment): each compiled shape is timed on the context's own
  // buffers (CUDA events, one warm-up and five timed launches) before the first
  // step records its graph, and the fastest is kept. The choice is cached per
  // (device, degree, scheme, grid) for the other contexts of the process.
  // LBFEM_TUNE=0 keeps the default shape; LBFEM_TUNE=alt / small fix the other
  // two (for tests). Every shape gives bitwise the same
  // results (the per-node arithmetic does not depend on the tile).
  struct TuneKey
  {
    int dev, P, mode, nfx, nfy;
    bool
    operator<(const TuneKey &o) const
    {
      return std::tie(dev, P, mode, nfx, nfy) < std::tie(o.dev, o.P, o.mode, o.nfx, o.nfy);
    }
  };
  std::mutex tune_mutex;
  constexpr int N_SHAPES = 3;
  std::map<TuneKey, std::pair<int, std::array<float, N_SHAPES>>> tune_cache;

  int
  tune_pair(lbfem_gpu_ctx *ctx)
  {
    if (!ctx->mixed || ctx->pair_tuned || ctx->distorted)
      return LBFEM_OK;
    const char *env = std::getenv("LBFEM_TUNE");
    if (env && (env[0] == '0' || std::strcmp(env, "alt") == 0 || std::strcmp(env, "small") == 0))
      {
        // a fixed shape: the default ("0"), the alternative ("alt") or the small one ("small")
        ctx->pair_shape = env[0] == '0' ? 0 : env[0] == 'a' ? 1 : 2;
        ctx->pair_tuned = true;
        return LBFEM_OK;
      }
    const bool bardow = ctx->prm.scheme == LBFEM_SCHEME_BARDOW;
    const TuneKey key{ctx->device, ctx->P, bardow ? 1 : 0, ctx->grid.nfx, ctx->grid.nfy};
    {
      std::lock_guard<std::mutex> lock(tune_mutex);
      const auto it = tune_cache.find(key);
      if (it != tune_cache.end())
        {
          ctx->pair_shape = it->second.first;
          for (int k = 0; k < N_SHAPES; ++k)
            ctx->tune_ms[k] = it->second.second[k];
          ctx->pair_tuned = true;
          return LBFEM_OK;
        }
    }
    const double dt = ctx->dt, lam = ctx->lambda, b = -0.5 * dt * dt / lam;
    const AdvCoef ac = bardow ? adv_coef(-dt, 0., -0.5 * dt * dt, d2q9_e(), dt / (lam + 0.5 * dt))
                              : adv_coef(-dt - b, b, -0.5 * dt * dt, d2q9_e(), 0.);
    float *d = ctx->d_fs[ctx->cur], *g = bardow ? ctx->d_fs[1 - ctx->cur] : nullptr;
    std::array<float, N_SHAPES> ms{};
    int st;
    for (int shape = 0; shape < N_SHAPES; ++shape)
      {
        if ((st = launch_pair(ctx, bardow ? PAIR_BARDOW : PAIR_LEELIN, d, g, ctx->d_rhs_s, ac, nullptr, shape)))
          return st;
        CK(cudaEventRecord(ctx->ev[14], ctx->stream));
        for (int k = 0; k < 5; ++k)
          if ((st = launch_pair(ctx, bardow ? PAIR_BARDOW : PAIR_LEELIN, d, g, ctx->d_rhs_s, ac, nullptr, shape)))
            return st;
        CK(cudaEventRecord(ctx->ev[15], ctx->stream));
        CK(cudaEventSynchronize(ctx->ev[15]));
        CK(cudaEventElapsedTime(&ms[shape], ctx->ev[14], ctx->ev[15]));
        ms[shape] /= 5.f;
      }
    ctx->pair_shape = 0;
    for (int k = 0; k < N_SHAPES; ++k)
      {
        ctx->tune_ms[k] = ms[k];
        if (ms[k] < ms[ctx->pair_shape])
          ctx->pair_shape = k;
      }
    ctx->pair_tuned = true;
    std::lock_guard<std::mutex> lock(tune_mutex);
    tune_cache[key] = {ctx->pair_shape, ms};
    return LBFEM_OK;
  }

  FaceCoef face_coef(const lbfem_gpu_ctx *ctx, const double *e, double dt, bool remove);

  template <typename R>
  int
  launch_wall_faces(lbfem_gpu_ctx *ctx, const R *f, R *rhs, const double *e, double dt, bool remove)
  {
    if (ctx->n_bnodes == 0)
      return LBFEM_OK;
    const FaceCoef fc = face_coef(ctx, e, dt, remove);
    const Geo geo = geo_of(ctx);
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      k_wall_faces<P, R><<<(ctx->n_bnodes * 8 + 127) / 128, 128, 0, ctx->stream>>>(geo, f, rhs, ctx->d_bnode,
                                                                           ctx->n_bnodes, fc);
      LAUNCHED();
      return LBFEM_OK;
    });
  }

  // The wall-face coefficients of directions e (9 x 2) and time step dt.
  FaceCoef
  face_coef(const lbfem_gpu_ctx *ctx, const double *e, double dt, bool remove)
  {
    FaceCoef fc{};
    fc.half_dt2 = 0.5 * dt * dt;
    for (int al = 0; al < NM; ++al)
      {
        fc.ex[al] = e[2 * (al + 1)];
        fc.ey[al] = e[2 * (al + 1) + 1];
      }
    fc.remove = remove ? 1 : 0;
    for (int a = 0; a <= ctx->P; ++a)
      {
        fc.d0[a] = ctx->basis->d0[a];
        fc.d1[a] = ctx->basis->d1[a];
      }
    fc.hx0 = ctx->ax.h_first;
    fc.hx1 = ctx->ax.h_last;
    fc.hy0 = ctx->ay.h_first;
    fc.hy1 = ctx->ay.h_last;
    return fc;
  }

  // ------------------------------------------------------ mass solve (K2-K4)
  // The work buffers of one CG run: residual, two search directions, per-tile
  // partial sums, reduced sums and the per-system solver state.
  template <typename R>
  struct CgScratch
  {
    R *r, *p[2];
    double *partials, *sums;
    CgState *state;
  };

  int
  reduce_into(lbfem_gpu_ctx *ctx, const double *partials, double *sums, int n_blocks, int nq)
  {
    k_reduce_partials<<<nq, 256, 0, ctx->stream>>>(partials, n_blocks, sums);
    LAUNCHED();
    return LBFEM_OK;
  }

  // The relative tolerance of the mixed-precision mass solve.
  // ------------------------------------------------ y-strip decomposition
  // The sums buffer the solvers reduce into: the caller's (summed over the
  // ranks by its ALLREDUCE) in strip mode, else the context's.
  double *
  sums_buf(lbfem_gpu_ctx *ctx)
  {
    return ctx->strip ? ctx->sd.sums : ctx->d_sums;
  }

  // Strip mode: the first n doubles of sums_buf summed over the ranks.
  int
  strip_allreduce(lbfem_gpu_ctx *ctx, int n)
  {
    if (!ctx->strip)
      return LBFEM_OK;
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->sd.comm(ctx->sd.user, LBFEM_COMM_ALLREDUCE, n) != 0)
      return fail(ctx, LBFEM_ERR_ARG, "strip: the allreduce of %d sums failed", n);
    return LBFEM_OK;
  }

  // Strip mode: the ghost rows of nb blocks (element size es, block stride N)
  // of the field at base <- the neighbours' owned rows. Rows are contiguous
  // in a block, so each side is one strided copy: 1 row down and `degree`
  // rows up out of the owned rows, `degree` rows below and 1 row above in.
  int
  strip_exchange(lbfem_gpu_ctx *ctx, void *base, int nb, size_t es)
  {
    if (!ctx->strip)
      return LBFEM_OK;
    const Grid &g = ctx->grid;
    const size_t row = size_t(g.nfx) * es, pitch = size_t(g.N) * es;
    const int P = ctx->P;
    char *b = static_cast<char *>(base);
    const lbfem_strip_desc &sd = ctx->sd;
    if (sd.ghost_below)
      CK(cudaMemcpy2DAsync(sd.send_below, row, b + size_t(g.oy0) * row, pitch, row, nb, cudaMemcpyDeviceToDevice,
                           ctx->stream));
    if (sd.ghost_above)
      CK(cudaMemcpy2DAsync(sd.send_above, P * row, b + size_t(g.oy1 - P) * row, pitch, P * row, nb,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (sd.comm(sd.user, LBFEM_COMM_EXCHANGE, int64_t(nb) * int64_t(row)) != 0)
      return fail(ctx, LBFEM_ERR_ARG, "strip: the ghost exchange failed");
    if (sd.ghost_below)
      CK(cudaMemcpy2DAsync(b + size_t(g.oy0 - P) * row, pitch, sd.recv_below, P * row, P * row, nb,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    if (sd.ghost_above)
      CK(cudaMemcpy2DAsync(b + size_t(g.oy1) * row, pitch, sd.recv_above, row, row, nb, cudaMemcpyDeviceToDevice,
                           ctx->stream));
    return LBFEM_OK;
  }

  double
  mixed_tolerance(const lbfem_params &p)
  {
    return std::max(p.cg_tolerance, p.mixed_tolerance > 0 ? p.mixed_tolerance : LBFEM_MIXED_TOLERANCE);
  }

  // One FP64 CG solve: x_new <- A^{-1} b for nsys systems, from the extrapolated
  // start 2 x_cur - x_prev or from the given x_new. A (opk) is the mass matrix, the
  // streaming matrix M + c K_e of each system (sc), or the Laplace operator of the
  // stream function; the systems of skip are left alone (populations at rest in a
  // split TG3 sweep). tol / max_its < 0: the context's CG settings.
  struct CgCall
  {
    const double *b = nullptr;
    double *x_new = nullptr;
    const double *x_cur = nullptr, *x_prev = nullptr;
    int extrapolate = 0, nsys = NM;
    int opk = OPK_MASS;
    StreamCoef sc{};
    int skip = 0;
    double tol = -1;
    int max_its = -1;
  };

  template <typename F>
  int
  with_op(int opk, F &&f)
  {
    switch (opk)
      {
        case OPK_TG3:
          return f(std::integral_constant<int, OPK_TG3>());
        case OPK_LAPLACE:
          return f(std::integral_constant<int, OPK_LAPLACE>());
        default:
          return f(std::integral_constant<int, OPK_MASS>());
      }
  }

  // r = b - A x_start and the start sums; *n_tiles: the tiles of one system.
  int
  cg_launch_start(lbfem_gpu_ctx *ctx, const CgScratch<double> &w, const CgCall &c, int *n_tiles)
  {
    const Geo geo = geo_of(ctx);
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      dim3 grid = tile_grid<P>(ctx->grid);
      *n_tiles = int(grid.x * grid.y);
      grid.z = c.nsys;
      return with_op(c.opk, [&](auto OO) -> int {
        constexpr int OPK = decltype(OO)::value;
        k_cg_start<P, double, double, double, OPK><<<grid, THREADS, cg_smem<P, double, OPK>(OPK == OPK_MASS ? 0 : 1, true), ctx->stream>>>(
          geo, c.b, c.x_cur, c.x_prev, c.x_new, w.r, c.extrapolate, w.partials, c.sc, c.skip);
        LAUNCHED();
        return LBFEM_OK;
      });
    });
  }

  // p[1-pi] <- D^{-1} r + beta p[pi] and the sums p.Ap.
  int
  cg_launch_p(lbfem_gpu_ctx *ctx, const CgScratch<double> &w, const CgCall &c, int pi)
  {
    const Geo geo = geo_of(ctx);
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      dim3 grid = tile_grid<P>(ctx->grid);
      grid.z = c.nsys;
      return with_op(c.opk, [&](auto OO) -> int {
        constexpr int OPK = decltype(OO)::value;
        k_cg_p<P, double, OPK><<<grid, THREADS, cg_smem<P, double, OPK>(0), ctx->stream>>>(
          geo, w.r, w.p[pi], w.p[1 - pi], w.state, w.partials, c.sc);
        LAUNCHED();
        return LBFEM_OK;
      });
    });
  }

  // x += alpha p, r -= alpha A p with p = p[pi], and the sums r.r, r.D^{-1}r.
  int
  cg_launch_update(lbfem_gpu_ctx *ctx, const CgScratch<double> &w, const CgCall &c, int pi)
  {
    const Geo geo = geo_of(ctx);
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      dim3 grid = tile_grid<P>(ctx->grid);
      grid.z = c.nsys;
      return with_op(c.opk, [&](auto OO) -> int {
        constexpr int OPK = decltype(OO)::value;
        k_cg_update<P, double, OPK><<<grid, THREADS, cg_smem<P, double, OPK>(OPK == OPK_MASS ? 0 : 2), ctx->stream>>>(
          geo, c.x_new, w.r, w.p[pi], w.state, w.partials, c.sc);
        LAUNCHED();
        return LBFEM_OK;
      });
    });
  }

  // x <- 0 for the systems flagged by the solver's start (right-hand side exactly zero).
  template <typename R>
  int
  zero_flagged(lbfem_gpu_ctx *ctx, R *x, const CgState *state, int nsys)
  {
    k_zero_flagged<R><<<dim3(148, nsys), THREADS, 0, ctx->stream>>>(x, state, ctx->grid.N, nsys);
    LAUNCHED();
    return LBFEM_OK;
  }

  // Jacobi-PCG in the order of updates of deal.II SolverCG (mass.h:204-211),
  // host-driven, with the work buffers w. *its_out: CG iterations summed over
  // the systems.
  int
  cg_run(lbfem_gpu_ctx *ctx, const CgScratch<double> &w, const CgCall &c, int64_t *its_out)
  {
    const double tol = c.tol >= 0 ? c.tol : ctx->prm.cg_tolerance;
    const int max_its = c.max_its > 0 ? c.max_its : ctx->prm.cg_max_iterations;
    const int nsys = c.nsys;
    CK(cudaMemsetAsync(w.state, 0, sizeof(CgState), ctx->stream));
    int n_tiles = 0, st;
    if ((st = cg_launch_start(ctx, w, c, &n_tiles)) || (st = reduce_into(ctx, w.partials, w.sums, n_tiles, 3 * NM)) ||
        (st = strip_allreduce(ctx, 3 * NM)))
      return st;
    k_cg_scalars<<<1, 32, 0, ctx->stream>>>(w.state, w.sums, nsys, 0, tol, max_its);
    LAUNCHED();
    if ((st = zero_flagged(ctx, c.x_new, w.state, nsys)) || (st = strip_exchange(ctx, w.r, nsys, sizeof(double))))
      return st;
    int pi = 0;
    for (int it = 0;; ++it)
      {
        CK(cudaMemcpyAsync(ctx->h_cg, w.state, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->trace)
          {
            std::fprintf(stderr, "lbfem cg: it %d active %d res/tol", it, ctx->h_cg->n_active);
            for (int q = 0; q < nsys; ++q)
              std::fprintf(stderr, " %.2e", ctx->h_cg->tol[q] > 0 ? ctx->h_cg->res[q] / ctx->h_cg->tol[q] : 0.0);
            std::fprintf(stderr, "\n");
          }
        if (ctx->h_cg->n_active == 0)
          break;
        if ((st = cg_launch_p(ctx, w, c, pi)) || (st = reduce_into(ctx, w.partials, w.sums, n_tiles, NM)) ||
            (st = strip_allreduce(ctx, NM)))
          return st;
        k_cg_scalars<<<1, 32, 0, ctx->stream>>>(w.state, w.sums, nsys, 1, tol, max_its);
        LAUNCHED();
        pi = 1 - pi;
        if ((st = cg_launch_update(ctx, w, c, pi)) || (st = reduce_into(ctx, w.partials, w.sums, n_tiles, 2 * NM)) ||
            (st = strip_allreduce(ctx, 2 * NM)))
          return st;
        k_cg_scalars<<<1, 32, 0, ctx->stream>>>(w.state, w.sums, nsys, 2, tol, max_its);
        LAUNCHED();
        if ((st = strip_exchange(ctx, w.r, nsys, sizeof(double))))
          return st;
      }
    if (its_out)
      *its_out = ctx->h_cg->total_its;
    if (ctx->h_cg->status == 2)
      return fail(ctx, LBFEM_ERR_NO_CONVERGENCE, "CG: iteration cap %d reached", max_its);
    if (ctx->h_cg->status == 3)
      return fail(ctx, LBFEM_ERR_NONFINITE, "CG: non-finite residual");
    return LBFEM_OK;
  }

  CgScratch<double>
  ctx_scratch(lbfem_gpu_ctx *ctx)
  {
    return CgScratch<double>{ctx->d_r, {ctx->d_p[0], ctx->d_p[1]}, ctx->d_partials, sums_buf(ctx), ctx->d_cg};
  }

  // The context's own work buffers.
  int
  cg_solve(lbfem_gpu_ctx *ctx, const CgCall &c, int64_t *its_out)
  {
    int64_t its = 0;
    const int st = cg_run(ctx, ctx_scratch(ctx), c, &its);
    if (its_out)
      *its_out = its;
    ctx->cg_its += its;
    return st;
  }

  // The streaming matrix coefficients of the directions e (2 Q values) and the dt^2 coefficient c.
  StreamCoef
  stream_coef(const double *e, double c)
  {
    StreamCoef sc{};
    for (int al = 0; al < NM; ++al)
      {
        const double ex = e[2 * (al + 1)], ey = e[2 * (al + 1) + 1];
        sc.kxx[al] = c * ex * ex;
        sc.kyy[al] = c * ey * ey;
        sc.kxy[al] = c * ex * ey;
      }
    return sc;
  }

  // The moving populations at rest in the directions e, as a system mask.
  int
  resting(const double *e)
  {
    int m = 0;
    for (int al = 0; al < NM; ++al)
      if (e[2 * (al + 1)] == 0. && e[2 * (al + 1) + 1] == 0.)
        m |= 1 << al;
    return m;
  }

  // The status code of a failed mixed-precision solve (CgState status, 0: none).
  int
  mixed_status(lbfem_gpu_ctx *ctx, int status, double tol)
  {
    switch (status)
      {
        case 0:
          return LBFEM_OK;
        case 3:
          return fail(ctx, LBFEM_ERR_NONFINITE, "mixed mass solve: non-finite residual");
        case 4:
          return fail(ctx, LBFEM_ERR_NO_CONVERGENCE,
                      "mixed mass solve: a correction no longer halves the residual (the tolerance %.1e is below the "
                      "FP32 resolution of the solution)",
                      tol);
        default:
          return fail(ctx, LBFEM_ERR_NO_CONVERGENCE, "mixed mass solve: no convergence within %d corrections",
                      ctx->prm.cg_max_iterations);
      }
  }

  // The mixed-precision mass solve of the 8 moving populations: FP64 iterative
  // refinement around the tensor-product window solve, on the FP32 solution
  // history of the context. The start is the extrapolation x0 = 2 x_cur - x_prev
  // with its residual r0 = b - A x0 (FP32 arithmetic: it only feeds the first
  // correction). Each round then adds the FP32 correction
  // M^{-1} r (window solves) and forms the new residual b - A x in FP64
  // arithmetic, in one kernel; the systems whose residual meets the tolerance
  // stop. The first round corrects every system: accepting the extrapolation
  // whenever it meets the tolerance would march on extrapolated increments,
  // whose errors accumulate from step to step. A correction reduces the
  // residual to a few 1e-8 of itself, so one round is the rule; the tolerance
  // floor is the FP32 rounding of x (about 1e-7 relative). On return x_cur holds
  // the solution and the history has moved on by one step. *its_out:
  // corrections, summed over the systems.
  int
  mixed_solve(lbfem_gpu_ctx *ctx, const float *b, int nsys, int64_t *its_out)
  {
    const Geo geo = geo_of(ctx);
    const Grid &g = ctx->grid;
    const double tol = mixed_tolerance(ctx->prm);
    const int max_rounds = ctx->prm.cg_max_iterations;
    const int ic = ctx->x_cur, ip = ctx->x_prev, in = ctx->x_new;
    CK(cudaMemsetAsync(ctx->d_cg, 0, sizeof(CgState), ctx->stream));
    int st = with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      // FP32 arithmetic: r0 only feeds the FP32 correction (the rounds form the FP64 residuals)
      k_mixed_start<P><<<start_grid<P>(g, nsys), StartShape<P>::THREADS, 0, ctx->stream>>>(
        geo, b, ctx->d_x_s[ic], ctx->d_x_s[ip], ctx->d_x_s[in], ctx->d_r_s);
      LAUNCHED();
      return LBFEM_OK;
    });
    if (st || (st = strip_exchange(ctx, ctx->d_r_s, nsys, sizeof(float))))
      return st;
    double *sums = sums_buf(ctx);
    // the rounds alternate between x_new and x_prev's buffer (free once the start has read it)
    int xi = in, xo = ip;
    float *r_in = ctx->d_r_s, *r_out = ctx->d_p_s[0];
    for (int round = 0;; ++round)
      {
        int n_tiles = 0;
        st = with_degree(ctx->P, [&](auto PP) -> int {
          constexpr int P = decltype(PP)::value;
          using S = WinShape<P>;
          const dim3 grid(tiles_along(g.nfx, g.nux, g.px, S::TX), tiles_along(g.nfy, g.nuy, g.py, S::TY), nsys);
          n_tiles = int(grid.x * grid.y);
          k_window_correct<P><<<grid, S::THREADS, window_smem<P>(), ctx->stream>>>(
            geo, ctx->d_winx, ctx->d_winy, r_in, ctx->d_x_s[xi], b, ctx->d_x_s[xo], r_out, ctx->d_cg, round == 0,
            ctx->d_partials);
          LAUNCHED();
          return LBFEM_OK;
        });
        if (st)
          return st;
        std::swap(xi, xo);
        std::swap(r_in, r_out);
        if (ctx->strip)
          {
            // The round's residual near the strip's edges saw the locally corrected
            // ghost rows. With the neighbours' corrected rows in place, the residual
            // b - A x of the owned rows is formed again (FP64 arithmetic), its ghost
            // rows exchanged and its sums added over the ranks.
            float *xs = ctx->d_x_s[xi];
            if ((st = strip_exchange(ctx, xs, nsys, sizeof(float))))
              return st;
            st = with_degree(ctx->P, [&](auto PP) -> int {
              constexpr int P = decltype(PP)::value;
              dim3 grid = tile_grid<P>(g);
              n_tiles = int(grid.x * grid.y);
              grid.z = nsys;
              k_cg_start<P, float, float, double><<<grid, THREADS, cg_smem<P, float>(1, true), ctx->stream>>>(
                geo, b, nullptr, nullptr, xs, r_in, 0, ctx->d_partials, StreamCoef{}, 0);
              LAUNCHED();
              return LBFEM_OK;
            });
            if (st || (st = reduce_into(ctx, ctx->d_partials, sums, n_tiles, 3 * NM)) ||
                (st = strip_allreduce(ctx, 2 * NM)) || (st = strip_exchange(ctx, r_in, nsys, sizeof(float))))
              return st;
          }
        else if ((st = reduce_into(ctx, ctx->d_partials, sums, n_tiles, 2 * NM)))
          return st;
        k_mixed_round<<<1, 32, 0, ctx->stream>>>(ctx->d_cg, sums, nullptr, nsys, tol, max_rounds, 0, 0);
        LAUNCHED();
        if (round == 0 && (st = zero_flagged(ctx, ctx->d_x_s[xi], ctx->d_cg, nsys)))
          return st; // xi: the round's output after the swap above
        CK(cudaMemcpyAsync(ctx->h_cg, ctx->d_cg, sizeof(CgState), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->trace)
          {
            std::fprintf(stderr, "lbfem mixed solve: round %d still active %d res/tol", round, ctx->h_cg->n_active);
            for (int q = 0; q < nsys; ++q)
              std::fprintf(stderr, " %.2e", ctx->h_cg->tol[q] > 0 ? ctx->h_cg->res[q] / ctx->h_cg->tol[q] : 0.0);
            std::fprintf(stderr, "\n");
          }
        if ((st = mixed_status(ctx, ctx->h_cg->status, tol)))
          return st;
        if (ctx->h_cg->n_active == 0)
          break;
      }
    // the solution is in buffer xi
    ctx->x_prev = ic;
    ctx->x_cur = xi;
    ctx->x_new = xi == in ? ip : in;
    if (its_out)
      *its_out = int64_t(ctx->h_cg->total_its);
    ctx->cg_its += int64_t(ctx->h_cg->total_its);
    return LBFEM_OK;
  }

  // The iterated lumping of MassSolver::solve (mass.h:193-202): x = M_L^{-1} b, then
  // prm.richardson passes x += M_L^{-1} (b - M x). The passes alternate between
  // out and scratch; the result is in out (an odd count ends with a copy-free
  // swap of the roles: the first pass reads out and writes scratch).
  template <typename R>
  int
  richardson_passes(lbfem_gpu_ctx *ctx, const R *b, R *out, R *scratch, int nsys)
  {
    const Geo geo = geo_of(ctx);
    const int k = ctx->prm.richardson;
    R *first = (k % 2) ? scratch : out; // the lumped start, so that the last pass writes out
    k_lumped<R, R><<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo, b, first, nsys);
    LAUNCHED();
    int st0;
    if ((st0 = strip_exchange(ctx, first, nsys, sizeof(R))))
      return st0;
    R *in = first, *to = first == out ? scratch : out;
    for (int j = 0; j < k; ++j)
      {
        int st = with_degree(ctx->P, [&](auto PP) -> int {
          constexpr int P = decltype(PP)::value;
          dim3 grid = tile_grid<P>(ctx->grid);
          grid.z = nsys;
          k_richardson_pass<P, R><<<grid, THREADS, cg_smem<P, R>(0), ctx->stream>>>(geo, b, in, to);
          LAUNCHED();
          return LBFEM_OK;
        });
        if (st || (st = strip_exchange(ctx, to, nsys, sizeof(R))))
          return st;
        std::swap(in, to);
      }
    return LBFEM_OK;
  }

  // One system of MassSolver::solve (mass.h:185-213) on device buffers: x_new <-
  // A^{-1} b, CG from the start in x_new; sc / tg3: the TG3 matrix of system 0.
  int
  mass_solve_dev(lbfem_gpu_ctx *ctx, const double *b, double *x_new, bool tg3, const StreamCoef &sc, int64_t *its)
  {
    const int nsys = 1;
    if (ctx->distorted)
      {
        if (tg3)
          return fail(ctx, LBFEM_ERR_UNSUPPORTED, "general quadrilaterals: no TG3 matrix");
        int64_t q = 0;
        const int st = quad_solve(ctx, b, x_new, nsys, &q);
        if (its)
          *its = q;
        ctx->cg_its += q;
        return st;
      }
    if (ctx->prm.mass == LBFEM_MASS_LUMPED)
      {
        k_lumped<double, double><<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), b, x_new,
                                                                                               nsys);
        LAUNCHED();
        if (its)
          *its = 0;
        return strip_exchange(ctx, x_new, nsys, sizeof(double));
      }
    if (ctx->prm.mass == LBFEM_MASS_RICHARDSON)
      {
        // x_new <- the passes (the start in x_new is not used, as in the reference)
        int st = richardson_passes<double>(ctx, b, x_new, ctx->d_v, nsys);
        if (its)
          *its = 0;
        return st;
      }
    CgCall c;
    c.b = b;
    c.x_new = x_new;
    c.nsys = nsys;
    c.opk = tg3 ? OPK_TG3 : OPK_MASS;
    c.sc = sc;
    return cg_solve(ctx, c, its);
  }

  // ------------------------------------------------------- host <-> device
  // Copies nb blocks of a caller-numbered host vector into structured device storage.
  int
  upload(lbfem_gpu_ctx *ctx, const double *host, double *dst, int nb)
  {
    const long long N = ctx->grid.N;
    if (ctx->identity)
      {
        CK(cudaMemcpyAsync(dst, host, sizeof(double) * nb * N, cudaMemcpyHostToDevice, ctx->stream));
        return LBFEM_OK;
      }
    CK(cudaMemcpyAsync(ctx->d_stage, host, sizeof(double) * nb * ctx->n_dofs, cudaMemcpyHostToDevice, ctx->stream));
    k_gather<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(ctx->d_stage, ctx->d_dof, dst, N, ctx->n_dofs, nb);
    LAUNCHED();
    return LBFEM_OK;
  }

  int
  download(lbfem_gpu_ctx *ctx, const double *src, double *host, int nb)
  {
    const long long N = ctx->grid.N;
    if (ctx->identity)
      {
        CK(cudaMemcpyAsync(host, src, sizeof(double) * nb * N, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return LBFEM_OK;
      }
    k_scatter<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(src, ctx->d_dof, ctx->d_stage, N, ctx->n_dofs, nb);
    LAUNCHED();
    CK(cudaMemcpyAsync(host, ctx->d_stage, sizeof(double) * nb * ctx->n_dofs, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LBFEM_OK;
  }

  // Copies nb blocks of a caller-numbered DEVICE vector into structured device
  // storage (a permutation gather; with the structured numbering the caller's
  // buffer is used in place and nothing is copied: *use points at it).
  int
  gather_dev(lbfem_gpu_ctx *ctx, const double *src, double *dst, int nb, const double **use)
  {
    if (ctx->identity)
      {
        *use = src;
        return LBFEM_OK;
      }
    k_gather<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(src, ctx->d_dof, dst, ctx->grid.N,
                                                                           ctx->n_dofs, nb);
    LAUNCHED();
    *use = dst;
    return LBFEM_OK;
  }

  // The output side of gather_dev: where a kernel writes so that the caller's
  // device vector dst ends up holding the result (dst itself with the
  // structured numbering, else the context's scratch, scattered by scatter_dev).
  double *
  out_dev(const lbfem_gpu_ctx *ctx, double *dst, double *scratch)
  {
    return ctx->identity ? dst : scratch;
  }

  int
  scatter_dev(lbfem_gpu_ctx *ctx, const double *src, double *dst, int nb)
  {
    if (ctx->identity)
      return LBFEM_OK;
    k_scatter<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(src, ctx->d_dof, dst, ctx->grid.N,
                                                                            ctx->n_dofs, nb);
    LAUNCHED();
    return LBFEM_OK;
  }

  // Orders the context's stream after the work queued so far on the caller's
  // stream (an event wait on the device; the host does not wait).
  int
  join_caller(lbfem_gpu_ctx *ctx, void *stream)
  {
    CK(cudaEventRecord(ctx->ev_join[0], static_cast<cudaStream_t>(stream)));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join[0], 0));
    return LBFEM_OK;
  }

  // Makes the work queued later on the caller's stream wait for the context's stream.
  int
  release_caller(lbfem_gpu_ctx *ctx, void *stream)
  {
    CK(cudaEventRecord(ctx->ev_join[1], ctx->stream));
    CK(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), ctx->ev_join[1], 0));
    return LBFEM_OK;
  }

  // ------------------------------------------------------------ one step
  // A step is front (streaming right-hand side, wall faces), solve (the mass
  // solve of the 8 increments) and back (the nodal update that completes it).
  // LeeLin::step is schemes.h:92-98, Bardow::step schemes.h:118-124 (collide,
  // then stream, streaming.h:88-100). The mixed-precision step runs the same
  // sequence on FP32 deviations d = f - w.
  // The number of sweeps of a step: 2 for split TG3 (x, then y), else 1.
  int
  n_sweeps(const lbfem_gpu_ctx *ctx)
  {
    return ctx->prm.streaming == LBFEM_STREAMING_TG3_SPLIT ? 2 : 1;
  }

  // The directions of the populations in sweep s: D2Q9::e, or for the split TG3
  // sweeps D2Q9::e with the other component zeroed (TaylorGalerkin::axis,
  // streaming.h:107-115).
  void
  sweep_directions(const lbfem_gpu_ctx *ctx, int s, double *e)
  {
    const double *e0 = d2q9_e();
    const bool split = n_sweeps(ctx) == 2;
    for (int k = 0; k < Q; ++k)
      {
        e[2 * k] = split && s == 1 ? 0. : e0[2 * k];
        e[2 * k + 1] = split && s == 0 ? 0. : e0[2 * k + 1];
      }
  }

  // The CG solve of sweep s of an FP64 step (TaylorGalerkin::increment,
  // streaming.h:66-85): TG2 / TG3 start from the extrapolation of the two
  // previous increments into x_new; a split sweep starts from its own previous
  // increment in d_x[s] and skips the populations at rest in the sweep.
  CgCall
  step_cg_call(const lbfem_gpu_ctx *ctx, int s)
  {
    double e[2 * Q];
    sweep_directions(ctx, s, e);
    CgCall c;
    c.b = ctx->d_rhs;
    c.nsys = NM;
    const bool tg3 = ctx->prm.streaming != LBFEM_STREAMING_TG2;
    c.opk = tg3 ? OPK_TG3 : OPK_MASS;
    c.sc = stream_coef(e, tg3 ? ctx->dt * ctx->dt / 6. : 0.);
    if (n_sweeps(ctx) == 2)
      {
        c.x_new = ctx->d_x[s];
        c.extrapolate = 0;
        c.skip = resting(e);
      }
    else
      {
        c.x_new = ctx->d_x[ctx->x_new];
        c.x_cur = ctx->d_x[ctx->x_cur];
        c.x_prev = ctx->d_x[ctx->x_prev];
        c.extrapolate = 1;
      }
    return c;
  }

  // Sweep s of the front of a step: the streaming right-hand side of the sweep's
  // directions. The first sweep of Bardow collides on the fly into the other
  // population buffer; the second split sweep streams that buffer as it stands.
  struct FrontCoef
  {
    double e[2 * Q]; // the sweep's directions
    AdvCoef ac;      // the streaming right-hand side's coefficients
    bool bardow, remove;
  };

  FrontCoef
  front_coef(const lbfem_gpu_ctx *ctx, int sweep)
  {
    FrontCoef fr;
    const double dt = ctx->dt, lam = ctx->lambda;
    sweep_directions(ctx, sweep, fr.e);
    const int rm = ctx->prm.remove_wall_mass_flux;
    fr.bardow = ctx->prm.scheme == LBFEM_SCHEME_BARDOW;
    const double b = -0.5 * dt * dt / lam;
    fr.ac = fr.bardow ? adv_coef(-dt, 0., -0.5 * dt * dt, fr.e, dt / (lam + 0.5 * dt))
                      : adv_coef(-dt - b, b, -0.5 * dt * dt, fr.e, 0.);
    fr.remove = rm < 0 ? fr.bardow : rm != 0;
    return fr;
  }

  int
  step_front(lbfem_gpu_ctx *ctx, int sweep = 0)
  {
    const FrontCoef fr = front_coef(ctx, sweep);
    const double dt = ctx->dt;
    const double *e = fr.e;
    const AdvCoef &ac = fr.ac;
    const bool bardow = fr.bardow, remove = fr.remove;
    int st;
    if (ctx->mixed)
      {
        float *d = ctx->d_fs[ctx->cur], *g = ctx->d_fs[1 - ctx->cur];
        if ((st = launch_pair(ctx, bardow ? PAIR_BARDOW : PAIR_LEELIN, d, bardow ? g : nullptr, ctx->d_rhs_s, ac,
                              ctx->d_stats)))
          return st;
        return launch_wall_faces<float>(ctx, bardow ? g : d, ctx->d_rhs_s, e, dt, remove);
      }
    double *f = ctx->d_f[ctx->cur], *g = ctx->d_f[1 - ctx->cur];
    if (sweep > 0)
      st = launch_advection<double>(ctx, ADV_TG, g, nullptr, nullptr, ctx->d_rhs, ac, ctx->d_stats);
    else
      st = launch_advection<double>(ctx, bardow ? ADV_TG_COLLIDE : ADV_LEELIN_FUSED, f, nullptr, bardow ? g : nullptr,
                                    ctx->d_rhs, ac, ctx->d_stats);
    if (st)
      return st;
    return launch_wall_faces<double>(ctx, bardow ? g : f, ctx->d_rhs, e, dt, remove);
  }

  // The nodal update of sweep s with its increment (x_cur, or d_x[s] for a split
  // sweep). Bardow: f = g* + x (TaylorGalerkin::stream, streaming.h:88-100),
  // which flips the population buffers after the last sweep; Lee-Lin: the
  // predictor-corrector.
  int
  step_back(lbfem_gpu_ctx *ctx, int sweep = 0)
  {
    const Geo geo = geo_of(ctx);
    const int nb = n_pointwise_blocks(ctx->grid.N);
    const double theta = ctx->dt / ctx->lambda;
    if (ctx->prm.scheme == LBFEM_SCHEME_BARDOW)
      {
        const bool last = sweep == n_sweeps(ctx) - 1;
        if (ctx->mixed)
          k_add_increment<float><<<nb, THREADS, 0, ctx->stream>>>(geo, ctx->d_stats, ctx->d_fs[1 - ctx->cur],
                                                                  ctx->d_x_s[ctx->x_cur], 1);
        else
          k_add_increment<double><<<nb, THREADS, 0, ctx->stream>>>(
            geo, ctx->d_stats, ctx->d_f[1 - ctx->cur], n_sweeps(ctx) == 2 ? ctx->d_x[sweep] : ctx->d_x[ctx->x_cur],
            last ? 1 : 0);
        LAUNCHED();
        if (last)
          ctx->cur = 1 - ctx->cur;
        return LBFEM_OK;
      }
    if (ctx->mixed)
      k_predictor_corrector_dev<<<nb, THREADS, 0, ctx->stream>>>(geo, ctx->d_stats, ctx->d_fs[ctx->cur],
                                                                 ctx->d_x_s[ctx->x_cur], theta);
    else
      k_predictor_corrector<<<nb, THREADS, 0, ctx->stream>>>(geo, ctx->d_stats, ctx->d_f[ctx->cur], nullptr,
                                                             ctx->d_x[ctx->x_cur], theta);
    LAUNCHED();
    return LBFEM_OK;
  }

  // The lumped solve x_cur = M_L^{-1} rhs, or the iterated lumping into x_cur with
  // x_new's buffer as scratch (no history either way).
  int
  lumped_solve(lbfem_gpu_ctx *ctx)
  {
    const Geo geo = geo_of(ctx);
    const int nb = n_pointwise_blocks(ctx->grid.N);
    if (ctx->prm.mass == LBFEM_MASS_RICHARDSON)
      return ctx->mixed ? richardson_passes<float>(ctx, ctx->d_rhs_s, ctx->d_x_s[ctx->x_cur],
                                                   ctx->d_x_s[ctx->x_new], NM)
                        : richardson_passes<double>(ctx, ctx->d_rhs, ctx->d_x[ctx->x_cur], ctx->d_x[ctx->x_new], NM);
    if (ctx->mixed)
      k_lumped<float, float><<<nb, THREADS, 0, ctx->stream>>>(geo, ctx->d_rhs_s, ctx->d_x_s[ctx->x_cur], NM);
    else
      k_lumped<double, double><<<nb, THREADS, 0, ctx->stream>>>(geo, ctx->d_rhs, ctx->d_x[ctx->x_cur], NM);
    LAUNCHED();
    if (ctx->mixed)
      return strip_exchange(ctx, ctx->d_x_s[ctx->x_cur], NM, sizeof(float));
    return strip_exchange(ctx, ctx->d_x[ctx->x_cur], NM, sizeof(double));
  }

  // ------------------------------------------------ general quadrilaterals
  // FP64, host-driven: cell-coloured kernels (quad.cuh) and the CG of the
  // oracle's order (deal.II SolverCG), one system at a time.
  template <typename F>
  int
  quad_colours(const lbfem_gpu_ctx *ctx, F &&launch)
  {
    const Grid &g = ctx->grid;
    const int nx = (g.px && (g.ncx & 1)) ? 3 : 2, ny = (g.py && (g.ncy & 1)) ? 3 : 2;
    for (int cy = 0; cy < ny; ++cy)
      for (int cx = 0; cx < nx; ++cx)
        {
          QuadGeo qg{ctx->d_qgeo, cx, cy, g.ncx, g.ncy, nx == 3, ny == 3};
          int st = launch(qg);
          if (st)
            return st;
        }
    return LBFEM_OK;
  }

  long long
  quad_threads(const lbfem_gpu_ctx *ctx, int per_cell)
  {
    const Grid &g = ctx->grid;
    return (long long)((g.ncx + 1) / 2 + 1) * ((g.ncy + 1) / 2 + 1) * per_cell;
  }

  // rhs (8 blocks) <- the advection of f (and feq) on the mapped cells
  int
  quad_advection(lbfem_gpu_ctx *ctx, const double *f, const double *feq, double *rhs, const AdvCoef &ac)
  {
    CK(cudaMemsetAsync(rhs, 0, sizeof(double) * NM * ctx->grid.N, ctx->stream));
    const Geo geo = geo_of(ctx);
    const int nb = int((quad_threads(ctx, NM) + 127) / 128);
    return with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      return quad_colours(ctx, [&](const QuadGeo &qg) -> int {
        k_quad_advection<P><<<nb, 128, 0, ctx->stream>>>(geo, qg, f, feq, rhs, ac);
        LAUNCHED();
        return LBFEM_OK;
      });
    });
  }

  // y <- M x for nsys systems (constrained rows the identity)
  int
  quad_vmult(lbfem_gpu_ctx *ctx, const double *x, double *y, int nsys)
  {
    CK(cudaMemsetAsync(y, 0, sizeof(double) * nsys * ctx->grid.N, ctx->stream));
    const Geo geo = geo_of(ctx);
    const int nb = int((quad_threads(ctx, nsys) + 127) / 128);
    int st = with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      return quad_colours(ctx, [&](const QuadGeo &qg) -> int {
        k_quad_mass<P><<<nb, 128, 0, ctx->stream>>>(geo, qg, x, y, nsys);
        LAUNCHED();
        return LBFEM_OK;
      });
    });
    if (st)
      return st;
    k_quad_images<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo, x, y, nsys);
    LAUNCHED();
    return LBFEM_OK;
  }

  int
  quad_dot(lbfem_gpu_ctx *ctx, const double *a, const double *b, double *out)
  {
    const int nb = n_pointwise_blocks(ctx->grid.N);
    k_quad_dot<<<nb, THREADS, 0, ctx->stream>>>(geo_of(ctx), a, b, ctx->d_partials);
    LAUNCHED();
    k_reduce_partials<<<1, 256, 0, ctx->stream>>>(ctx->d_partials, nb, ctx->d_sums);
    LAUNCHED();
    CK(cudaMemcpyAsync(out, ctx->d_sums, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LBFEM_OK;
  }

  // y = a x + b y (mode 0) or y = x * d (mode 1), one system
  int
  quad_axpby(lbfem_gpu_ctx *ctx, double a, const double *x, double b, double *y, const double *d = nullptr)
  {
    k_quad_axpby<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(ctx->grid.N, a, x, b, y, d,
                                                                              d ? 1 : 0);
    LAUNCHED();
    return LBFEM_OK;
  }

  // x <- M^{-1} b, Jacobi-PCG from the start in x, in deal.II SolverCG's order of
  // updates (mass.h:204-211), as the oracle; work vectors r, z, p, v of N values.
  int
  quad_cg(lbfem_gpu_ctx *ctx, const double *b, double *x, int64_t *its)
  {
    const long long N = ctx->grid.N;
    double *r = ctx->d_r, *z = ctx->d_r + N, *p = ctx->d_r + 2 * N, *v = ctx->d_r + 3 * N;
    const double tol0 = ctx->prm.cg_tolerance;
    int st;
    double bb = 0, res = 0, rz = 0;
    *its = 0;
    if ((st = quad_dot(ctx, b, b, &bb)))
      return st;
    const double tol = tol0 * std::sqrt(bb);
    if (bb == 0.)
      {
        // an exactly zero right-hand side: x = 0 (deal.II would iterate toward a tolerance of 0)
        CK(cudaMemsetAsync(x, 0, sizeof(double) * N, ctx->stream));
        return LBFEM_OK;
      }
    // r = b - A x (A 0 = 0 exactly, so a zero start gives r = b as deal.II's)
    if ((st = quad_vmult(ctx, x, v, 1)))
      return st;
    CK(cudaMemcpyAsync(r, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
    if ((st = quad_axpby(ctx, -1., v, 1., r)) || (st = quad_dot(ctx, r, r, &res)))
      return st;
    res = std::sqrt(res);
    if (std::isnan(res))
      return fail(ctx, LBFEM_ERR_NONFINITE, "CG: non-finite residual");
    if (res <= tol)
      return LBFEM_OK;
    for (int it = 1;; ++it)
      {
        if ((st = quad_axpby(ctx, 0., r, 0., z, ctx->d_qijac)))
          return st;
        const double rz_prev = rz;
        if ((st = quad_dot(ctx, r, z, &rz)))
          return st;
        if (it > 1)
          st = quad_axpby(ctx, 1., z, rz / rz_prev, p);
        else
          st = cudaMemcpyAsync(p, z, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream) == cudaSuccess
                 ? LBFEM_OK
                 : fail(ctx, LBFEM_ERR_CUDA, "CG: copy failed");
        double pAp = 0;
        if (st || (st = quad_vmult(ctx, p, v, 1)) || (st = quad_dot(ctx, p, v, &pAp)))
          return st;
        const double alpha = rz / pAp;
        if ((st = quad_axpby(ctx, alpha, p, 1., x)) || (st = quad_axpby(ctx, -alpha, v, 1., r)) ||
            (st = quad_dot(ctx, r, r, &res)))
          return st;
        res = std::sqrt(res);
        *its = it;
        if (std::isnan(res))
          return fail(ctx, LBFEM_ERR_NONFINITE, "CG: non-finite residual");
        if (res <= tol)
          return LBFEM_OK;
        if (it >= ctx->prm.cg_max_iterations)
          return fail(ctx, LBFEM_ERR_NO_CONVERGENCE, "CG: iteration cap %d reached", ctx->prm.cg_max_iterations);
      }
  }

  // The mass solve of nsys systems on the mapped cells: lumped, iterated lumping, or CG
  // per system from the start in x.
  int
  quad_solve(lbfem_gpu_ctx *ctx, const double *b, double *x, int nsys, int64_t *its)
  {
    const long long N = ctx->grid.N;
    int st;
    *its = 0;
    if (ctx->prm.mass != LBFEM_MASS_CG)
      {
        for (int s = 0; s < nsys; ++s)
          if ((st = quad_axpby(ctx, 0., b + s * N, 0., x + s * N, ctx->d_qilump)))
            return st;
        if (ctx->prm.mass == LBFEM_MASS_RICHARDSON)
          for (int k = 0; k < ctx->prm.richardson; ++k)
            for (int s = 0; s < nsys; ++s)
              {
                // x += M_L^{-1} (b - M x)
                double *v = ctx->d_v, *w = ctx->d_v + N;
                if ((st = quad_vmult(ctx, x + s * N, v, 1)))
                  return st;
                CK(cudaMemcpyAsync(w, b + s * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
                if ((st = quad_axpby(ctx, -1., v, 1., w)) || (st = quad_axpby(ctx, 0., w, 0., v, ctx->d_qilump)) ||
                    (st = quad_axpby(ctx, 1., v, 1., x + s * N)))
                  return st;
              }
        return LBFEM_OK;
      }
    for (int s = 0; s < nsys; ++s)
      {
        int64_t it = 0;
        if ((st = quad_cg(ctx, b + s * N, x + s * N, &it)))
          return st;
        *its += it;
      }
    return LBFEM_OK;
  }

  // Scheme::step on the mapped cells (LeeLin schemes.h:92-98, Bardow 118-124), FP64 TG2.
  int
  step_quad(lbfem_gpu_ctx *ctx, int64_t *its)
  {
    const Geo geo = geo_of(ctx);
    const long long N = ctx->grid.N;
    const int nb = n_pointwise_blocks(N);
    const double dt = ctx->dt, lam = ctx->lambda;
    const bool bardow = ctx->prm.scheme == LBFEM_SCHEME_BARDOW;
    double *f = ctx->d_f[ctx->cur];
    int st;
    if (bardow)
      {
        k_collide<<<nb, THREADS, 0, ctx->stream>>>(geo, f, dt / (lam + 0.5 * dt));
        LAUNCHED();
        st = quad_advection(ctx, f, nullptr, ctx->d_rhs, adv_coef(-dt, 0., -0.5 * dt * dt, d2q9_e(), 0.));
      }
    else
      {
        k_equilibrium<<<nb, THREADS, 0, ctx->stream>>>(geo, f, ctx->d_feq);
        LAUNCHED();
        const double b = -0.5 * dt * dt / lam;
        st = quad_advection(ctx, f, ctx->d_feq, ctx->d_rhs, adv_coef(-dt - b, b, -0.5 * dt * dt, d2q9_e(), 0.));
      }
    if (st)
      return st;
    // the CG start 2 x^n - x^{n-1} (TaylorGalerkin::increment, streaming.h:76-80)
    double *xn = ctx->d_x[ctx->x_new], *xc = ctx->d_x[ctx->x_cur], *xp = ctx->d_x[ctx->x_prev];
    if (ctx->prm.mass == LBFEM_MASS_CG)
      {
        CK(cudaMemcpyAsync(xn, xp, sizeof(double) * NM * N, cudaMemcpyDeviceToDevice, ctx->stream));
        k_quad_axpby<<<nb, THREADS, 0, ctx->stream>>>(NM * N, 2., xc, -1., xn, nullptr, 0);
        LAUNCHED();
      }
    if ((st = quad_solve(ctx, ctx->d_rhs, xn, NM, its)))
      return st;
    const int old_prev = ctx->x_prev;
    ctx->x_prev = ctx->x_cur;
    ctx->x_cur = ctx->x_new;
    ctx->x_new = old_prev;
    if (bardow)
      k_add_increment<double><<<nb, THREADS, 0, ctx->stream>>>(geo, nullptr, f, xn, 0);
    else
      k_predictor_corrector<<<nb, THREADS, 0, ctx->stream>>>(geo, nullptr, f, ctx->d_feq, xn, dt / lam);
    LAUNCHED();
    return LBFEM_OK;
  }

  // One host-driven step: the solver loops read their state back after every
  // iteration (the path of LBFEM_TRACE).
  int
  step_once(lbfem_gpu_ctx *ctx, int64_t *its)
  {
    int st;
    if (its)
      *its = 0;
    if (ctx->distorted)
      {
        int64_t q = 0;
        st = step_quad(ctx, &q);
        if (its)
          *its = q;
        return st;
      }
    for (int s = 0; s < n_sweeps(ctx); ++s)
      {
        if ((st = step_front(ctx, s)))
          return st;
        int64_t sweep_its = 0;
        if (ctx->prm.mass != LBFEM_MASS_CG)
          st = lumped_solve(ctx);
        else if (ctx->mixed)
          st = mixed_solve(ctx, ctx->d_rhs_s, NM, &sweep_its);
        else
          {
            st = cg_solve(ctx, step_cg_call(ctx, s), &sweep_its);
            if (!st && n_sweeps(ctx) == 1)
              {
                const int old_prev = ctx->x_prev;
                ctx->x_prev = ctx->x_cur;
                ctx->x_cur = ctx->x_new;
                ctx->x_new = old_prev;
              }
          }
        if (its)
          *its += sweep_its;
        if (st || (st = step_back(ctx, s)))
          return st;
      }
    return LBFEM_OK;
  }

  // ------------------------------------------------------- graph-launched steps
  // A whole step as one CUDA graph: the solver loops become conditional WHILE
  // nodes whose bodies end in a control kernel that sets the condition on the
  // device (no host round trip per iteration). Failures are recorded in the
  // sticky status of DevStats; the step-completing kernels then do nothing, so
  // the populations stay those before the failing step.

  // Appends a WHILE node after the work captured so far on ctx->stream and
  // captures body() into it on ctx->cap; *body_kernels: the kernels of one body.
  template <typename Body>
  int
  capture_while(lbfem_gpu_ctx *ctx, cudaGraphConditionalHandle h, Body &&body, int64_t *body_kernels)
  {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo_v3(ctx->stream, &cs, nullptr, &g, &deps, nullptr, &nd));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &np));
    CK(cudaStreamBeginCaptureToGraph(ctx->cap, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    const int64_t l0 = ctx->launches;
    std::swap(ctx->stream, ctx->cap);
    const int st = body();
    std::swap(ctx->stream, ctx->cap);
    cudaGraph_t bg = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->cap, &bg);
    if (st)
      return st;
    if (e != cudaSuccess)
      return fail(ctx, LBFEM_ERR_CUDA, "loop body capture: %s", cudaGetErrorString(e));
    *body_kernels = ctx->launches - l0;
    CK(cudaStreamUpdateCaptureDependencies_v2(ctx->stream, &node, nullptr, 1, cudaStreamSetCaptureDependencies));
    return LBFEM_OK;
  }

  // Jacobi-PCG of the FP64 step (the order of cg_run), with the loop on the
  // device. One loop body is two iterations: the search directions alternate
  // between two buffers, and an iteration of a converged system does nothing.
  int
  cg_graph(lbfem_gpu_ctx *ctx, const CgCall &c, int64_t *body_kernels)
  {
    const double tol = c.tol >= 0 ? c.tol : ctx->prm.cg_tolerance;
    const int max_its = c.max_its > 0 ? c.max_its : ctx->prm.cg_max_iterations;
    const CgScratch<double> w = ctx_scratch(ctx);
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamGetCaptureInfo_v3(ctx->stream, &cs, nullptr, &graph, nullptr, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault)); // 0 at every launch
    CK(cudaMemsetAsync(w.state, 0, sizeof(CgState), ctx->stream));
    int n_tiles = 0, st;
    if ((st = cg_launch_start(ctx, w, c, &n_tiles)) || (st = reduce_into(ctx, w.partials, w.sums, n_tiles, 3 * NM)))
      return st;
    k_cg_scalars<<<1, 32, 0, ctx->stream>>>(w.state, w.sums, c.nsys, 0, tol, max_its);
    LAUNCHED();
    if ((st = zero_flagged(ctx, c.x_new, w.state, c.nsys)))
      return st;
    k_cg_control<<<1, 32, 0, ctx->stream>>>(w.state, ctx->d_stats, h, 0);
    LAUNCHED();
    auto iteration = [&](int pi) -> int {
      int s2;
      if ((s2 = cg_launch_p(ctx, w, c, pi)) || (s2 = reduce_into(ctx, w.partials, w.sums, n_tiles, NM)))
        return s2;
      k_cg_scalars<<<1, 32, 0, ctx->stream>>>(w.state, w.sums, c.nsys, 1, tol, max_its);
      LAUNCHED();
      if ((s2 = cg_launch_update(ctx, w, c, 1 - pi)) || (s2 = reduce_into(ctx, w.partials, w.sums, n_tiles, 2 * NM)))
        return s2;
      k_cg_scalars<<<1, 32, 0, ctx->stream>>>(w.state, w.sums, c.nsys, 2, tol, max_its);
      LAUNCHED();
      return LBFEM_OK;
    };
    return capture_while(
      ctx, h,
      [&]() -> int {
        int s2;
        if ((s2 = iteration(0)) || (s2 = iteration(1)))
          return s2;
        k_cg_control<<<1, 32, 0, ctx->stream>>>(w.state, ctx->d_stats, h, 1);
        LAUNCHED();
        return LBFEM_OK;
      },
      body_kernels);
  }

  // The mixed-precision solve of mixed_solve with the rounds on the device. One
  // loop body is two rounds, x_prev's buffer -> x_new's -> x_prev's; a round of a
  // converged system copies, so the solution always ends in x_prev's buffer.
  int
  mixed_graph(lbfem_gpu_ctx *ctx, int64_t *body_kernels)
  {
    const Geo geo = geo_of(ctx);
    const Grid &g = ctx->grid;
    const double tol = mixed_tolerance(ctx->prm);
    const int max_rounds = ctx->prm.cg_max_iterations;
    const float *b = ctx->d_rhs_s;
    float *xn = ctx->d_x_s[ctx->x_new], *xp = ctx->d_x_s[ctx->x_prev];
    const float *xc = ctx->d_x_s[ctx->x_cur];
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamGetCaptureInfo_v3(ctx->stream, &cs, nullptr, &graph, nullptr, nullptr, nullptr));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault)); // 0 at every launch
    CK(cudaMemsetAsync(ctx->d_cg, 0, sizeof(CgState), ctx->stream));
    int st = with_degree(ctx->P, [&](auto PP) -> int {
      constexpr int P = decltype(PP)::value;
      k_mixed_start<P><<<start_grid<P>(g, NM), StartShape<P>::THREADS, 0, ctx->stream>>>(geo, b, xc, xp, xn,
                                                                                       ctx->d_r_s);
      LAUNCHED();
      return LBFEM_OK;
    });
    if (st)
      return st;
    auto round = [&](const float *r_in, const float *x_in, float *x_out, float *r_out, int all, int set) -> int {
      int n_tiles = 0;
      int s2 = with_degree(ctx->P, [&](auto PP) -> int {
        constexpr int P = decltype(PP)::value;
        using S = WinShape<P>;
        const dim3 grid(tiles_along(g.nfx, g.nux, g.px, S::TX), tiles_along(g.nfy, g.nuy, g.py, S::TY), NM);
        n_tiles = int(grid.x * grid.y);
        k_window_correct<P><<<grid, S::THREADS, window_smem<P>(), ctx->stream>>>(
          geo, ctx->d_winx, ctx->d_winy, r_in, x_in, b, x_out, r_out, ctx->d_cg, all, ctx->d_partials);
        LAUNCHED();
        return LBFEM_OK;
      });
      if (s2 || (s2 = reduce_into(ctx, ctx->d_partials, ctx->d_sums, n_tiles, 2 * NM)))
        return s2;
      k_mixed_round<<<1, 32, 0, ctx->stream>>>(ctx->d_cg, ctx->d_sums, ctx->d_stats, NM, tol, max_rounds, h, set);
      LAUNCHED();
      return LBFEM_OK;
    };
    float *r0 = ctx->d_r_s, *r1 = ctx->d_p_s[0];
    if ((st = round(r0, xn, xp, r1, 1, 1)) || (st = zero_flagged(ctx, xp, ctx->d_cg, NM)))
      return st;
    return capture_while(
      ctx, h,
      [&]() -> int {
        int s2;
        if ((s2 = round(r1, xp, xn, r0, 0, 0)) || (s2 = round(r0, xn, xp, r1, 0, 1)))
          return s2;
        return LBFEM_OK;
      },
      body_kernels);
  }

  // The buffer rotation a graph-launched step applies (host bookkeeping).
  void
  rotate_after_step(lbfem_gpu_ctx *ctx)
  {
    if (ctx->prm.mass == LBFEM_MASS_CG && n_sweeps(ctx) == 1)
      {
        const int c = ctx->x_cur, p = ctx->x_prev, n = ctx->x_new;
        if (ctx->mixed)
          {
            ctx->x_cur = p; // the rounds end in x_prev's buffer
            ctx->x_prev = c;
            ctx->x_new = n;
          }
        else
          {
            ctx->x_cur = n;
            ctx->x_prev = c;
            ctx->x_new = p;
          }
      }
    if (ctx->prm.scheme == LBFEM_SCHEME_BARDOW)
      ctx->cur = 1 - ctx->cur;
  }

  int
  graph_key(const lbfem_gpu_ctx *ctx)
  {
    return ctx->cur * 9 + ctx->x_cur * 3 + ctx->x_prev;
  }

  // Records one step of the current buffer state on ctx->stream, which is being
  // captured (into a step graph of its own or into a batch graph); the buffer
  // state is left as it was. *fixed: the kernels outside the solver loop; *body:
  // the kernels of one loop body.
  int
  record_step(lbfem_gpu_ctx *ctx, int64_t *fixed, int64_t *body)
  {
    const int cur0 = ctx->cur, c0 = ctx->x_cur, p0 = ctx->x_prev, n0 = ctx->x_new;
    const int64_t l0 = ctx->launches;
    *body = 0;
    int64_t bodies = 0; // kernels of the loop bodies of all sweeps (the same in each)
    int st = LBFEM_OK;
    const int ns = n_sweeps(ctx);
    for (int s = 0; s < ns && !st; ++s)
      {
        st = step_front(ctx, s);
        if (!st && ctx->prm.mass == LBFEM_MASS_CG)
          {
            int64_t b = 0;
            st = ctx->mixed ? mixed_graph(ctx, &b) : cg_graph(ctx, step_cg_call(ctx, s), &b);
            *body = b;
            bodies += b;
          }
        else if (!st)
          st = lumped_solve(ctx);
        if (!st)
          {
            if (s == ns - 1)
              {
                rotate_after_step(ctx);
                if (ctx->prm.scheme == LBFEM_SCHEME_BARDOW)
                  ctx->cur = 1 - ctx->cur; // step_back flips it again
              }
            st = step_back(ctx, s);
          }
      }
    *fixed = ctx->launches - l0 - bodies;
    ctx->cur = cur0;
    ctx->x_cur = c0;
    ctx->x_prev = p0;
    ctx->x_new = n0;
    ctx->launches = l0;
    return st;
  }

  // Captures and instantiates the step graph of the current buffer state.
  int
  capture_step(lbfem_gpu_ctx *ctx, lbfem_gpu_ctx::StepGraph &sg)
  {
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int64_t fixed = 0, body = 0;
    const int st = record_step(ctx, &fixed, &body);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st || e != cudaSuccess)
      {
        if (graph)
          cudaGraphDestroy(graph);
        return st ? st : fail(ctx, LBFEM_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
      }
    const cudaError_t ei = cudaGraphInstantiate(&sg.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess)
      return fail(ctx, LBFEM_ERR_CUDA, "step graph instantiation: %s", cudaGetErrorString(ei));
    sg.fixed = fixed;
    sg.body = body;
    return LBFEM_OK;
  }

  // The buffer state and counters of a context before a run of graph-launched steps.
  struct RunStart
  {
    DevStats stats;
    int cur, x_cur, x_prev, x_new;
    int64_t fixed = 0, body = 0; // kernels of the launched steps outside the loops; per loop body
  };

  RunStart
  run_start(const lbfem_gpu_ctx *ctx, const DevStats &stats)
  {
    RunStart r{};
    r.stats = stats;
    r.cur = ctx->cur;
    r.x_cur = ctx->x_cur;
    r.x_prev = ctx->x_prev;
    r.x_new = ctx->x_new;
    return r;
  }

  // The step graph of the current buffer state (captured on first use).
  int
  current_step_graph(lbfem_gpu_ctx *ctx, lbfem_gpu_ctx::StepGraph **out)
  {
    auto &sg = ctx->graphs[graph_key(ctx)];
    int st;
    if (!sg.exec && (st = capture_step(ctx, sg)))
      return st;
    *out = &sg;
    return LBFEM_OK;
  }

  int finish_run(lbfem_gpu_ctx *ctx, const RunStart &r0, const DevStats &after, int64_t *its_total,
                 int64_t *launches);

  // n steps as graph launches, with one synchronisation at the end.
  int
  step_graphs(lbfem_gpu_ctx *ctx, int n, int64_t *its_total, int64_t *launches)
  {
    CK(cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    RunStart r0 = run_start(ctx, *ctx->h_stats);
    for (int k = 0; k < n; ++k)
      {
        lbfem_gpu_ctx::StepGraph *sg;
        int st;
        if ((st = current_step_graph(ctx, &sg)))
          return st;
        CK(cudaGraphLaunch(sg->exec, ctx->stream));
        r0.fixed += sg->fixed;
        r0.body = sg->body;
        rotate_after_step(ctx);
      }
    CK(cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return finish_run(ctx, r0, *ctx->h_stats, its_total, launches);
  }

  // After a run: the counters, and on a failure the buffer state of the completed steps, a
  // restarted extrapolation history and the failure's status.
  int
  finish_run(lbfem_gpu_ctx *ctx, const RunStart &r0, const DevStats &after, int64_t *its_total, int64_t *launches)
  {
    const DevStats &before = r0.stats;
    const int cur0 = r0.cur, c0 = r0.x_cur, p0 = r0.x_prev, n0 = r0.x_new;
    *its_total = int64_t(after.its - before.its);
    *launches = r0.fixed + int64_t(after.bodies - before.bodies) * r0.body;
    if (after.sticky)
      {
        // the steps after the failing one did nothing: put the buffer state back to
        // the completed steps, restart the extrapolation history, clear the failure
        ctx->cur = cur0;
        ctx->x_cur = c0;
        ctx->x_prev = p0;
        ctx->x_new = n0;
        for (unsigned long long k = 0; k < after.steps_done - before.steps_done; ++k)
          rotate_after_step(ctx);
        const long long N = ctx->grid.N;
        for (int k = 0; k < 3; ++k)
          {
            CK(cudaMemsetAsync(ctx->d_x[k], 0, sizeof(double) * NM * N, ctx->stream));
            if (ctx->mixed)
              CK(cudaMemsetAsync(ctx->d_x_s[k], 0, sizeof(float) * NM * N, ctx->stream));
          }
        CK(cudaMemsetAsync(&ctx->d_stats->sticky, 0, sizeof(int), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const double tol = ctx->mixed ? mixed_tolerance(ctx->prm) : ctx->prm.cg_tolerance;
        if (ctx->mixed)
          return mixed_status(ctx, after.sticky, tol);
        if (after.sticky == 3)
          return fail(ctx, LBFEM_ERR_NONFINITE, "CG: non-finite residual");
        return fail(ctx, LBFEM_ERR_NO_CONVERGENCE, "CG: iteration cap %d reached", ctx->prm.cg_max_iterations);
      }
    return LBFEM_OK;
  }

  int
  check_ctx(lbfem_gpu_ctx *ctx)
  {
    if (!ctx)
      return LBFEM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    return LBFEM_OK;
  }
} // namespace


namespace
{
  // The raw population checkpoint shared by write and read (io.h:137-165).
  std::string
  checkpoint_path(const char *name, int32_t rank)
  {
    return std::string(name) + "." + std::to_string(rank);
  }

  int
  write_raw(const std::string &file, const std::vector<double> &f)
  {
    const std::string tmp = file + ".tmp";
    FILE *out = std::fopen(tmp.c_str(), "wb");
    if (!out)
      return LBFEM_ERR_ARG;
    const size_t n = std::fwrite(f.data(), sizeof(double), f.size(), out);
    const int closed = std::fclose(out);
    if (n != f.size() || closed != 0 || std::rename(tmp.c_str(), file.c_str()) != 0)
      {
        std::remove(tmp.c_str());
        return LBFEM_ERR_ARG;
      }
    return LBFEM_OK;
  }

  int
  read_raw(const std::string &file, std::vector<double> &f)
  {
    FILE *in = std::fopen(file.c_str(), "rb");
    if (!in)
      return LBFEM_ERR_ARG;
    const size_t n = std::fread(f.data(), sizeof(double), f.size(), in);
    const bool more = std::fgetc(in) != EOF;
    std::fclose(in);
    return n == f.size() && !more ? LBFEM_OK : LBFEM_ERR_ARG;
  }
} // namespace

extern "C" {

void
lbfem_gpu_default_params(lbfem_params *p)
{
  if (!p)
    return;
  p->scheme = LBFEM_SCHEME_BARDOW;
  p->mass = LBFEM_MASS_CG;
  p->richardson = 2;
  p->streaming = LBFEM_STREAMING_TG2;
  p->precision = LBFEM_PRECISION_FP64;
  p->cg_max_iterations = 200;
  p->cg_tolerance = 1e-8;
  p->remove_wall_mass_flux = -1;
  p->device = 0;
  p->mixed_tolerance = 0.0;
}

const char *
lbfem_gpu_status_string(int s)
{
  switch (s)
    {
      case LBFEM_OK:
        return "ok";
      case LBFEM_ERR_ARG:
        return "bad argument";
      case LBFEM_ERR_NO_CONVERGENCE:
        return "CG did not converge within the iteration cap";
      case LBFEM_ERR_NONFINITE:
        return "non-finite value";
      case LBFEM_ERR_CUDA:
        return "CUDA error";
      case LBFEM_ERR_UNSUPPORTED:
        return "unsupported option";
      case LBFEM_ERR_TIMEOUT:
        return "device-side wait timed out";
      case LBFEM_ERR_STATE:
        return "call out of order";
      default:
        return "unknown status";
    }
}

const char *
lbfem_gpu_last_error(const lbfem_gpu_ctx *ctx)
{
  return ctx ? ctx->err.c_str() : "";
}

int
lbfem_gpu_device_count(void)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess)
    {
      cudaGetLastError();
      return 0;
    }
  return n;
}

int
lbfem_gpu_reference_matrix(int32_t degree, int32_t op, double *ref64, float *ref32)
{
  if (degree < 1 || degree > MAXPD || op < 0 || op > 2)
    return LBFEM_ERR_ARG;
  static double ref[MAXPD][3][MAXPD + 1][MAXPD + 1];
  static float reff[MAXPD][3][MAXPD + 1][MAXPD + 1];
  static std::once_flag once;
  std::call_once(once, [] { reference_matrices(ref, reff); });
  for (int a = 0; a <= degree; ++a)
    for (int c = 0; c <= degree; ++c)
      {
        if (ref64)
          ref64[a * (degree + 1) + c] = ref[degree - 1][op][a][c];
        if (ref32)
          ref32[a * (degree + 1) + c] = reff[degree - 1][op][a][c];
      }
  return LBFEM_OK;
}

void *
lbfem_gpu_host_alloc(size_t bytes)
{
  void *p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess)
    {
      cudaGetLastError();
      return nullptr;
    }
  return p;
}

void
lbfem_gpu_host_free(void *p)
{
  if (p)
    cudaFreeHost(p);
}

int
lbfem_gpu_destroy(lbfem_gpu_ctx *ctx)
{
  if (!ctx)
    return LBFEM_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream)
    cudaStreamSynchronize(ctx->stream);
  void *bufs[] = {ctx->d_hx, ctx->d_hxi, ctx->d_hy, ctx->d_hyi, ctx->d_ijx, ctx->d_ijy, ctx->d_ilx, ctx->d_ily,
                  ctx->d_rowx, ctx->d_rowy, ctx->d_diagx, ctx->d_diagy, ctx->d_lumpx, ctx->d_lumpy, ctx->d_wall,
                  ctx->d_wall_u, ctx->d_dof, ctx->d_bnode, ctx->d_f[0], ctx->d_f[1], ctx->d_rhs, ctx->d_x[0],
                  ctx->d_x[1], ctx->d_x[2], ctx->d_r, ctx->d_p[0], ctx->d_p[1], ctx->d_v, ctx->d_feq, ctx->d_stage,
                  ctx->d_partials, ctx->d_sums, ctx->d_cg, ctx->d_fs[0], ctx->d_fs[1], ctx->d_rhs_s,
                  ctx->d_x_s[0], ctx->d_x_s[1], ctx->d_x_s[2], ctx->d_r_s, ctx->d_p_s[0], ctx->d_p_s[1],
                  ctx->d_winx, ctx->d_winy, ctx->d_qgeo, ctx->d_qijac, ctx->d_qlump, ctx->d_qilump};
  for (void *b : bufs)
    if (b)
      cudaFree(b);
  if (ctx->h_cg)
    cudaFreeHost(ctx->h_cg);
  for (auto &kv : ctx->graphs)
    if (kv.second.exec)
      cudaGraphExecDestroy(kv.second.exec);
  if (ctx->d_stats)
    cudaFree(ctx->d_stats);
  if (ctx->h_stats)
    cudaFreeHost(ctx->h_stats);
  if (ctx->cap)
    cudaStreamDestroy(ctx->cap);
  for (auto &e : ctx->ev)
    if (e)
      cudaEventDestroy(e);
  for (auto &e : ctx->ev_join)
    if (e)
      cudaEventDestroy(e);
  if (ctx->stream)
    cudaStreamDestroy(ctx->stream);
  delete ctx;
  return LBFEM_OK;
}

int
lbfem_gpu_create(const lbfem_mesh_desc *m, const lbfem_params *prm, lbfem_gpu_ctx **out)
{
  if (!m || !prm || !out)
    return LBFEM_ERR_ARG;
  *out = nullptr;
  if (m->degree < 1 || m->degree > MAXP || m->n_cells_x < 1 || m->n_cells_y < 1 || !m->vertex_x || !m->vertex_y)
    return LBFEM_ERR_ARG;
  if ((m->periodic_x && m->n_cells_x < 2) || (m->periodic_y && m->n_cells_y < 2))
    return LBFEM_ERR_ARG;
  for (int i = 0; i < m->n_cells_x; ++i)
    if (!(m->vertex_x[i + 1] > m->vertex_x[i]))
      return LBFEM_ERR_ARG;
  for (int i = 0; i < m->n_cells_y; ++i)
    if (!(m->vertex_y[i + 1] > m->vertex_y[i]))
      return LBFEM_ERR_ARG;
  if (prm->scheme != LBFEM_SCHEME_BARDOW && prm->scheme != LBFEM_SCHEME_LEELIN)
    return LBFEM_ERR_ARG;
  if (prm->streaming < LBFEM_STREAMING_TG2 || prm->streaming > LBFEM_STREAMING_TG3_SPLIT)
    return LBFEM_ERR_ARG;
  // TG3 needs the consistent mass (streaming.h:51-52); Lee-Lin streams with TG2 only (schemes.h:87)
  if (prm->streaming != LBFEM_STREAMING_TG2 && (prm->mass != LBFEM_MASS_CG || prm->scheme != LBFEM_SCHEME_BARDOW))
    return LBFEM_ERR_ARG;
  if ((prm->precision != LBFEM_PRECISION_FP64 && prm->precision != LBFEM_PRECISION_MIXED) ||
      (prm->mass != LBFEM_MASS_CG && prm->mass != LBFEM_MASS_LUMPED && prm->mass != LBFEM_MASS_RICHARDSON))
    return LBFEM_ERR_UNSUPPORTED;
  if (prm->streaming != LBFEM_STREAMING_TG2 && prm->precision == LBFEM_PRECISION_MIXED)
    return LBFEM_ERR_UNSUPPORTED; // TG3 runs in FP64
  if (prm->mass == LBFEM_MASS_RICHARDSON && prm->richardson < 0)
    return LBFEM_ERR_ARG;
  if (!(prm->cg_tolerance >= 0) || prm->cg_max_iterations < 1 || !(prm->mixed_tolerance >= 0))
    return LBFEM_ERR_ARG;
  const int P = m->degree;
  // the kernels index a population array with 32-bit storage indices: fewer than 2^31 nodes
  if (((long long)P * m->n_cells_x + 1) * ((long long)P * m->n_cells_y + 1) >= (1LL << 31))
    return LBFEM_ERR_UNSUPPORTED;
  const int nfx = P * m->n_cells_x + 1, nfy = P * m->n_cells_y + 1;
  const long long N = (long long)nfx * nfy;
  if (m->dof_index == nullptr && m->n_dofs != N)
    return LBFEM_ERR_ARG;
  if (m->dof_index != nullptr && m->n_dofs != N)
    return LBFEM_ERR_ARG; // every DoF appears once: n_dofs is the node count
  if (m->n_walls < 0 || (m->n_walls > 0 && (!m->wall_dof || !m->wall_velocity)))
    return LBFEM_ERR_ARG;

  auto ctx = new lbfem_gpu_ctx();
  std::unique_ptr<lbfem_gpu_ctx, int (*)(lbfem_gpu_ctx *)> guard(ctx, lbfem_gpu_destroy);
  ctx->device = prm->device;
  ctx->prm = *prm;
  ctx->trace = std::getenv("LBFEM_TRACE") != nullptr;
  ctx->P = P;
  ctx->n_dofs = m->n_dofs;
  ctx->identity = m->dof_index == nullptr;
  ctx->grid = Grid{nfx,
                   nfy,
                   m->periodic_x ? nfx - 1 : nfx,
                   m->periodic_y ? nfy - 1 : nfy,
                   m->n_cells_x,
                   m->n_cells_y,
                   m->periodic_x ? 1 : 0,
                   m->periodic_y ? 1 : 0,
                   N,
                   0,
                   nfy};
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  for (auto &e : ctx->ev)
    CK(cudaEventCreate(&e));
  for (auto &e : ctx->ev_join)
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  ctx->basis = std::make_unique<Basis1D>(P);
  ctx->ax = make_axis(*ctx->basis, m->vertex_x, m->n_cells_x, m->periodic_x != 0);
  ctx->ay = make_axis(*ctx->basis, m->vertex_y, m->n_cells_y, m->periodic_y != 0);

  auto put = [&](double **d, const std::vector<double> &h) -> int {
    CK(cudaMalloc(d, sizeof(double) * h.size()));
    CK(cudaMemcpy(*d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
    return LBFEM_OK;
  };
  int st;
  if ((st = put(&ctx->d_rowx, ctx->ax.rows)) || (st = put(&ctx->d_rowy, ctx->ay.rows)) ||
      (st = put(&ctx->d_diagx, ctx->ax.diag)) || (st = put(&ctx->d_diagy, ctx->ay.diag)) ||
      (st = put(&ctx->d_lumpx, ctx->ax.lump)) || (st = put(&ctx->d_lumpy, ctx->ay.lump)) ||
      (st = put(&ctx->d_hx, ctx->ax.h)) || (st = put(&ctx->d_hxi, ctx->ax.hinv)) || (st = put(&ctx->d_hy, ctx->ay.h)) ||
      (st = put(&ctx->d_hyi, ctx->ay.hinv)) || (st = put(&ctx->d_ijx, ctx->ax.invdiag)) ||
      (st = put(&ctx->d_ijy, ctx->ay.invdiag)) || (st = put(&ctx->d_ilx, ctx->ax.invlump)) ||
      (st = put(&ctx->d_ily, ctx->ay.invlump)))
    return st;
  {
    // reference element matrices of every degree, into constant memory
    static double ref[MAXPD][3][MAXPD + 1][MAXPD + 1];
    static float reff[MAXPD][3][MAXPD + 1][MAXPD + 1];
    reference_matrices(ref, reff);
    CK(cudaMemcpyToSymbol(c_ref, ref, sizeof ref));
    CK(cudaMemcpyToSymbol(c_reff, reff, sizeof reff));
    static float2 ref2[MAXPD][3][MAXPD + 1][MAXPD + 1];
    for (int q = 0; q < MAXPD; ++q)
      for (int o = 0; o < 3; ++o)
        for (int a = 0; a <= MAXPD; ++a)
          for (int c = 0; c <= MAXPD; ++c)
            ref2[q][o][a][c] = make_float2(reff[q][o][a][c], reff[q][o][a][c]);
    CK(cudaMemcpyToSymbol(c_ref2, ref2, sizeof ref2));
    // the 1-D basis at the Gauss points, for the cell kernels of general quadrilaterals
    static double gs[MAXPD][MAXPD + 1][MAXPD + 1], gd[MAXPD][MAXPD + 1][MAXPD + 1];
    std::memset(gs, 0, sizeof gs);
    std::memset(gd, 0, sizeof gd);
    for (int q = 1; q <= MAXPD; ++q)
      {
        const Basis1D b(q);
        for (int k = 0; k <= q; ++k)
          for (int a = 0; a <= q; ++a)
            {
              gs[q - 1][k][a] = b.gS[k][a];
              gd[q - 1][k][a] = b.gD[k][a];
            }
      }
    CK(cudaMemcpyToSymbol(c_gS, gs, sizeof gs));
    CK(cudaMemcpyToSymbol(c_gD, gd, sizeof gd));
  }
  if (m->vertex_xy)
    {
      // general quadrilaterals: FP64, TG2, no walls (the reference's --distort is a Taylor-Green option)
      if (prm->precision != LBFEM_PRECISION_FP64 || prm->streaming != LBFEM_STREAMING_TG2 || m->n_walls > 0 ||
          !m->periodic_x || !m->periodic_y)
        return fail(ctx, LBFEM_ERR_UNSUPPORTED,
                    "general quadrilaterals: FP64, TG2, periodic in x and y (no boundary faces) only");
      ctx->distorted = true;
      const std::vector<double> qg = quad_geometry(*ctx->basis, m->vertex_xy, m->n_cells_x, m->n_cells_y);
      std::vector<double> jac, lump;
      quad_diagonals(*ctx->basis, qg, m->n_cells_x, m->n_cells_y, m->periodic_x != 0, m->periodic_y != 0, jac, lump);
      for (const double v : qg)
        if (!std::isfinite(v))
          return fail(ctx, LBFEM_ERR_ARG, "general quadrilaterals: a degenerate cell");
      std::vector<double> ijac(jac.size()), ilump(lump.size());
      for (size_t k = 0; k < jac.size(); ++k)
        {
          ijac[k] = 1. / jac[k];
          ilump[k] = 1. / lump[k];
        }
      if ((st = put(&ctx->d_qgeo, qg)) || (st = put(&ctx->d_qijac, ijac)) || (st = put(&ctx->d_qlump, lump)) ||
          (st = put(&ctx->d_qilump, ilump)))
        return st;
    }

  // numbering: structured node -> caller DoF, and its inverse for the wall list
  std::vector<long long> node_of_dof;
  if (!ctx->identity)
    {
      node_of_dof.assign(N, -1);
      std::vector<long long> dof(m->dof_index, m->dof_index + N);
      for (long long s = 0; s < N; ++s)
        {
          if (dof[s] < 0 || dof[s] >= N || node_of_dof[dof[s]] >= 0)
            return fail(ctx, LBFEM_ERR_ARG, "dof_index is not a permutation");
          node_of_dof[dof[s]] = s;
        }
      CK(cudaMalloc(&ctx->d_dof, sizeof(long long) * N));
      CK(cudaMemcpy(ctx->d_dof, dof.data(), sizeof(long long) * N, cudaMemcpyHostToDevice));
    }

  // walls: one class per distinct velocity
  if (m->n_walls > 0)
    {
      std::vector<uint8_t> cls(N, 0);
      std::map<std::pair<double, double>, int> classes;
      std::vector<double> table;
      for (int64_t k = 0; k < m->n_walls; ++k)
        {
          const int64_t d = m->wall_dof[k];
          if (d < 0 || d >= N)
            return fail(ctx, LBFEM_ERR_ARG, "wall DoF %lld out of range", (long long)d);
          const long long s = ctx->identity ? d : node_of_dof[d];
          const auto key = std::make_pair(m->wall_velocity[2 * k], m->wall_velocity[2 * k + 1]);
          auto it = classes.find(key);
          if (it == classes.end())
            {
              if (classes.size() >= 255)
                return fail(ctx, LBFEM_ERR_UNSUPPORTED, "more than 255 distinct wall velocities");
              it = classes.emplace(key, int(classes.size()) + 1).first;
              table.push_back(key.first);
              table.push_back(key.second);
            }
          cls[s] = uint8_t(it->second);
        }
      CK(cudaMalloc(&ctx->d_wall, N));
      CK(cudaMemcpy(ctx->d_wall, cls.data(), N, cudaMemcpyHostToDevice));
      if ((st = put(&ctx->d_wall_u, table)))
        return st;
    }

  // boundary nodes of the non-periodic sides (images excluded: their face integrals belong to the source)
  {
    std::vector<int4> bn;
    const Grid &g = ctx->grid;
    for (int j = 0; j < nfy; ++j)
      for (int i = 0; i < nfx; ++i)
        {
          int sides = 0;
          if (!g.py && j == 0)
            sides |= 1;
          if (!g.py && j == nfy - 1)
            sides |= 2;
          if (!g.px && i == 0)
            sides |= 4;
          if (!g.px && i == nfx - 1)
            sides |= 8;
          const bool image = (g.px && i == g.nux) || (g.py && j == g.nuy);
          if (sides && !image)
            bn.push_back(make_int4(i, j, sides, 0));
        }
    ctx->n_bnodes = int(bn.size());
    if (!bn.empty())
      {
        CK(cudaMalloc(&ctx->d_bnode, sizeof(int4) * bn.size()));
        CK(cudaMemcpy(ctx->d_bnode, bn.data(), sizeof(int4) * bn.size(), cudaMemcpyHostToDevice));
      }
  }

  // state and scratch
  auto zeros = [&](double **d, size_t n) -> int {
    CK(cudaMalloc(d, sizeof(double) * n));
    CK(cudaMemset(*d, 0, sizeof(double) * n));
    return LBFEM_OK;
  };
  if ((st = zeros(&ctx->d_f[0], Q * N)) || (st = zeros(&ctx->d_f[1], Q * N)) || (st = zeros(&ctx->d_rhs, NM * N)) ||
      (st = zeros(&ctx->d_x[0], NM * N)) || (st = zeros(&ctx->d_x[1], NM * N)) ||
      (st = zeros(&ctx->d_x[2], NM * N)) || (st = zeros(&ctx->d_r, NM * N)) || (st = zeros(&ctx->d_p[0], NM * N)) ||
      (st = zeros(&ctx->d_p[1], NM * N)) || (st = zeros(&ctx->d_v, NM * N)) || (st = zeros(&ctx->d_feq, Q * N)))
    return st;
  if (!ctx->identity && (st = zeros(&ctx->d_stage, Q * N)))
    return st;
  ctx->mixed = prm->precision == LBFEM_PRECISION_MIXED;
  if (ctx->mixed)
    {
      auto zerosf = [&](float **d, size_t n) -> int {
        CK(cudaMalloc(d, sizeof(float) * n));
        CK(cudaMemset(*d, 0, sizeof(float) * n));
        return LBFEM_OK;
      };
      if ((st = zerosf(&ctx->d_fs[0], Q * N)) || (st = zerosf(&ctx->d_fs[1], Q * N)) ||
          (st = zerosf(&ctx->d_rhs_s, NM * N)) || (st = zerosf(&ctx->d_x_s[0], NM * N)) ||
          (st = zerosf(&ctx->d_x_s[1], NM * N)) || (st = zerosf(&ctx->d_x_s[2], NM * N)) ||
          (st = zerosf(&ctx->d_r_s, NM * N)) || (st = zerosf(&ctx->d_p_s[0], NM * N)) ||
          (st = zerosf(&ctx->d_p_s[1], NM * N)))
        return st;
      if (prm->mass == LBFEM_MASS_CG)
        {
          // the window factors of the mixed-precision mass solve
          st = with_degree(P, [&](auto PP) -> int {
            using S = WinShape<decltype(PP)::value>;
            const int ntx = (nfx + S::TX - 1) / S::TX, nty = (nfy + S::TY - 1) / S::TY;
            const std::vector<float> wx = window_ldl(ctx->ax, S::TX, S::W, ntx, S::NC);
            const std::vector<float> wy = window_ldl(ctx->ay, S::TY, S::W, nty, S::NC);
            CK(cudaMalloc(&ctx->d_winx, sizeof(float) * wx.size()));
            CK(cudaMalloc(&ctx->d_winy, sizeof(float) * wy.size()));
            CK(cudaMemcpy(ctx->d_winx, wx.data(), sizeof(float) * wx.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ctx->d_winy, wy.data(), sizeof(float) * wy.size(), cudaMemcpyHostToDevice));
            return LBFEM_OK;
          });
          if (st)
            return st;
        }
    }
  const long long tiles = with_degree(P, [&](auto PP) -> int {
    constexpr int Pd = decltype(PP)::value;
    const dim3 tg = tile_grid<Pd>(ctx->grid);
    return int(tg.x * tg.y);
  });
  ctx->partial_cap = size_t(std::max<long long>(tiles, 148 * 8)) * 3 * NM;
  if ((st = zeros(&ctx->d_partials, ctx->partial_cap)) || (st = zeros(&ctx->d_sums, 64)))
    return st;
  CK(cudaMalloc(&ctx->d_cg, sizeof(CgState)));
  CK(cudaHostAlloc(&ctx->h_cg, sizeof(CgState), cudaHostAllocDefault));
  CK(cudaMalloc(&ctx->d_stats, sizeof(DevStats)));
  CK(cudaMemset(ctx->d_stats, 0, sizeof(DevStats)));
  CK(cudaHostAlloc(&ctx->h_stats, sizeof(DevStats), cudaHostAllocDefault));
  CK(cudaStreamCreateWithFlags(&ctx->cap, cudaStreamNonBlocking));
  if ((st = with_degree(P, [&](auto PP) -> int { return set_smem_attributes<decltype(PP)::value>(ctx); })))
    return st;
  *out = guard.release();
  return LBFEM_OK;
}

int
lbfem_gpu_set_time_step(lbfem_gpu_ctx *ctx, double dt, double lambda)
{
  if (!ctx)
    return LBFEM_ERR_ARG;
  if (!(dt > 0) || !(lambda > 0) || !std::isfinite(dt) || !std::isfinite(lambda))
    return fail(ctx, LBFEM_ERR_ARG, "set_time_step: dt and lambda must be positive");
  ctx->dt = dt;
  ctx->lambda = lambda;
  ctx->have_ts = true;
  // the step graphs hold the coefficients of the old time step
  cudaSetDevice(ctx->device);
  for (auto &kv : ctx->graphs)
    if (kv.second.exec)
      cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs.clear();
  ++ctx->graph_epoch;
  return LBFEM_OK;
}

int
lbfem_gpu_set_populations(lbfem_gpu_ctx *ctx, const double *f)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f)
    return fail(ctx, LBFEM_ERR_ARG, "set_populations: null buffer");
  if ((st = upload(ctx, f, ctx->d_f[ctx->cur], Q)))
    return st;
  if (ctx->mixed)
    {
      k_to_dev<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(ctx->d_f[ctx->cur], ctx->d_fs[ctx->cur],
                                                                             ctx->grid.N);
      LAUNCHED();
    }
  return LBFEM_OK;
}

int
lbfem_gpu_get_populations(lbfem_gpu_ctx *ctx, double *f)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f)
    return fail(ctx, LBFEM_ERR_ARG, "get_populations: null buffer");
  if (ctx->mixed)
    {
      k_from_dev<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(ctx->d_fs[ctx->cur],
                                                                               ctx->d_f[ctx->cur], ctx->grid.N);
      LAUNCHED();
    }
  return download(ctx, ctx->d_f[ctx->cur], f, Q);
}

int
lbfem_gpu_write_checkpoint(lbfem_gpu_ctx *ctx, const char *name, int32_t rank)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!name || rank < 0)
    return fail(ctx, LBFEM_ERR_ARG, "write_checkpoint: bad argument");
  std::vector<double> f(size_t(Q) * ctx->n_dofs);
  if ((st = lbfem_gpu_get_populations(ctx, f.data())))
    return st;
  const std::string file = checkpoint_path(name, rank);
  if ((st = write_raw(file, f)))
    return fail(ctx, st, "write_checkpoint: cannot write %s", file.c_str());
  return LBFEM_OK;
}

int
lbfem_gpu_read_checkpoint(lbfem_gpu_ctx *ctx, const char *name, int32_t rank)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!name || rank < 0)
    return fail(ctx, LBFEM_ERR_ARG, "read_checkpoint: bad argument");
  std::vector<double> f(size_t(Q) * ctx->n_dofs);
  const std::string file = checkpoint_path(name, rank);
  if ((st = read_raw(file, f)))
    return fail(ctx, st, "cannot read checkpoint %s (9 x %lld doubles expected)", file.c_str(),
                (long long)ctx->n_dofs);
  return lbfem_gpu_set_populations(ctx, f.data());
}

int
lbfem_gpu_set_initial_populations(lbfem_gpu_ctx *ctx, const double *f)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f)
    return fail(ctx, LBFEM_ERR_ARG, "set_initial_populations: null buffer");
  if (!ctx->have_ts)
    return fail(ctx, LBFEM_ERR_STATE, "set_initial_populations needs the time step");
  if ((st = upload(ctx, f, ctx->d_f[ctx->cur], Q)))
    return st;
  const long long N = ctx->grid.N;
  for (int k = 0; k < 3; ++k)
    CK(cudaMemsetAsync(ctx->d_x[k], 0, sizeof(double) * NM * N, ctx->stream));
  if (ctx->mixed)
    {
      for (int k = 0; k < 3; ++k)
        CK(cudaMemsetAsync(ctx->d_x_s[k], 0, sizeof(float) * NM * N, ctx->stream));
      k_to_dev<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(ctx->d_f[ctx->cur], ctx->d_fs[ctx->cur], N);
      LAUNCHED();
      if (ctx->prm.scheme == LBFEM_SCHEME_BARDOW)
        {
          k_bardow_transform_dev<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(
            geo_of(ctx), ctx->d_fs[ctx->cur], float(0.5 * ctx->dt / ctx->lambda));
          LAUNCHED();
        }
    }
  else if (ctx->prm.scheme == LBFEM_SCHEME_BARDOW)
    {
      k_bardow_transform<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_f[ctx->cur],
                                                                             0.5 * ctx->dt / ctx->lambda);
      LAUNCHED();
    }
  CK(cudaStreamSynchronize(ctx->stream));
  return LBFEM_OK;
}

int
lbfem_gpu_step(lbfem_gpu_ctx *ctx, int32_t n_steps)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (n_steps < 0)
    return fail(ctx, LBFEM_ERR_ARG, "step: negative count");
  if (!ctx->have_ts)
    return fail(ctx, LBFEM_ERR_STATE, "step needs the time step");
  if ((st = tune_pair(ctx)))
    return st;
  const int64_t launches0 = ctx->launches;
  int64_t its_total = 0;
  if (ctx->trace || ctx->strip || ctx->distorted)
    {
      // host-driven steps (the solver rounds print their residuals)
      for (int s = 0; s < n_steps; ++s)
        {
          int64_t its = 0;
          if ((st = step_once(ctx, &its)))
            return st;
          its_total += its;
        }
      CK(cudaStreamSynchronize(ctx->stream));
    }
  else
    {
      int64_t launched = 0;
      st = step_graphs(ctx, n_steps, &its_total, &launched);
      ctx->launches += launched;
      ctx->cg_its += its_total;
      if (st)
        return st;
    }
  ctx->last_launches = ctx->launches - launches0;
  ctx->last_its_per_solve = n_steps > 0 ? double(its_total) / (double(n_steps) * NM) : 0.0;
  return LBFEM_OK;
}

int
lbfem_gpu_step_host(lbfem_gpu_ctx *ctx, double *f, int32_t n_steps)
{
  int st;
  if ((st = lbfem_gpu_set_populations(ctx, f)))
    return st;
  if ((st = lbfem_gpu_step(ctx, n_steps)))
    return st;
  return lbfem_gpu_get_populations(ctx, f);
}

int
lbfem_gpu_synchronize(lbfem_gpu_ctx *ctx)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  CK(cudaStreamSynchronize(ctx->stream));
  return LBFEM_OK;
}

int
lbfem_gpu_advection(lbfem_gpu_ctx *ctx, const double *f, const double *feq, const double *e, double dt, double lambda,
                    int32_t kind, int32_t remove, double *rhs)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f || !e || !rhs || !(dt > 0))
    return fail(ctx, LBFEM_ERR_ARG, "advection: bad argument");
  const bool leelin = kind == LBFEM_ADVECTION_LEELIN;
  if (!leelin && kind != LBFEM_ADVECTION_TAYLOR_GALERKIN)
    return fail(ctx, LBFEM_ERR_ARG, "advection: unknown kind %d", kind);
  if (leelin && (!feq || !(lambda > 0)))
    return fail(ctx, LBFEM_ERR_ARG, "LeeLinAdvection needs the equilibria");
  double *fs = ctx->d_f[1 - ctx->cur];
  if ((st = upload(ctx, f, fs, Q)))
    return st;
  if (leelin && (st = upload(ctx, feq, ctx->d_feq, Q)))
    return st;
  AdvCoef ac;
  if (leelin)
    {
      const double b = -0.5 * dt * dt / lambda;
      ac = adv_coef(-dt - b, b, -0.5 * dt * dt, e, 0.);
    }
  else
    ac = adv_coef(-dt, 0., -0.5 * dt * dt, e, 0.);
  if ((st = launch_advection<double>(ctx, leelin ? ADV_LEELIN_FEQ : ADV_TG, fs, ctx->d_feq, nullptr, ctx->d_rhs, ac)))
    return st;
  const bool rmv = remove < 0 ? !leelin : remove != 0;
  if ((st = launch_wall_faces<double>(ctx, fs, ctx->d_rhs, e, dt, rmv)))
    return st;
  return download(ctx, ctx->d_rhs, rhs, NM);
}

int
lbfem_gpu_advection_resident(lbfem_gpu_ctx *ctx)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!ctx->have_ts)
    return fail(ctx, LBFEM_ERR_STATE, "advection_resident needs the time step");
  if (ctx->distorted)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "advection_resident: not on general quadrilaterals");
  const double dt = ctx->dt, lam = ctx->lambda;
  const double b = -0.5 * dt * dt / lam;
  const bool bardow = ctx->prm.scheme == LBFEM_SCHEME_BARDOW;
  const AdvCoef ac = bardow ? adv_coef(-dt, 0., -0.5 * dt * dt, d2q9_e(), dt / (lam + 0.5 * dt))
                            : adv_coef(-dt - b, b, -0.5 * dt * dt, d2q9_e(), 0.);
  const int mode = bardow ? ADV_TG_COLLIDE : ADV_LEELIN_FUSED;
  if ((st = tune_pair(ctx)))
    return st;
  if (ctx->mixed)
    return launch_pair(ctx, bardow ? PAIR_BARDOW : PAIR_LEELIN, ctx->d_fs[ctx->cur],
                       bardow ? ctx->d_fs[1 - ctx->cur] : nullptr, ctx->d_rhs_s, ac);
  return launch_advection<double>(ctx, mode, ctx->d_f[ctx->cur], nullptr, bardow ? ctx->d_f[1 - ctx->cur] : nullptr,
                                  ctx->d_rhs, ac);
}

int
lbfem_gpu_solve_round_resident(lbfem_gpu_ctx *ctx)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!ctx->mixed || ctx->prm.mass != LBFEM_MASS_CG)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "solve_round_resident: mixed precision with consistent mass only");
  const Geo geo = geo_of(ctx);
  const Grid &g = ctx->grid;
  return with_degree(ctx->P, [&](auto PP) -> int {
    constexpr int P = decltype(PP)::value;
    using S = WinShape<P>;
    const dim3 grid(tiles_along(g.nfx, g.nux, g.px, S::TX), tiles_along(g.nfy, g.nuy, g.py, S::TY), NM);
    k_window_correct<P><<<grid, S::THREADS, window_smem<P>(), ctx->stream>>>(
      geo, ctx->d_winx, ctx->d_winy, ctx->d_r_s, ctx->d_x_s[ctx->x_cur], ctx->d_rhs_s, ctx->d_p_s[1], ctx->d_p_s[0],
      ctx->d_cg, 1, ctx->d_partials);
    LAUNCHED();
    return LBFEM_OK;
  });
}

int
lbfem_gpu_mass_solve(lbfem_gpu_ctx *ctx, double *x, const double *r, const double *e, double tg3)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!x || !r)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve: null buffer");
  if (tg3 != 0. && !e)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve: the TG3 matrix needs the direction e");
  if (tg3 != 0. && ctx->prm.mass == LBFEM_MASS_RICHARDSON)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "mass_solve: the TG3 matrix with iterated lumping is not implemented");
  StreamCoef sc{};
  if (tg3 != 0.)
    {
      sc.kxx[0] = tg3 * e[0] * e[0];
      sc.kyy[0] = tg3 * e[1] * e[1];
      sc.kxy[0] = tg3 * e[0] * e[1];
    }
  double *xn = ctx->d_x[ctx->x_new];
  if ((st = upload(ctx, r, ctx->d_rhs, 1)) || (st = upload(ctx, x, xn, 1)))
    return st;
  const int solve_st = mass_solve_dev(ctx, ctx->d_rhs, xn, tg3 != 0., sc, nullptr);
  if (solve_st != LBFEM_OK && solve_st != LBFEM_ERR_NO_CONVERGENCE && solve_st != LBFEM_ERR_NONFINITE)
    return solve_st;
  if ((st = download(ctx, xn, x, 1)))
    return st;
  return solve_st;
}

int
lbfem_gpu_stream_function(lbfem_gpu_ctx *ctx, const double *velocity, double *psi)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!velocity || !psi)
    return fail(ctx, LBFEM_ERR_ARG, "stream_function: null buffer");
  if (ctx->strip || ctx->distorted)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "stream_function: not on a strip or on general quadrilaterals");
  const long long N = ctx->grid.N;
  double *vel = ctx->d_x[ctx->x_new], *b = ctx->d_rhs, *x = ctx->d_rhs + N; // scratch between steps
  if ((st = upload(ctx, velocity, vel, 2)))
    return st;
  st = with_degree(ctx->P, [&](auto PP) -> int {
    constexpr int P = decltype(PP)::value;
    k_psi_rhs<P><<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(geo_of(ctx), vel, vel + N, b);
    LAUNCHED();
    return LBFEM_OK;
  });
  if (st)
    return st;
  CK(cudaMemsetAsync(x, 0, sizeof(double) * N, ctx->stream));
  // SolverCG with the Laplace diagonal from zero to 1e-12 |b|, at most 10000 iterations (io.h:90-93)
  CgCall c;
  c.b = b;
  c.x_new = x;
  c.nsys = 1;
  c.opk = OPK_LAPLACE;
  c.tol = 1e-12;
  c.max_its = 10000;
  int64_t its = 0;
  const int solve_st = cg_run(ctx, ctx_scratch(ctx), c, &its);
  if (solve_st != LBFEM_OK)
    return solve_st;
  return download(ctx, x, psi, 1);
}

int
lbfem_gpu_mass_vmult(lbfem_gpu_ctx *ctx, double *y, const double *x)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!x || !y)
    return fail(ctx, LBFEM_ERR_ARG, "mass_vmult: null buffer");
  if ((st = upload(ctx, x, ctx->d_r, 1)))
    return st;
  if (ctx->distorted)
    {
      if ((st = quad_vmult(ctx, ctx->d_r, ctx->d_v, 1)))
        return st;
      return download(ctx, ctx->d_v, y, 1);
    }
  const Geo geo = geo_of(ctx);
  st = with_degree(ctx->P, [&](auto PP) -> int {
    constexpr int P = decltype(PP)::value;
    k_mass_vmult<P><<<tile_grid<P>(ctx->grid), THREADS, mass_smem<P>(), ctx->stream>>>(geo, ctx->d_r, ctx->d_v, 1);
    LAUNCHED();
    return LBFEM_OK;
  });
  if (st)
    return st;
  return download(ctx, ctx->d_v, y, 1);
}

int
lbfem_gpu_cg_iterations(const lbfem_gpu_ctx *ctx, int64_t *its)
{
  if (!ctx || !its)
    return LBFEM_ERR_ARG;
  *its = ctx->cg_its;
  return LBFEM_OK;
}

int
lbfem_gpu_collide_bgk(lbfem_gpu_ctx *ctx, double *g, double omega)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!g)
    return fail(ctx, LBFEM_ERR_ARG, "collide_bgk: null buffer");
  double *d = ctx->d_f[1 - ctx->cur];
  if ((st = upload(ctx, g, d, Q)))
    return st;
  k_collide<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), d, omega);
  LAUNCHED();
  return download(ctx, d, g, Q);
}

int
lbfem_gpu_compute_equilibrium(lbfem_gpu_ctx *ctx, const double *f, double *feq)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f || !feq)
    return fail(ctx, LBFEM_ERR_ARG, "compute_equilibrium: null buffer");
  double *d = ctx->d_f[1 - ctx->cur];
  if ((st = upload(ctx, f, d, Q)))
    return st;
  k_equilibrium<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), d, ctx->d_feq);
  LAUNCHED();
  return download(ctx, ctx->d_feq, feq, Q);
}

int
lbfem_gpu_predictor_corrector(lbfem_gpu_ctx *ctx, double *f, const double *feq, const double *incr, double theta)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f || !feq || !incr)
    return fail(ctx, LBFEM_ERR_ARG, "predictor_corrector: null buffer");
  double *d = ctx->d_f[1 - ctx->cur];
  if ((st = upload(ctx, f, d, Q)) || (st = upload(ctx, feq, ctx->d_feq, Q)) || (st = upload(ctx, incr, ctx->d_r, NM)))
    return st;
  k_predictor_corrector<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), nullptr, d,
                                                                                      ctx->d_feq, ctx->d_r, theta);
  LAUNCHED();
  return download(ctx, d, f, Q);
}

// ---------------------------------------------------------------------------
// Device-pointer forms of the operators, ordered on the caller's stream.
int
lbfem_gpu_advection_dev(lbfem_gpu_ctx *ctx, const double *f, const double *feq, const double *e, double dt,
                        double lambda, int32_t kind, int32_t remove, double *rhs, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f || !e || !rhs || !(dt > 0))
    return fail(ctx, LBFEM_ERR_ARG, "advection_dev: bad argument");
  const bool leelin = kind == LBFEM_ADVECTION_LEELIN;
  if (!leelin && kind != LBFEM_ADVECTION_TAYLOR_GALERKIN)
    return fail(ctx, LBFEM_ERR_ARG, "advection_dev: unknown kind %d", kind);
  if (leelin && (!feq || !(lambda > 0)))
    return fail(ctx, LBFEM_ERR_ARG, "LeeLinAdvection needs the equilibria");
  if ((st = join_caller(ctx, stream)))
    return st;
  const double *fs = nullptr, *feqs = nullptr;
  if ((st = gather_dev(ctx, f, ctx->d_f[1 - ctx->cur], Q, &fs)))
    return st;
  if (leelin && (st = gather_dev(ctx, feq, ctx->d_feq, Q, &feqs)))
    return st;
  AdvCoef ac;
  if (leelin)
    {
      const double b = -0.5 * dt * dt / lambda;
      ac = adv_coef(-dt - b, b, -0.5 * dt * dt, e, 0.);
    }
  else
    ac = adv_coef(-dt, 0., -0.5 * dt * dt, e, 0.);
  double *out = out_dev(ctx, rhs, ctx->d_rhs);
  if ((st = launch_advection<double>(ctx, leelin ? ADV_LEELIN_FEQ : ADV_TG, fs, feqs, nullptr, out, ac)))
    return st;
  const bool rmv = remove < 0 ? !leelin : remove != 0;
  if ((st = launch_wall_faces<double>(ctx, fs, out, e, dt, rmv)) || (st = scatter_dev(ctx, out, rhs, NM)))
    return st;
  return release_caller(ctx, stream);
}

int
lbfem_gpu_mass_solve_dev(lbfem_gpu_ctx *ctx, double *x, const double *r, const double *e, double tg3, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!x || !r)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve_dev: null buffer");
  if (tg3 != 0. && !e)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve_dev: the TG3 matrix needs the direction e");
  if (tg3 != 0. && ctx->prm.mass == LBFEM_MASS_RICHARDSON)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "mass_solve_dev: the TG3 matrix with iterated lumping is not implemented");
  StreamCoef sc{};
  if (tg3 != 0.)
    {
      sc.kxx[0] = tg3 * e[0] * e[0];
      sc.kyy[0] = tg3 * e[1] * e[1];
      sc.kxy[0] = tg3 * e[0] * e[1];
    }
  if ((st = join_caller(ctx, stream)))
    return st;
  const double *b = nullptr;
  if ((st = gather_dev(ctx, r, ctx->d_rhs, 1, &b)))
    return st;
  double *xn = ctx->d_x[ctx->x_new];
  if (ctx->identity)
    xn = x;
  else
    {
      k_gather<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(x, ctx->d_dof, xn, ctx->grid.N,
                                                                             ctx->n_dofs, 1);
      LAUNCHED();
    }
  const int solve_st = mass_solve_dev(ctx, b, xn, tg3 != 0., sc, nullptr);
  if (solve_st != LBFEM_OK && solve_st != LBFEM_ERR_NO_CONVERGENCE && solve_st != LBFEM_ERR_NONFINITE)
    return solve_st;
  if ((st = scatter_dev(ctx, xn, x, 1)) || (st = release_caller(ctx, stream)))
    return st;
  return solve_st;
}

int
lbfem_gpu_collide_bgk_dev(lbfem_gpu_ctx *ctx, double *g, double omega, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!g)
    return fail(ctx, LBFEM_ERR_ARG, "collide_bgk_dev: null buffer");
  if ((st = join_caller(ctx, stream)))
    return st;
  const double *gs = nullptr;
  if ((st = gather_dev(ctx, g, ctx->d_f[1 - ctx->cur], Q, &gs)))
    return st;
  double *d = const_cast<double *>(gs); // g itself, or the context's gathered copy
  k_collide<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), d, omega);
  LAUNCHED();
  if ((st = scatter_dev(ctx, d, g, Q)))
    return st;
  return release_caller(ctx, stream);
}

int
lbfem_gpu_compute_equilibrium_dev(lbfem_gpu_ctx *ctx, const double *f, double *feq, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f || !feq)
    return fail(ctx, LBFEM_ERR_ARG, "compute_equilibrium_dev: null buffer");
  if ((st = join_caller(ctx, stream)))
    return st;
  const double *fs = nullptr;
  if ((st = gather_dev(ctx, f, ctx->d_f[1 - ctx->cur], Q, &fs)))
    return st;
  double *out = out_dev(ctx, feq, ctx->d_feq);
  k_equilibrium<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), fs, out);
  LAUNCHED();
  if ((st = scatter_dev(ctx, out, feq, Q)))
    return st;
  return release_caller(ctx, stream);
}

int
lbfem_gpu_predictor_corrector_dev(lbfem_gpu_ctx *ctx, double *f, const double *feq, const double *incr,
                                  double theta, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f || !feq || !incr)
    return fail(ctx, LBFEM_ERR_ARG, "predictor_corrector_dev: null buffer");
  if ((st = join_caller(ctx, stream)))
    return st;
  const double *fs = nullptr, *feqs = nullptr, *xs = nullptr;
  if ((st = gather_dev(ctx, f, ctx->d_f[1 - ctx->cur], Q, &fs)) || (st = gather_dev(ctx, feq, ctx->d_feq, Q, &feqs)) ||
      (st = gather_dev(ctx, incr, ctx->d_r, NM, &xs)))
    return st;
  double *d = const_cast<double *>(fs); // f itself, or the context's gathered copy
  k_predictor_corrector<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), nullptr, d, feqs,
                                                                                      xs, theta);
  LAUNCHED();
  if ((st = scatter_dev(ctx, d, f, Q)))
    return st;
  return release_caller(ctx, stream);
}

int
lbfem_gpu_set_populations_dev(lbfem_gpu_ctx *ctx, const double *f, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f)
    return fail(ctx, LBFEM_ERR_ARG, "set_populations_dev: null buffer");
  if ((st = join_caller(ctx, stream)))
    return st;
  double *dst = ctx->d_f[ctx->cur];
  if (ctx->identity)
    CK(cudaMemcpyAsync(dst, f, sizeof(double) * Q * ctx->grid.N, cudaMemcpyDeviceToDevice, ctx->stream));
  else
    {
      k_gather<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(f, ctx->d_dof, dst, ctx->grid.N,
                                                                             ctx->n_dofs, Q);
      LAUNCHED();
    }
  if (ctx->mixed)
    {
      k_to_dev<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(dst, ctx->d_fs[ctx->cur], ctx->grid.N);
      LAUNCHED();
    }
  return release_caller(ctx, stream);
}

int
lbfem_gpu_get_populations_dev(lbfem_gpu_ctx *ctx, double *f, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!f)
    return fail(ctx, LBFEM_ERR_ARG, "get_populations_dev: null buffer");
  if ((st = join_caller(ctx, stream)))
    return st;
  double *src = ctx->d_f[ctx->cur];
  if (ctx->mixed)
    {
      k_from_dev<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(ctx->d_fs[ctx->cur], src, ctx->grid.N);
      LAUNCHED();
    }
  if (ctx->identity)
    CK(cudaMemcpyAsync(f, src, sizeof(double) * Q * ctx->grid.N, cudaMemcpyDeviceToDevice, ctx->stream));
  else if ((st = scatter_dev(ctx, src, f, Q)))
    return st;
  return release_caller(ctx, stream);
}

int
lbfem_gpu_step_stream(lbfem_gpu_ctx *ctx, int32_t n_steps, void *stream)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if ((st = join_caller(ctx, stream)))
    return st;
  if ((st = lbfem_gpu_step(ctx, n_steps)))
    return st;
  return release_caller(ctx, stream);
}

int
lbfem_gpu_tuning(const lbfem_gpu_ctx *ctx, int32_t *shape, float *ms)
{
  if (!ctx || !shape || !ms)
    return LBFEM_ERR_ARG;
  *shape = ctx->pair_tuned ? ctx->pair_shape : -1;
  for (int k = 0; k < N_SHAPES; ++k)
    ms[k] = ctx->tune_ms[k];
  return LBFEM_OK;
}

int
lbfem_gpu_strip_buffer_bytes(const lbfem_gpu_ctx *ctx, int64_t *bytes)
{
  if (!ctx || !bytes)
    return LBFEM_ERR_ARG;
  // the widest exchange: the 9 FP64 population blocks, `degree` rows
  *bytes = int64_t(Q) * ctx->P * ctx->grid.nfx * int64_t(sizeof(double));
  return LBFEM_OK;
}

int
lbfem_gpu_set_strip(lbfem_gpu_ctx *ctx, const lbfem_strip_desc *sd)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!sd || !sd->comm || !sd->sums)
    return fail(ctx, LBFEM_ERR_ARG, "set_strip: the collective and the sums buffer are required");
  const Grid &g = ctx->grid;
  if (g.py || ctx->distorted)
    return fail(ctx, LBFEM_ERR_ARG, "set_strip: the local mesh of a strip is an axis-parallel mesh, not periodic in y");
  if ((sd->ghost_below != 0 && sd->ghost_below != ctx->P) || (sd->ghost_above != 0 && sd->ghost_above != 1))
    return fail(ctx, LBFEM_ERR_ARG, "set_strip: ghost rows are `degree` below and 1 above, or none");
  if ((sd->ghost_below && (!sd->send_below || !sd->recv_below)) ||
      (sd->ghost_above && (!sd->send_above || !sd->recv_above)))
    return fail(ctx, LBFEM_ERR_ARG, "set_strip: missing exchange buffer");
  const int oy0 = sd->ghost_below, oy1 = g.nfy - sd->ghost_above;
  // the owned rows must hold whole cells' worth of rows to send `degree` rows up
  if (oy1 - oy0 < ctx->P + 1)
    return fail(ctx, LBFEM_ERR_ARG, "set_strip: the strip owns %d node rows, fewer than degree + 1", oy1 - oy0);
  if (!(sd->cell_below >= 0) || !(sd->cell_above >= 0))
    return fail(ctx, LBFEM_ERR_ARG, "set_strip: negative cell width");
  // The end rows of the local mesh lack the neighbours' cell in their mass
  // diagonals; add its share (M_hat is symmetric under a -> p - a, so a vertex
  // row's diagonal and row sum scale with the summed width of its two cells).
  Axis &ay = ctx->ay;
  const int last = ay.n_nodes - 1;
  const double fb = (ay.h.front() + sd->cell_below) / ay.h.front(), fa = (ay.h.back() + sd->cell_above) / ay.h.back();
  ay.diag[0] *= fb;
  ay.lump[0] *= fb;
  ay.diag[last] *= fa;
  ay.lump[last] *= fa;
  for (int k : {0, last})
    {
      ay.invdiag[k] = 1. / ay.diag[k];
      ay.invlump[k] = 1. / ay.lump[k];
    }
  const size_t nb = sizeof(double) * ay.n_nodes;
  CK(cudaMemcpy(ctx->d_diagy, ay.diag.data(), nb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_lumpy, ay.lump.data(), nb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_ijy, ay.invdiag.data(), nb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_ily, ay.invlump.data(), nb, cudaMemcpyHostToDevice));
  ctx->sd = *sd;
  ctx->strip = true;
  ctx->grid.oy0 = oy0;
  ctx->grid.oy1 = oy1;
  // recorded step graphs are not used in strip mode; drop them
  for (auto &kv : ctx->graphs)
    if (kv.second.exec)
      cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs.clear();
  ++ctx->graph_epoch;
  return LBFEM_OK;
}

int
lbfem_gpu_node_weight(lbfem_gpu_ctx *ctx, double *w)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!w)
    return fail(ctx, LBFEM_ERR_ARG, "node_weight: null buffer");
  k_diagonal<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_v, 0);
  LAUNCHED();
  return download(ctx, ctx->d_v, w, 1);
}

int
lbfem_gpu_jacobi_diagonal(lbfem_gpu_ctx *ctx, double *d)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!d)
    return fail(ctx, LBFEM_ERR_ARG, "jacobi_diagonal: null buffer");
  k_diagonal<<<n_pointwise_blocks(ctx->grid.N), THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_v, 1);
  LAUNCHED();
  return download(ctx, ctx->d_v, d, 1);
}

int
lbfem_gpu_moments(lbfem_gpu_ctx *ctx, double *rho, double *ux, double *uy)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  const long long N = ctx->grid.N;
  double *d = ctx->d_r; // 3 of its 8 blocks
  if (ctx->mixed)
    k_moments_dev<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_fs[ctx->cur], d, d + N,
                                                                      d + 2 * N);
  else
    k_moments<<<n_pointwise_blocks(N), THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_f[ctx->cur], d, d + N,
                                                                  d + 2 * N);
  LAUNCHED();
  double *outs[3] = {rho, ux, uy};
  for (int k = 0; k < 3; ++k)
    if (outs[k] && (st = download(ctx, d + k * N, outs[k], 1)))
      return st;
  return LBFEM_OK;
}

int
lbfem_gpu_conservation(lbfem_gpu_ctx *ctx, double out[5])
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!out)
    return fail(ctx, LBFEM_ERR_ARG, "conservation: null buffer");
  const int nb = n_pointwise_blocks(ctx->grid.N);
  if (ctx->mixed)
    k_conservation_dev<<<nb, THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_fs[ctx->cur], ctx->d_partials);
  else
    k_conservation<<<nb, THREADS, 0, ctx->stream>>>(geo_of(ctx), ctx->d_f[ctx->cur], ctx->d_partials);
  LAUNCHED();
  if ((st = reduce(ctx, nb, 5)))
    return st;
  CK(cudaMemcpyAsync(out, ctx->d_sums, 5 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return LBFEM_OK;
}

int
lbfem_gpu_event_record(lbfem_gpu_ctx *ctx, int32_t slot)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (slot < 0 || slot >= 16)
    return fail(ctx, LBFEM_ERR_ARG, "event slot out of range");
  CK(cudaEventRecord(ctx->ev[slot], ctx->stream));
  return LBFEM_OK;
}

int
lbfem_gpu_event_elapsed(lbfem_gpu_ctx *ctx, int32_t a, int32_t b, float *ms)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (a < 0 || a >= 16 || b < 0 || b >= 16 || !ms)
    return fail(ctx, LBFEM_ERR_ARG, "event slot out of range");
  CK(cudaEventSynchronize(ctx->ev[b]));
  CK(cudaEventElapsedTime(ms, ctx->ev[a], ctx->ev[b]));
  return LBFEM_OK;
}

int
lbfem_gpu_last_step_stats(const lbfem_gpu_ctx *ctx, double *its, int64_t *launches)
{
  if (!ctx)
    return LBFEM_ERR_ARG;
  if (its)
    *its = ctx->last_its_per_solve;
  if (launches)
    *launches = ctx->last_launches;
  return LBFEM_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Batched stepping: one graph launch per step of all instances, whose steps are
// independent branches of the graph (no edges between them).
struct lbfem_gpu_batch
{
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::vector<lbfem_gpu_ctx *> ctxs;
  struct Entry
  {
    cudaGraphExec_t exec = nullptr;
    std::vector<int64_t> epochs;      // the time-step epochs of the instances it was recorded with
    std::vector<int64_t> fixed, body; // per instance: kernels outside the loops, per loop body
    void *d_group = nullptr;          // the grouped launches' instance table and tile lists
    int64_t group_fixed = 0, group_body = 0; // the grouped launches outside the loop, per loop body
  };
  std::map<std::vector<int>, Entry> graphs; // by the buffer states of the instances
  // the instances stepped by grouped launches (mixed precision, consistent mass,
  // TG2, Cartesian, whole mesh), largest first; the others are graph branches
  std::vector<size_t> grouped;
  cudaStream_t gstream = nullptr, gcap = nullptr; // the grouped launches' capture streams
  static constexpr int MAX_CLASSES = 8;           // (degree, scheme) pairs
  cudaStream_t cs[MAX_CLASSES] = {}, bs[MAX_CLASSES] = {}; // class branches outside and inside the loop
  cudaEvent_t gfork = nullptr, gjoin = nullptr;
  unsigned long long *d_loops = nullptr;          // loop bodies the grouped solve ran
  unsigned long long *h_loops = nullptr;          // pinned copy
  // LBFEM_TRACE: the grouped step is launched kernel by kernel with its loop on
  // the host (the graph holds the other instances' branches only)
  bool trace = false;
  int *d_flag = nullptr;          // the host-driven loop's condition
  void *d_trace_plan = nullptr;   // the host-driven step's argument lists
  size_t trace_plan_bytes = 0;
  DevStats *h_stats = nullptr;              // pinned, one per instance
  cudaEvent_t t0 = nullptr, t1 = nullptr;   // device time of the last batch_step's launches
  float last_ms = 0.f;
  int64_t last_launches = 0; // kernels launched by the last batch_step (all instances)
  std::string err;
};

namespace
{
  int
  batch_fail(lbfem_gpu_batch *b, int status, const char *fmt, ...)
  {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    b->err = buf;
    return status;
  }

#define BCK(call)                                                                                         \
  do                                                                                                      \
    {                                                                                                     \
      const cudaError_t e_ = (call);                                                                      \
      if (e_ != cudaSuccess)                                                                              \
        return batch_fail(b, LBFEM_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                                     \
  while (0)

  // ------------------------------------------------------- grouped launches
  // The instances whose step the grouped kernels of batch_group.cuh run.
  bool
  groupable(const lbfem_gpu_ctx *c)
  {
    return c->mixed && c->prm.mass == LBFEM_MASS_CG && n_sweeps(c) == 1 &&
           c->prm.streaming == LBFEM_STREAMING_TG2 && !c->distorted && !c->strip;
  }

  // A class of grouped instances: one degree and one scheme, a contiguous range
  // [i0, i1) of the instance table, and the (instance, tile) or (instance, node
  // chunk) references of its launches (instance indices into the whole table).
  struct GroupClass
  {
    int P = 1, mode = PAIR_LEELIN;
    int i0 = 0, i1 = 0;
    size_t pair_off = 0, wall_off = 0, start_off = 0, win_off = 0, chunk_off = 0;
    int pair_n = 0;  // streaming tiles (Tile<P>)
    int wall_n = 0;  // (instance, first boundary node) per 16 wall nodes
    int start_n = 0; // start tiles (StartShape<P>)
    int win_n = 0;   // window tiles (WinShape<P>)
    int chunk_n = 0; // node chunks of GROUP_CHUNK nodes
  };

  // The argument lists of the grouped launches for the instances' current
  // buffer states, laid out for one device allocation: the instance table
  // (sorted by class, largest instances first within a class), then the
  // reference lists of every class.
  struct GroupPlan
  {
    std::vector<unsigned char> bytes;
    int n = 0;      // instances
    size_t tab = 0; // offset of the instance table
    std::vector<GroupClass> cls;
  };

  template <typename T>
  size_t
  plan_put(std::vector<unsigned char> &bytes, const std::vector<T> &v)
  {
    const size_t off = (bytes.size() + 15) & ~size_t(15);
    bytes.resize(off + sizeof(T) * v.size());
    if (!v.empty())
      std::memcpy(bytes.data() + off, v.data(), sizeof(T) * v.size());
    return off;
  }

  // The arguments of the instances b->grouped, as record_step would pass them
  // to the single-instance kernels of a mixed-precision step (step_front,
  // mixed_graph, step_back).
  GroupPlan
  group_plan(const lbfem_gpu_batch *b)
  {
    GroupPlan gp;
    std::vector<size_t> idx = b->grouped; // largest first
    auto class_of = [&](size_t k) {
      const lbfem_gpu_ctx *c = b->ctxs[k];
      return 2 * c->P + (c->prm.scheme == LBFEM_SCHEME_BARDOW ? 1 : 0);
    };
    // the classes with the most nodes first: their branches are recorded, and start, first
    std::map<int, long long> class_nodes;
    for (size_t k : idx)
      class_nodes[class_of(k)] += b->ctxs[k]->grid.N;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
      const int cx = class_of(x), cy = class_of(y);
      return cx != cy && (class_nodes[cx] != class_nodes[cy] ? class_nodes[cx] > class_nodes[cy] : cx < cy);
    });
    gp.n = int(idx.size());
    std::vector<GroupInst> tab(idx.size());
    struct Lists
    {
      std::vector<TileRef> pair, start, win;
      std::vector<int2> wall, chunks;
    };
    std::vector<Lists> lists;
    for (size_t j = 0; j < idx.size(); ++j)
      {
        const lbfem_gpu_ctx *c = b->ctxs[idx[j]];
        const FrontCoef fr = front_coef(c, 0);
        const int k = int(j), mode = fr.bardow ? PAIR_BARDOW : PAIR_LEELIN;
        GroupInst &I = tab[j];
        I.geo = geo_of(c);
        I.ds = c->d_stats;
        I.ac = fr.ac;
        I.fc = face_coef(c, fr.e, c->dt, fr.remove);
        I.bnode = c->d_bnode;
        I.n_bnodes = int(c->n_bnodes);
        I.bardow = fr.bardow ? 1 : 0;
        I.f = c->d_fs[c->cur];
        I.g = fr.bardow ? c->d_fs[1 - c->cur] : nullptr;
        I.rhs = c->d_rhs_s;
        I.xc = c->d_x_s[c->x_cur];
        I.xp = c->d_x_s[c->x_prev];
        I.xn = c->d_x_s[c->x_new];
        I.r0 = c->d_r_s;
        I.r1 = c->d_p_s[0];
        I.winx = c->d_winx;
        I.winy = c->d_winy;
        I.cg = c->d_cg;
        I.partials = c->d_partials;
        I.sums = c->d_sums;
        I.tol = mixed_tolerance(c->prm);
        I.max_rounds = c->prm.cg_max_iterations;
        I.theta = c->dt / c->lambda;
        I.N = c->grid.N;
        with_degree(c->P, [&](auto PP) -> int {
          constexpr int P = decltype(PP)::value;
          const dim3 tg = tile_grid<P>(c->grid), sg = start_grid<P>(c->grid, 1);
          using S = WinShape<P>;
          I.nb_pair_x = int(tg.x);
          I.nb_pair_y = int(tg.y);
          I.nb_start_x = int(sg.x);
          I.nb_start_y = int(sg.y);
          I.nb_win_x = tiles_along(c->grid.nfx, c->grid.nux, c->grid.px, S::TX);
          I.nb_win_y = tiles_along(c->grid.nfy, c->grid.nuy, c->grid.py, S::TY);
          return 0;
        });
        if (gp.cls.empty() || gp.cls.back().P != c->P || gp.cls.back().mode != mode)
          {
            GroupClass gc;
            gc.P = c->P;
            gc.mode = mode;
            gc.i0 = k;
            gp.cls.push_back(gc);
            lists.emplace_back();
          }
        gp.cls.back().i1 = k + 1;
        Lists &L = lists.back();
        for (int by = 0; by < I.nb_pair_y; ++by)
          for (int bx = 0; bx < I.nb_pair_x; ++bx)
            L.pair.push_back({k, bx, by});
        for (int by = 0; by < I.nb_start_y; ++by)
          for (int bx = 0; bx < I.nb_start_x; ++bx)
            L.start.push_back({k, bx, by});
        for (int by = 0; by < I.nb_win_y; ++by)
          for (int bx = 0; bx < I.nb_win_x; ++bx)
            L.win.push_back({k, bx, by});
        for (int t = 0; t < I.n_bnodes; t += 16) // 8 threads per node, 128 per CTA
          L.wall.push_back(make_int2(k, t));
        for (long long ch = 0; ch * GROUP_CHUNK < I.N; ++ch)
          L.chunks.push_back(make_int2(k, int(ch)));
      }
    gp.tab = plan_put(gp.bytes, tab);
    for (size_t q = 0; q < gp.cls.size(); ++q)
      {
        GroupClass &gc = gp.cls[q];
        const Lists &L = lists[q];
        gc.pair_off = plan_put(gp.bytes, L.pair);
        gc.pair_n = int(L.pair.size());
        gc.wall_off = plan_put(gp.bytes, L.wall);
        gc.wall_n = int(L.wall.size());
        gc.start_off = plan_put(gp.bytes, L.start);
        gc.start_n = int(L.start.size());
        gc.win_off = plan_put(gp.bytes, L.win);
        gc.win_n = int(L.win.size());
        gc.chunk_off = plan_put(gp.bytes, L.chunks);
        gc.chunk_n = int(L.chunks.size());
      }
    return gp;
  }

  // The grouped step of the instances b->grouped: the kernel sequence of
  // record_step for a mixed-precision step, each kernel over the tiles of all
  // instances of one class (degree and scheme). The classes run as concurrent
  // branches (streams b->cs, and b->bs inside the loop body) that join only for
  // the loop condition, so the launches of small classes overlap. The solve's
  // loop runs while any instance is active; a round of an instance that has
  // stopped carries its solution and residual over and counts nothing (the
  // single-instance loop's bodies after convergence), so each instance's
  // results are those of its own step. Recorded on b->gstream, which is being
  // captured, with the loop as a conditional WHILE node; or (host_driven)
  // launched from b->stream with the loop on the host, which reads the loop
  // condition after every body (the path of LBFEM_TRACE, whose kernels
  // profilers can see one by one). *fixed, *body: the kernels outside the loop
  // and per loop body.
  int
  record_group(lbfem_gpu_batch *b, const GroupPlan &gp, const void *d_plan, bool host_driven, int64_t *fixed,
               int64_t *body)
  {
    const unsigned char *base = static_cast<const unsigned char *>(d_plan);
    const GroupInst *tab = reinterpret_cast<const GroupInst *>(base + gp.tab);
    auto tiles = [&](size_t off) { return reinterpret_cast<const TileRef *>(base + off); };
    auto refs = [&](size_t off) { return reinterpret_cast<const int2 *>(base + off); };
    cudaStream_t s = host_driven ? b->stream : b->gstream;
    const int nc = int(gp.cls.size());
    int64_t n_fixed = 0, n_body = 0;
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    cudaGraphConditionalHandle h = 0;
    if (!host_driven)
      {
        BCK(cudaStreamGetCaptureInfo_v3(s, &cs, nullptr, &graph, nullptr, nullptr, nullptr));
        BCK(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault)); // 0 at every launch
      }
    const int use_h = host_driven ? 0 : 1;
    int *flag = host_driven ? b->d_flag : nullptr;

    // the class streams q[0..nc) wait for the work queued on `from`; `to` waits for theirs
    auto fork = [&](cudaStream_t from, cudaStream_t *q) -> cudaError_t {
      cudaError_t e = cudaEventRecord(b->gfork, from);
      for (int c = 0; c < nc && e == cudaSuccess; ++c)
        e = cudaStreamWaitEvent(q[c], b->gfork, 0);
      return e;
    };
    auto join = [&](cudaStream_t *q, cudaStream_t to) -> cudaError_t {
      cudaError_t e = cudaSuccess;
      for (int c = 0; c < nc && e == cudaSuccess; ++c)
        if ((e = cudaEventRecord(b->gjoin, q[c])) == cudaSuccess)
          e = cudaStreamWaitEvent(to, b->gjoin, 0);
      return e;
    };
    // one round of the mixed solve for class gc on stream q: the window
    // correction (phase: the buffer roles of kg_window), the sums, the bookkeeping
    auto round = [&](const GroupClass &gc, cudaStream_t q, int phase, int all) -> int64_t {
      with_degree(gc.P, [&](auto PP) -> int {
        constexpr int P = decltype(PP)::value;
        kg_window<P><<<dim3(gc.win_n, NM), WinShape<P>::THREADS, window_smem<P>(), q>>>(tab, tiles(gc.win_off),
                                                                                       phase, all);
        return 0;
      });
      kg_reduce<<<(gc.i1 - gc.i0) * 2 * NM, 256, 0, q>>>(tab + gc.i0, 2 * NM);
      kg_mixed_round<<<gc.i1 - gc.i0, 32, 0, q>>>(tab + gc.i0);
      return 3;
    };

    // per class: the front (step_front), the solve's start, round 0 and the zero
    // rule (mixed_graph); then the loop condition of all classes
    kg_clear<<<gp.n, 64, 0, s>>>(tab);
    ++n_fixed;
    BCK(cudaGetLastError());
    BCK(fork(s, b->cs));
    for (int c = 0; c < nc; ++c)
      {
        const GroupClass &gc = gp.cls[c];
        cudaStream_t q = b->cs[c];
        with_degree(gc.P, [&](auto PP) -> int {
          constexpr int P = decltype(PP)::value;
          if (gc.mode == PAIR_BARDOW)
            kg_stream_pair<P, PAIR_BARDOW><<<gc.pair_n, THREADS, pair_smem<P, PAIR_BARDOW>(), q>>>(
              tab, tiles(gc.pair_off));
          else
            kg_stream_pair<P, PAIR_LEELIN><<<gc.pair_n, THREADS, pair_smem<P, PAIR_LEELIN>(), q>>>(
              tab, tiles(gc.pair_off));
          if (gc.wall_n)
            kg_wall_faces<P><<<gc.wall_n, 128, 0, q>>>(tab, refs(gc.wall_off));
          kg_mixed_start<P><<<dim3(gc.start_n, NM), StartShape<P>::THREADS, 0, q>>>(tab, tiles(gc.start_off));
          return 0;
        });
        n_fixed += gc.wall_n ? 3 : 2;
        n_fixed += round(gc, q, 0, 1);
        kg_zero<<<dim3(gc.chunk_n, NM), THREADS, 0, q>>>(tab, refs(gc.chunk_off));
        ++n_fixed;
      }
    BCK(cudaGetLastError());
    BCK(join(b->cs, s));
    kg_control<<<1, 256, 0, s>>>(tab, gp.n, h, use_h, nullptr, flag);
    ++n_fixed;
    BCK(cudaGetLastError());

    // the loop: one body is two rounds of every class (x_prev -> x_new -> x_prev)
    if (host_driven)
      {
        int any = 0;
        for (;;)
          {
            BCK(cudaMemcpyAsync(&any, b->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
            BCK(cudaStreamSynchronize(s));
            if (!any)
              break;
            BCK(fork(s, b->cs));
            n_body = 1;
            for (int c = 0; c < nc; ++c)
              n_body += round(gp.cls[c], b->cs[c], 1, 0) + round(gp.cls[c], b->cs[c], 0, 0);
            BCK(cudaGetLastError());
            BCK(join(b->cs, s));
            kg_control<<<1, 256, 0, s>>>(tab, gp.n, h, 0, b->d_loops, flag);
            BCK(cudaGetLastError());
          }
      }
    else
      {
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        BCK(cudaStreamGetCaptureInfo_v3(s, &cs, nullptr, &graph, &deps, nullptr, &nd));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        BCK(cudaGraphAddNode(&node, graph, deps, nd, &np));
        BCK(cudaStreamBeginCaptureToGraph(b->gcap, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
        cudaError_t le = fork(b->gcap, b->bs);
        n_body = 1;
        for (int c = 0; c < nc && le == cudaSuccess; ++c)
          n_body += round(gp.cls[c], b->bs[c], 1, 0) + round(gp.cls[c], b->bs[c], 0, 0);
        if (le == cudaSuccess)
          le = cudaGetLastError();
        if (le == cudaSuccess)
          le = join(b->bs, b->gcap);
        if (le == cudaSuccess)
          {
            kg_control<<<1, 256, 0, b->gcap>>>(tab, gp.n, h, 1, b->d_loops, nullptr);
            le = cudaGetLastError();
          }
        cudaGraph_t bg = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(b->gcap, &bg);
        BCK(le);
        BCK(ee);
        BCK(cudaStreamUpdateCaptureDependencies_v2(s, &node, nullptr, 1, cudaStreamSetCaptureDependencies));
      }

    // per class: the nodal update (step_back)
    BCK(fork(s, b->cs));
    for (int c = 0; c < nc; ++c)
      {
        const GroupClass &gc = gp.cls[c];
        if (gc.mode == PAIR_BARDOW)
          kg_nodal<PAIR_BARDOW><<<gc.chunk_n, THREADS, 0, b->cs[c]>>>(tab, refs(gc.chunk_off));
        else
          kg_nodal<PAIR_LEELIN><<<gc.chunk_n, THREADS, 0, b->cs[c]>>>(tab, refs(gc.chunk_off));
        ++n_fixed;
      }
    BCK(cudaGetLastError());
    BCK(join(b->cs, s));
    *fixed = n_fixed;
    *body = n_body;
    return LBFEM_OK;
  }

  bool
  create_class_streams(lbfem_gpu_batch *b)
  {
    for (int c = 0; c < lbfem_gpu_batch::MAX_CLASSES; ++c)
      if (cudaStreamCreateWithFlags(&b->cs[c], cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&b->bs[c], cudaStreamNonBlocking) != cudaSuccess)
        return false;
    return true;
  }

  // The batch graph of the instances' current buffer states: one capture in
  // which every instance's step is recorded on its own stream, forked from and
  // joined to the batch stream, so the instances are independent branches
  // (recorded on first use, again when an instance's time step changed).
  int
  batch_graph(lbfem_gpu_batch *b, lbfem_gpu_batch::Entry **out)
  {
    std::vector<int> key;
    std::vector<int64_t> epochs;
    for (auto *c : b->ctxs)
      {
        key.push_back(graph_key(c));
        epochs.push_back(c->graph_epoch);
      }
    auto &e = b->graphs[key];
    if (e.exec && e.epochs == epochs)
      {
        *out = &e;
        return LBFEM_OK;
      }
    if (e.exec)
      {
        cudaGraphExecDestroy(e.exec);
        e.exec = nullptr;
      }
    e.fixed.assign(b->ctxs.size(), 0);
    e.body.assign(b->ctxs.size(), 0);
    GroupPlan gp;
    const bool group = !b->grouped.empty() && !b->trace;
    if (group)
      {
        // the argument lists of the grouped launches, uploaded before the capture
        if (e.d_group)
          {
            BCK(cudaStreamSynchronize(b->stream)); // a launch of the previous graph may still read them
            BCK(cudaFree(e.d_group));
            e.d_group = nullptr;
          }
        gp = group_plan(b);
        BCK(cudaMalloc(&e.d_group, gp.bytes.size()));
        BCK(cudaMemcpy(e.d_group, gp.bytes.data(), gp.bytes.size(), cudaMemcpyHostToDevice));
      }
    std::vector<char> in_group(b->ctxs.size(), 0);
    for (size_t k : b->grouped)
      in_group[k] = 1;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = LBFEM_OK;
    cudaError_t ce = cudaEventRecord(b->fork, b->stream);
    if (ce == cudaSuccess && group && (ce = cudaStreamWaitEvent(b->gstream, b->fork, 0)) == cudaSuccess)
      {
        st = record_group(b, gp, e.d_group, false, &e.group_fixed, &e.group_body);
        if (!st && (ce = cudaEventRecord(b->join, b->gstream)) == cudaSuccess)
          ce = cudaStreamWaitEvent(b->stream, b->join, 0);
      }
    // the largest instances are recorded first, so that their branches start first;
    // results and failure indices stay those of the instance order
    std::vector<size_t> order(b->ctxs.size());
    for (size_t k = 0; k < order.size(); ++k)
      order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t x, size_t y) { return b->ctxs[x]->grid.N > b->ctxs[y]->grid.N; });
    for (size_t o = 0; o < order.size() && !st && ce == cudaSuccess; ++o)
      {
        const size_t k = order[o];
        if (in_group[k])
          continue;
        lbfem_gpu_ctx *c = b->ctxs[k];
        ce = cudaStreamWaitEvent(c->stream, b->fork, 0);
        if (ce != cudaSuccess)
          break;
        if ((st = record_step(c, &e.fixed[k], &e.body[k])))
          {
            batch_fail(b, st, "instance %zu: %s", k, c->err.c_str());
            break;
          }
        if ((ce = cudaEventRecord(b->join, c->stream)) == cudaSuccess)
          ce = cudaStreamWaitEvent(b->stream, b->join, 0);
      }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
    if (st || ce != cudaSuccess || ee != cudaSuccess)
      {
        if (graph)
          cudaGraphDestroy(graph);
        if (st)
          return st;
        return batch_fail(b, LBFEM_ERR_CUDA, "batch capture: %s",
                          cudaGetErrorString(ce != cudaSuccess ? ce : ee));
      }
    const cudaError_t ei = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess)
      {
        e.exec = nullptr;
        return batch_fail(b, LBFEM_ERR_CUDA, "batch graph instantiation: %s", cudaGetErrorString(ei));
      }
    e.epochs = epochs;
    *out = &e;
    return LBFEM_OK;
  }
} // namespace

extern "C" {

int
lbfem_gpu_batch_create(lbfem_gpu_ctx *const *ctxs, int32_t n, lbfem_gpu_batch **out)
{
  if (!ctxs || n < 1 || !out)
    return LBFEM_ERR_ARG;
  *out = nullptr;
  for (int k = 0; k < n; ++k)
    {
      if (!ctxs[k])
        return LBFEM_ERR_ARG;
      if (ctxs[k]->device != ctxs[0]->device || ctxs[k]->distorted || ctxs[k]->strip)
        return LBFEM_ERR_UNSUPPORTED;
      for (int j = 0; j < k; ++j)
        if (ctxs[j] == ctxs[k])
          return LBFEM_ERR_ARG;
    }
  auto b = std::make_unique<lbfem_gpu_batch>();
  b->device = ctxs[0]->device;
  b->ctxs.assign(ctxs, ctxs + n);
  b->trace = std::getenv("LBFEM_TRACE") != nullptr;
  // LBFEM_BATCH_GROUP=0 steps every instance as a graph branch of its own
  const char *genv = std::getenv("LBFEM_BATCH_GROUP");
  if (!(genv && genv[0] == '0'))
    {
      for (int k = 0; k < n; ++k)
        if (groupable(ctxs[k]))
          b->grouped.push_back(size_t(k));
      // largest first: their tiles lead the grouped launches' lists
      std::stable_sort(b->grouped.begin(), b->grouped.end(),
                       [&](size_t x, size_t y) { return ctxs[x]->grid.N > ctxs[y]->grid.N; });
    }
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->gstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->gcap, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->gfork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->gjoin, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess ||
      cudaHostAlloc(&b->h_stats, sizeof(DevStats) * n, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc(&b->h_loops, sizeof(unsigned long long), cudaHostAllocDefault) != cudaSuccess ||
      cudaMalloc(&b->d_loops, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(b->d_loops, 0, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->d_flag, sizeof(int)) != cudaSuccess || !create_class_streams(b.get()))
    {
      cudaGetLastError();
      lbfem_gpu_batch_destroy(b.release());
      return LBFEM_ERR_CUDA;
    }
  *out = b.release();
  return LBFEM_OK;
}

const char *
lbfem_gpu_batch_last_error(const lbfem_gpu_batch *b)
{
  return b ? b->err.c_str() : "";
}

int
lbfem_gpu_batch_last_ms(const lbfem_gpu_batch *b, float *ms)
{
  if (!b || !ms)
    return LBFEM_ERR_ARG;
  *ms = b->last_ms;
  return LBFEM_OK;
}

int
lbfem_gpu_batch_last_launches(const lbfem_gpu_batch *b, int64_t *launches)
{
  if (!b || !launches)
    return LBFEM_ERR_ARG;
  *launches = b->last_launches;
  return LBFEM_OK;
}

int
lbfem_gpu_batch_destroy(lbfem_gpu_batch *b)
{
  if (!b)
    return LBFEM_OK;
  cudaSetDevice(b->device);
  if (b->stream)
    cudaStreamSynchronize(b->stream);
  for (auto &kv : b->graphs)
    {
      if (kv.second.exec)
        cudaGraphExecDestroy(kv.second.exec);
      if (kv.second.d_group)
        cudaFree(kv.second.d_group);
    }
  if (b->h_stats)
    cudaFreeHost(b->h_stats);
  if (b->h_loops)
    cudaFreeHost(b->h_loops);
  if (b->d_loops)
    cudaFree(b->d_loops);
  if (b->d_flag)
    cudaFree(b->d_flag);
  if (b->d_trace_plan)
    cudaFree(b->d_trace_plan);
  if (b->gstream)
    cudaStreamDestroy(b->gstream);
  if (b->gcap)
    cudaStreamDestroy(b->gcap);
  for (int c = 0; c < lbfem_gpu_batch::MAX_CLASSES; ++c)
    {
      if (b->cs[c])
        cudaStreamDestroy(b->cs[c]);
      if (b->bs[c])
        cudaStreamDestroy(b->bs[c]);
    }
  if (b->gfork)
    cudaEventDestroy(b->gfork);
  if (b->gjoin)
    cudaEventDestroy(b->gjoin);
  if (b->fork)
    cudaEventDestroy(b->fork);
  if (b->join)
    cudaEventDestroy(b->join);
  if (b->t0)
    cudaEventDestroy(b->t0);
  if (b->t1)
    cudaEventDestroy(b->t1);
  if (b->stream)
    cudaStreamDestroy(b->stream);
  delete b;
  return LBFEM_OK;
}

int
lbfem_gpu_batch_step(lbfem_gpu_batch *b, int32_t n_steps)
{
  if (!b)
    return LBFEM_ERR_ARG;
  if (n_steps < 0)
    return batch_fail(b, LBFEM_ERR_ARG, "batch_step: negative count");
  BCK(cudaSetDevice(b->device));
  const size_t n = b->ctxs.size();
  for (size_t k = 0; k < n; ++k)
    {
      lbfem_gpu_ctx *c = b->ctxs[k];
      if (!c->have_ts)
        return batch_fail(b, LBFEM_ERR_STATE, "instance %zu: step needs the time step", k);
      // (the grouped launches use the default streaming tile)
      if (std::find(b->grouped.begin(), b->grouped.end(), k) == b->grouped.end() && tune_pair(c) != LBFEM_OK)
        return batch_fail(b, LBFEM_ERR_CUDA, "instance %zu: %s", k, c->err.c_str());
      // the instance's own queued work first, then its counters
      BCK(cudaStreamSynchronize(c->stream));
      BCK(cudaMemcpy(&b->h_stats[k], c->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost));
    }
  std::vector<RunStart> r0;
  for (size_t k = 0; k < n; ++k)
    r0.push_back(run_start(b->ctxs[k], b->h_stats[k]));
  BCK(cudaMemcpyAsync(b->h_loops, b->d_loops, sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  const unsigned long long loops0 = *b->h_loops;
  int64_t group_fixed = 0, group_body = 0; // kernels of the grouped launches
  BCK(cudaEventRecord(b->t0, b->stream));
  for (int s = 0; s < n_steps; ++s)
    {
      int st;
      if (!b->trace || b->grouped.size() < n)
        {
          lbfem_gpu_batch::Entry *e;
          if ((st = batch_graph(b, &e)))
            return st;
          BCK(cudaGraphLaunch(e->exec, b->stream));
          group_fixed += e->group_fixed;
          group_body = e->group_body;
          for (size_t k = 0; k < n; ++k)
            {
              r0[k].fixed += e->fixed[k];
              r0[k].body = e->body[k];
            }
        }
      if (b->trace && !b->grouped.empty())
        {
          const GroupPlan gp = group_plan(b);
          if (gp.bytes.size() > b->trace_plan_bytes)
            {
              BCK(cudaStreamSynchronize(b->stream));
              if (b->d_trace_plan)
                BCK(cudaFree(b->d_trace_plan));
              b->d_trace_plan = nullptr;
              BCK(cudaMalloc(&b->d_trace_plan, gp.bytes.size()));
              b->trace_plan_bytes = gp.bytes.size();
            }
          // the previous step's launches read the table until the stream gets here
          BCK(cudaMemcpyAsync(b->d_trace_plan, gp.bytes.data(), gp.bytes.size(), cudaMemcpyHostToDevice, b->stream));
          BCK(cudaStreamSynchronize(b->stream));
          int64_t f = 0, bd = 0;
          if ((st = record_group(b, gp, b->d_trace_plan, true, &f, &bd)))
            return st;
          group_fixed += f;
          if (bd)
            group_body = bd;
        }
      for (size_t k = 0; k < n; ++k)
        rotate_after_step(b->ctxs[k]);
    }
  BCK(cudaEventRecord(b->t1, b->stream));
  for (size_t k = 0; k < n; ++k)
    BCK(cudaMemcpyAsync(&b->h_stats[k], b->ctxs[k]->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemcpyAsync(b->h_loops, b->d_loops, sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  BCK(cudaEventElapsedTime(&b->last_ms, b->t0, b->t1));
  b->last_launches = group_fixed + int64_t(*b->h_loops - loops0) * group_body;
  int first = LBFEM_OK;
  for (size_t k = 0; k < n; ++k)
    {
      lbfem_gpu_ctx *c = b->ctxs[k];
      int64_t its = 0, launched = 0;
      const int st = finish_run(c, r0[k], b->h_stats[k], &its, &launched);
      c->cg_its += its;
      c->launches += launched;
      c->last_launches = launched; // 0 for a grouped instance (its kernels are the grouped launches)
      b->last_launches += launched;
      c->last_its_per_solve = n_steps > 0 ? double(its) / (double(n_steps) * NM) : 0.0;
      if (st && first == LBFEM_OK)
        {
          first = st;
          batch_fail(b, st, "instance %zu: %s", k, c->err.c_str());
        }
    }
  return first;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Mass solve without allocation.
//
// For callers that may not allocate device memory when they call in (a host
// framework that owns every device allocation, or a code whose memory pool is
// sized once at start-up): the CG work buffers of this entry point live in
// one file-scope device array of fixed size, which every GPU that loads the
// library holds until the process exits. Its device address is looked up once
// per device, on the first call with that device current (std::call_once, so
// two host threads making their first call together do not race on the
// cache). Calls share the array, so calls that overlap on the GPU (from
// several threads or streams) race; the solver state is cleared at the start
// of every call. The solve is host-driven: one small state read per CG
// iteration, so the call is synchronous and cannot be captured into a graph.
namespace
{
  constexpr long long NOALLOC_MAX_NODES = 1LL << 17; // 131072 nodes
  constexpr long long NOALLOC_MAX_TILES = 4096;
  constexpr long long NOALLOC_STATE_DOUBLES = (sizeof(CgState) + sizeof(double) - 1) / sizeof(double);
  constexpr long long NOALLOC_DOUBLES =
    3 * NOALLOC_MAX_NODES + 3 * NM * NOALLOC_MAX_TILES + 64 + NOALLOC_STATE_DOUBLES;

  static __device__ __align__(256) double noalloc_scratch[NOALLOC_DOUBLES];

  constexpr int NOALLOC_MAX_DEVICES = 64;
  double *noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
  cudaError_t noalloc_err[NOALLOC_MAX_DEVICES] = {};
  std::once_flag noalloc_once[NOALLOC_MAX_DEVICES];

  // The array's device address on the current device (looked up once per device).
  cudaError_t
  noalloc_base(int device, double **out)
  {
    std::call_once(noalloc_once[device], [device] {
      void *p = nullptr;
      noalloc_err[device] = cudaGetSymbolAddress(&p, noalloc_scratch);
      noalloc_ptr[device] = static_cast<double *>(p);
    });
    *out = noalloc_ptr[device];
    return noalloc_err[device];
  }
} // namespace

extern "C" int
lbfem_gpu_mass_solve_noalloc(lbfem_gpu_ctx *ctx, double *x, const double *r)
{
  int st;
  if ((st = check_ctx(ctx)))
    return st;
  if (!x || !r)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve_noalloc: null buffer");
  const long long N = ctx->grid.N;
  if (N > NOALLOC_MAX_NODES)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve_noalloc: %lld nodes exceed the fixed scratch of %lld nodes", N,
                NOALLOC_MAX_NODES);
  const long long tiles = with_degree(ctx->P, [&](auto PP) -> int {
    constexpr int P = decltype(PP)::value;
    const dim3 tg = tile_grid<P>(ctx->grid);
    return int(tg.x * tg.y);
  });
  if (tiles > NOALLOC_MAX_TILES)
    return fail(ctx, LBFEM_ERR_ARG, "mass_solve_noalloc: %lld tiles exceed the fixed scratch of %lld tiles", tiles,
                NOALLOC_MAX_TILES);
  if (!ctx->identity)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "mass_solve_noalloc: needs the structured DoF numbering");
  if (ctx->prm.mass != LBFEM_MASS_CG)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "mass_solve_noalloc: the consistent mass (CG) only");
  if (ctx->strip || ctx->distorted)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "mass_solve_noalloc: not on a strip or on general quadrilaterals");
  if (ctx->device < 0 || ctx->device >= NOALLOC_MAX_DEVICES)
    return fail(ctx, LBFEM_ERR_UNSUPPORTED, "mass_solve_noalloc: device ordinal %d too large", ctx->device);
  double *base = nullptr; // check_ctx made ctx's device current
  CK(noalloc_base(ctx->device, &base));
  CgScratch<double> w{};
  w.r = base;
  w.p[0] = base + NOALLOC_MAX_NODES;
  w.p[1] = base + 2 * NOALLOC_MAX_NODES;
  w.partials = base + 3 * NOALLOC_MAX_NODES;
  w.sums = w.partials + 3 * NM * NOALLOC_MAX_TILES;
  w.state = reinterpret_cast<CgState *>(w.sums + 64);
  CgCall c;
  c.b = r;
  c.x_new = x;
  c.nsys = 1;
  const int solve_st = cg_run(ctx, w, c, nullptr);
  if (solve_st != LBFEM_OK)
    return solve_st;
  CK(cudaStreamSynchronize(ctx->stream));
  return LBFEM_OK;
}

// ---------------------------------------------------------------------------
// The x-pass contraction on CUDA cores and on tensor cores (a measurement for
// the choice between the two; no step uses it).
namespace
{
  template <int P, typename R, bool TC>
  int
  run_study(int rows, int cells, int reps, float *ms, double *checksum)
  {
    using namespace lbfem_gpu::study;
    const long long n = (long long)rows * (P * cells + 1);
    R *buf = nullptr;
    if (cudaMalloc(&buf, sizeof(R) * 4 * n) != cudaSuccess)
      return LBFEM_ERR_CUDA;
    R *u = buf, *h = buf + n, *y1 = buf + 2 * n, *y2 = buf + 3 * n;
    Mats<R> m{};
    const Basis1D b(P);
    for (int a = 0; a <= P; ++a)
      for (int c = 0; c <= P; ++c)
        {
          m.M[a][c] = R(b.Mh[a][c]);
          m.C[a][c] = R(b.Ch[a][c]);
          m.K[a][c] = R(b.Kh[a][c]);
        }
    int st = LBFEM_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const dim3 grid((cells + cells_of<R>() - 1) / cells_of<R>(), (rows + ROWS - 1) / ROWS);
    auto kernel = k_xpass_study<P, R, TC>;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaMemset(y1, 0, sizeof(R) * 2 * n) != cudaSuccess ||
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem<P, R>())) != cudaSuccess)
      st = LBFEM_ERR_CUDA;
    if (!st)
      {
        k_study_fill<R><<<148 * 8, 256>>>(u, h, n);
        kernel<<<grid, NT, smem<P, R>()>>>(u, h, y1, y2, rows, cells, m); // warm-up
        cudaEventRecord(e0);
        for (int k = 0; k < reps; ++k)
          kernel<<<grid, NT, smem<P, R>()>>>(u, h, y1, y2, rows, cells, m);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess)
          st = LBFEM_ERR_CUDA;
      }
    if (!st)
      {
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        *ms = t / float(reps > 0 ? reps : 1);
        std::vector<R> hy(2 * n);
        if (cudaMemcpy(hy.data(), y1, sizeof(R) * 2 * n, cudaMemcpyDeviceToHost) != cudaSuccess)
          st = LBFEM_ERR_CUDA;
        double sum = 0;
        for (long long i = 0; i < 2 * n; ++i)
          sum += std::fabs(double(hy[i]));
        *checksum = sum;
      }
    if (e0)
      cudaEventDestroy(e0);
    if (e1)
      cudaEventDestroy(e1);
    cudaFree(buf);
    return st;
  }
} // namespace

extern "C" int
lbfem_gpu_contraction_study(int32_t device, int32_t degree, int32_t fp64, int32_t tensor, int32_t rows, int32_t cells,
                            int32_t reps, float *ms, double *checksum)
{
  if (degree < 2 || degree > 3 || rows < 1 || cells < 1 || reps < 1 || !ms || !checksum)
    return LBFEM_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess)
    return LBFEM_ERR_CUDA;
  auto pick = [&](auto PP) -> int {
    constexpr int P = decltype(PP)::value;
    if (fp64)
      return tensor ? run_study<P, double, true>(rows, cells, reps, ms, checksum)
                    : run_study<P, double, false>(rows, cells, reps, ms, checksum);
    return tensor ? run_study<P, float, true>(rows, cells, reps, ms, checksum)
                  : run_study<P, float, false>(rows, cells, reps, ms, checksum);
  };
  return degree == 2 ? pick(std::integral_constant<int, 2>()) : pick(std::integral_constant<int, 3>());
}
