// The batched mixed-precision step as grouped launches: one kernel per phase
// over the tiles of many instances, instead of one graph branch of about ten
// small kernels per instance. A table of per-instance arguments (one entry per
// instance, for one state of the buffer rotation) and a list of (instance,
// tile) references drive each launch; the tile bodies are those of the
// single-instance kernels, with the instance's own tile grid, so every
// instance computes bitwise what its own step computes. The instances fall in
// classes of one degree and one scheme; each class's launches form one branch
// of the step's graph (record_group in lbfem_gpu.cu).
#pragma once

#include "stream_pair.cuh"

namespace lbfem_gpu
{
  struct GroupInst
  {
    Geo geo;
    DevStats *ds;
    AdvCoef ac;
    FaceCoef fc;
    const int4 *bnode;
    int n_bnodes, bardow;
    float *f;                  // the deviations the streaming kernel reads (d_fs[cur])
    float *g;                  // Bardow: the collided deviations it writes (d_fs[1 - cur]); else null
    float *rhs;                // the streaming right-hand side (8 systems)
    const float *xc;           // x_cur: the extrapolation's newer term
    float *xp, *xn;            // x_prev (the rounds end here) and x_new
    float *r0, *r1;            // the residual buffers of the rounds
    const float *winx, *winy;  // window factors
    CgState *cg;
    double *partials, *sums;
    double tol;
    int max_rounds;
    int nb_pair_x, nb_pair_y;   // tile grid of the streaming kernel (Tile<P>)
    int nb_start_x, nb_start_y; // tile grid of the start (StartShape<P>)
    int nb_win_x, nb_win_y;     // tile grid of the window rounds (WinShape<P>)
    double theta;
    long long N;
  };

  struct TileRef
  {
    int inst, bx, by;
  };

  constexpr int GROUP_CHUNK = 1024; // nodes per CTA of the grouped node-wise kernels

  // The instance's arguments, copied into shared memory by the CTA (the tile
  // bodies read them many times; shared memory cannot alias their outputs).
  __device__ __forceinline__ const GroupInst &
  load_inst(const GroupInst *__restrict__ tab, int k)
  {
    __shared__ __align__(16) GroupInst si;
    static_assert(sizeof(GroupInst) % 4 == 0, "copied as words");
    const int *src = reinterpret_cast<const int *>(tab + k);
    int *dst = reinterpret_cast<int *>(&si);
    for (int t = threadIdx.x; t < int(sizeof(GroupInst) / 4); t += blockDim.x)
      dst[t] = src[t];
    __syncthreads();
    return si;
  }

  template <int P, int MODE>
  __global__ void __launch_bounds__(THREADS, 2)
    kg_stream_pair(const GroupInst *__restrict__ tab, const TileRef *__restrict__ tiles)
  {
    const TileRef t = tiles[blockIdx.x];
    const GroupInst &I = load_inst(tab, t.inst);
    stream_pair_tile<P, MODE, TileShape<P>>(I.geo, I.ds, I.f, I.g, I.rhs, I.ac, t.bx, t.by);
  }

  // refs: (instance, first boundary node) per CTA of 128 threads, 8 per node
  template <int P>
  __global__ void
  kg_wall_faces(const GroupInst *__restrict__ tab, const int2 *__restrict__ refs)
  {
    const int2 rf = refs[blockIdx.x];
    const GroupInst &I = load_inst(tab, rf.x);
    const int t = rf.y + (threadIdx.x >> 3);
    wall_face_pop<P, float>(I.geo, I.bardow ? I.g : I.f, I.rhs, I.bnode, I.fc, t, threadIdx.x & 7, t < I.n_bnodes);
  }

  // blockIdx.y: system
  template <int P>
  __global__ void __launch_bounds__(StartShape<P>::THREADS)
    kg_mixed_start(const GroupInst *__restrict__ tab, const TileRef *__restrict__ tiles)
  {
    const TileRef t = tiles[blockIdx.x];
    const GroupInst &I = load_inst(tab, t.inst);
    mixed_start_tile<P>(I.geo, I.rhs, I.xc, I.xp, I.xn, I.r0, t.bx, t.by, blockIdx.y);
  }

  // phase 0: r0, x_new -> x_prev, r1; phase 1: r1, x_prev -> x_new, r0 (the rounds of mixed_graph)
  template <int P>
  __global__ void __launch_bounds__(WinShape<P>::THREADS, WinShape<P>::MIN_CTAS)
    kg_window(const GroupInst *__restrict__ tab, const TileRef *__restrict__ tiles, int phase, int all)
  {
    const TileRef t = tiles[blockIdx.x];
    const GroupInst &I = load_inst(tab, t.inst);
    const float *r_in = phase ? I.r1 : I.r0, *x_in = phase ? I.xp : I.xn;
    float *x_out = phase ? I.xn : I.xp, *r_out = phase ? I.r0 : I.r1;
    window_correct_tile<P>(I.geo, I.winx, I.winy, r_in, x_in, I.rhs, x_out, r_out, I.cg, all, I.partials, t.bx,
                           t.by, blockIdx.y, I.nb_win_x, I.nb_win_y);
  }

  // CTA (instance k, quantity q), k = blockIdx.x / nq: the window rounds' sums
  __global__ void
  kg_reduce(const GroupInst *__restrict__ tab, int nq)
  {
    const GroupInst &I = tab[blockIdx.x / nq];
    reduce_partials_q(I.partials, I.nb_win_x * I.nb_win_y, I.sums, blockIdx.x % nq);
  }

  __global__ void
  kg_mixed_round(const GroupInst *__restrict__ tab)
  {
    const GroupInst &I = tab[blockIdx.x];
    mixed_round_body(I.cg, I.sums, I.ds, NM, I.tol, I.max_rounds);
  }

  // the solver states cleared before a step's solve (cudaMemsetAsync per instance otherwise)
  __global__ void
  kg_clear(const GroupInst *__restrict__ tab)
  {
    int *st = reinterpret_cast<int *>(tab[blockIdx.x].cg);
    for (int t = threadIdx.x; t < int(sizeof(CgState) / 4); t += blockDim.x)
      st[t] = 0;
  }

  // the loop condition of all instances: another loop body while any is active,
  // set as the graph's condition h (use_h: launched in a graph) or stored in
  // *flag (host-driven); *loops (if given) counts the bodies run
  __global__ void
  kg_control(const GroupInst *__restrict__ tab, int n, cudaGraphConditionalHandle h, int use_h,
             unsigned long long *loops, int *flag)
  {
    __shared__ int any;
    if (threadIdx.x == 0)
      any = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      if (tab[k].cg->n_active > 0)
        any = 1;
    __syncthreads();
    if (threadIdx.x == 0)
      {
        if (use_h)
          cudaGraphSetConditional(h, any ? 1u : 0u);
        if (flag)
          *flag = any;
        if (loops)
          ++*loops;
      }
  }

  // refs: (instance, chunk); blockIdx.y: system. x_prev <- 0 for the systems whose
  // right-hand side is exactly zero (after round 0, as zero_flagged).
  __global__ void
  kg_zero(const GroupInst *__restrict__ tab, const int2 *__restrict__ refs)
  {
    const int2 rf = refs[blockIdx.x];
    const GroupInst &I = tab[rf.x];
    const int s = blockIdx.y;
    if (!I.cg->zero[s])
      return;
    const long long i0 = (long long)rf.y * GROUP_CHUNK;
    float *x = I.xp + s * I.N;
    for (long long i = i0 + threadIdx.x; i < i0 + GROUP_CHUNK && i < I.N; i += blockDim.x)
      x[i] = 0.f;
  }

  // The nodal update that completes the step (the predictor-corrector, or
  // Bardow's streaming g* + x), skipped after a failure; chunk 0 counts the step.
  template <int MODE>
  __global__ void __launch_bounds__(THREADS, 4)
    kg_nodal(const GroupInst *__restrict__ tab, const int2 *__restrict__ refs)
  {
    const int2 rf = refs[blockIdx.x];
    const GroupInst &I = load_inst(tab, rf.x);
    DevStats *ds = I.ds;
    if (ds->sticky)
      return;
    if (rf.y == 0 && threadIdx.x == 0)
      atomicAdd(&ds->steps_done, 1ULL);
    const long long i0 = (long long)rf.y * GROUP_CHUNK, N = I.N;
    const float th = float(I.theta), inv = float(1. / (1. + I.theta));
    for (long long i = i0 + threadIdx.x; i < i0 + GROUP_CHUNK && i < N; i += blockDim.x)
      {
        if constexpr (MODE == PAIR_LEELIN)
          pc_dev_node(I.geo, I.f, I.xp, th, inv, i);
        else
#pragma unroll
          for (int a = 1; a < Q; ++a)
            I.g[a * N + i] += I.xp[(a - 1) * N + i];
      }
  }
} // namespace lbfem_gpu
