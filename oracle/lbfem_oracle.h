/*
 * lbfem_oracle.h -- CPU FP64 oracle of the lbm-fem hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA path is compared
 * against; it is never linked into, loaded by or called from the product
 * library. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * use it.
 *
 * It restates, without deal.II, the matrix-free algorithm of the reference
 * (ivan-pi/lbm-fem, include/lbfem/*.h): cell loops with sum-factorised
 * gradients at the (p+1)^2 Gauss points, the point operations of
 * advection.h, integration and scatter-add (distribute_local_to_global),
 * wall-face integrals, the MassOperator vmult, its lumped and Jacobi diagonals,
 * deal.II SolverCG with the Jacobi preconditioner, the nodal maps of
 * collision.h and the two schemes of schemes.h. Structured full-grid
 * numbering only (lbfem_mesh_desc::dof_index must be NULL).
 *
 * The functions mirror include/lbfem_gpu.h one for one.
 */
#ifndef LBFEM_ORACLE_H
#define LBFEM_ORACLE_H

#include "lbfem_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbfem_oracle lbfem_oracle;

int lbfem_oracle_create(const lbfem_mesh_desc *mesh, const lbfem_params *params, lbfem_oracle **h);
int lbfem_oracle_destroy(lbfem_oracle *h);
int lbfem_oracle_set_threads(int32_t n_threads);
int lbfem_oracle_set_time_step(lbfem_oracle *h, double dt, double lambda);
int lbfem_oracle_set_initial_populations(lbfem_oracle *h, const double *f);
int lbfem_oracle_set_populations(lbfem_oracle *h, const double *f);
int lbfem_oracle_get_populations(lbfem_oracle *h, double *f);
int lbfem_oracle_write_checkpoint(lbfem_oracle *h, const char *name, int32_t rank);
int lbfem_oracle_read_checkpoint(lbfem_oracle *h, const char *name, int32_t rank);
int lbfem_oracle_step(lbfem_oracle *h, int32_t n_steps);
int lbfem_oracle_advection(lbfem_oracle *h, const double *f, const double *feq, const double *e, double dt,
                           double lambda, int32_t kind, int32_t remove_wall_mass_flux, double *rhs);
int lbfem_oracle_mass_solve(lbfem_oracle *h, double *x, const double *r, const double *e, double tg3_coefficient);
int lbfem_oracle_mass_vmult(lbfem_oracle *h, double *y, const double *x);
int lbfem_oracle_cg_iterations(const lbfem_oracle *h, int64_t *iterations);
int lbfem_oracle_collide_bgk(lbfem_oracle *h, double *g, double omega);
int lbfem_oracle_compute_equilibrium(lbfem_oracle *h, const double *f, double *feq);
int lbfem_oracle_predictor_corrector(lbfem_oracle *h, double *f, const double *feq, const double *incr,
                                     double theta);
int lbfem_oracle_node_weight(lbfem_oracle *h, double *w);
int lbfem_oracle_jacobi_diagonal(lbfem_oracle *h, double *d);
int lbfem_oracle_conservation(lbfem_oracle *h, double out[5]);
/* compute_stream_function (io.h:31-95): velocity = (u, v), 2 blocks of n_dofs; psi: n_dofs. */
int lbfem_oracle_stream_function(lbfem_oracle *h, const double *velocity, double *psi);
/* One y-strip of a decomposed mesh (lbfem_gpu_set_strip); buffers in host memory. */
int lbfem_oracle_strip_buffer_bytes(const lbfem_oracle *h, int64_t *bytes);
int lbfem_oracle_set_strip(lbfem_oracle *h, const lbfem_strip_desc *strip);
/* 1-D reference data of FE_Q(p): Gauss-Lobatto support points (p+1), Gauss points and weights (p+1). */
int lbfem_oracle_basis_1d(int32_t p, double *support, double *gauss_points, double *gauss_weights);

#ifdef __cplusplus
}
#endif

#endif
