/*
 * mtlgpu fixtures -- deterministic host-side generators of the synthetic test
 * and benchmark systems (CSR int32 / float64).  Part of libmtlgpu.
 *
 * All generators are two-phase: call with NULL arrays to get the sizes, then
 * with arrays of those sizes.  Random streams use SplitMix64:
 *   state += 0x9E3779B97F4A7C15; z = state;
 *   z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9; z = (z ^ (z >> 27)) * 0x94D049BB133111EB;
 *   out = z ^ (z >> 31)
 * U[a,b] = a + (b - a) * (out >> 11) * 2^-53; N(0,1) by Box-Muller on the
 * same stream (two uniforms per pair of normals).
 */
#ifndef MTLGPU_FIXTURES_H
#define MTLGPU_FIXTURES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* laplacian_setup(A, m, n) (mtl/matrix/laplacian_setup.hpp:25-44): 5-point
 * stencil on an m x n grid, row = i*n + j, 4 on the diagonal, -1 for each
 * neighbour, columns ascending.  Returns nnz. */
long long mtlgpu_gen_laplacian2d(int m, int n, int32_t* rp, int32_t* ci, double* v);

/* 7-point Laplacian on N^3, row = (i*N + j)*N + k, 6 on the diagonal, -1 per
 * neighbour inside the grid (Dirichlet: outside neighbours dropped).
 * nnz = 7N^3 - 6N^2.  Returns nnz. */
long long mtlgpu_gen_laplacian3d(int N, int32_t* rp, int32_t* ci, double* v);

/* 27-point convection-diffusion on N^3 (unsymmetric, strictly diagonally
 * dominant).  Per cell c: kappa_c = exp(0.5 * g_c), g ~ N(0,1); velocity
 * u_c ~ U[-1,1]^3 (stream `seed`: N^3 normals, then 3N^3 uniforms).  For each
 * of the 26 offsets d with weight w(d) = 1, 1/2, 1/3 for |d|^2 = 1, 2, 3:
 *   D = hm(kappa_c, kappa_nb) * w(d)   (hm = harmonic mean; kappa_nb = kappa_c
 *                                        outside the grid)
 *   C = max(0, -(u_c . d)) * w(d)      (first-order upwind inflow)
 *   a(c, nb) = -(D + C) for neighbours inside the grid,
 *   a(c, c)  = (1 + 1e-3) * sum over all 26 offsets of (D + C).
 * nnz = (3N-2)^3.  Returns nnz. */
long long mtlgpu_gen_convdiff27(int N, uint64_t seed, int32_t* rp, int32_t* ci, double* v);

/* Random-graph Laplacian plus shift: n vertices, round(n * avg_deg / 2) edge
 * draws (i, j) uniform with i != j (stream `seed`), duplicates summed into
 * the edge weight; A = D - W + shift_frac * avg_deg * I.  SPD.  Returns nnz. */
long long mtlgpu_gen_random_graph(int n, double avg_deg, double shift_frac, uint64_t seed,
                                  int32_t* rp, int32_t* ci, double* v);

/* 2-D finite-volume variable-coefficient diffusion on N x N, 5-point.
 * g = white noise N(0,1) (stream `seed`) filtered by a separable Gaussian of
 * standard deviation `corr` cells (truncated at 3 sd, zero outside), scaled
 * to unit sample variance; kappa = exp(sigma * g).  Face transmissibility
 * T = 2 k_a k_b / (k_a + k_b); Dirichlet faces on the boundary T = 2 k_c.
 * a(c,c) = sum of the cell's face T, a(c,nb) = -T.  Returns nnz. */
long long mtlgpu_gen_fv2d(int N, double sigma, double corr, uint64_t seed, int32_t* rp,
                          int32_t* ci, double* v);

/* Batch of `count` random-graph systems for the batched solver: per system
 * n = round(exp(U[ln n_min, ln n_max])), avg_deg ~ U[deg_min, deg_max],
 * sub-seed from the stream `seed`.  Writes n and nnz of every system to
 * sizes[2*count] (pass NULL arrays for sizes only); the systems are stored
 * one after another (row pointers of each system start at 0, count * (n+1)
 * entries in total).  Returns the total nnz. */
long long mtlgpu_gen_graph_batch(int count, int n_min, int n_max, double deg_min, double deg_max,
                                 double shift_frac, uint64_t seed, int64_t* sizes, int32_t* rp,
                                 int32_t* ci, double* v);

/* n values U[a, b] from the stream `seed`. */
void mtlgpu_gen_uniform(long long n, uint64_t seed, double a, double b, double* out);
/* n values N(0, 1) from the stream `seed`. */
void mtlgpu_gen_normal(long long n, uint64_t seed, double* out);
/* y = A x on the host (row sums in column order), for building right-hand
 * sides b = A x_true of the fixtures. */
void mtlgpu_gen_csr_mult(int n, const int32_t* rp, const int32_t* ci, const double* v,
                         const double* x, double* y);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
