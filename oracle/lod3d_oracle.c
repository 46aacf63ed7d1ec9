/*
 * lod3d_oracle.c -- TEST INFRASTRUCTURE: plain-C restatement of the
 * reference's BioFVM 3-D LOD step and agent sources (see lod3d_oracle.h).
 *
 * Arithmetic contract.  The reference is C++ built by g++ -O3 with FMA
 * available, and g++ contracts `y += a*x` into one fused multiply-add and
 * `y -= a*x` into one fused negative multiply-add.  This file is compiled
 * with -ffp-contract=off and writes every such contraction as an explicit
 * fma(), so each value below is the one the reference computes, operation
 * by operation:
 *   forward  p[i] = fma(c1, p[i-1], p[i]);  p[i] = p[i] / denom[i]
 *   backward p[i] = fma(-cupper[i], p[i+1], p[i])
 * (BioFVM/BioFVM_solvers.cpp:365-376, 693-726, 742-775).
 */
#include "lod3d_oracle.h"

#include <math.h>
#include <stdio.h>
#include <string.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* halfstep = 0: the 3-D factorization (constant2 = lambda*dt/3); 1: the 2-D
 * one of diffusion_decay_solver__constant_coefficients_LOD_2D
 * (BioFVM_solvers.cpp:1696-1707: constant2 = lambda; *= dt; *= 0.5).  Every
 * other step is the same in both solvers. */
static void thomas_axis_k(int n, int S, const double* D, const double* decay, double dt, double dx, double* denom,
                          double* cupper, double* c1, int halfstep);

void orc_thomas_axis(int n, int S, const double* D, const double* decay, double dt, double dx,
                     double* denom, double* cupper, double* c1) {
  thomas_axis_k(n, S, D, decay, dt, dx, denom, cupper, c1, 0);
}

static void thomas_axis_k(int n, int S, const double* D, const double* decay, double dt, double dx, double* denom,
                          double* cupper, double* c1, int halfstep) {
  for (int d = 0; d < S; ++d) {
    /* BioFVM_solvers.cpp:196-218: constant1 = D; *= dt; /= dx; /= dx.
       constant1a = constant1 * -1.0; constant2 = lambda*dt/3;
       constant3 = ((1 + c1) + c1) + c2; constant3a = (1 + c1) + c2. */
    double k1 = D[d];
    k1 *= dt;
    k1 /= dx;
    k1 /= dx;
    double k1a = k1 * -1.0;
    double k2 = decay[d];
    k2 *= dt;
    if (halfstep)
      k2 *= 0.5;
    else
      k2 /= 3.0;
    double k3 = 1.0;
    k3 += k1;
    k3 += k1;
    k3 += k2;
    double k3a = 1.0;
    k3a += k1;
    k3a += k2;
    c1[d] = k1;
    /* :226-245 (x, one rank) and :297-312 / :314-329 (y, z): identical. */
    for (int i = 0; i < n; ++i) {
      cupper[(size_t)i * S + d] = k1a;
      denom[(size_t)i * S + d] = k3;
    }
    denom[d] = k3a;
    denom[(size_t)(n - 1) * S + d] = k3a;
    if (n == 1) {
      double v = 1.0;
      v += k2;
      denom[d] = v;
    }
    cupper[d] /= denom[d];
    for (int i = 1; i < n; ++i) {
      /* axpy(&denom[i], constant1, c[i-1])  (BioFVM_vector.cpp:333-340) */
      denom[(size_t)i * S + d] = fma(k1, cupper[(size_t)(i - 1) * S + d], denom[(size_t)i * S + d]);
      cupper[(size_t)i * S + d] /= denom[(size_t)i * S + d];
    }
  }
}

void orc_apply_dirichlet(double* field, int nx, int ny, int nz, int S, const unsigned char* active,
                         const double* dv) {
  /* Every face voxel is set from its own entry of dv, so the order in which
     the reference visits faces (x, then y, then z) cannot change the result. */
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        if (!(i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1)) continue;
        size_t v = ((size_t)i * ny + j) * nz + k;
        for (int d = 0; d < S; ++d)
          if (active[d]) field[v * S + d] = dv[v * S + d];
      }
}

void orc_lod3d_step(double* p, int nx, int ny, int nz, int S, const double* D, const double* decay,
                    double dt, double dx, const unsigned char* active, const double* dv, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  double* coef = (double*)malloc(sizeof(double) * (2 * ((size_t)nx + ny + nz) * S + S));
  double *dnx = coef, *cx = dnx + (size_t)nx * S, *dny = cx + (size_t)nx * S, *cy = dny + (size_t)ny * S;
  double *dnz = cy + (size_t)ny * S, *cz = dnz + (size_t)nz * S, *c1 = cz + (size_t)nz * S;
  orc_thomas_axis(nx, S, D, decay, dt, dx, dnx, cx, c1);
  orc_thomas_axis(ny, S, D, decay, dt, dx, dny, cy, c1);
  orc_thomas_axis(nz, S, D, decay, dt, dx, dnz, cz, c1);
  const size_t jx = (size_t)ny * nz * S; /* thomas_i_jump */
  const size_t jy = (size_t)nz * S;      /* thomas_j_jump */
  const size_t jz = (size_t)S;           /* thomas_k_jump */

  orc_apply_dirichlet(p, nx, ny, nz, S, active, dv);

  /* x sweep (BioFVM_solvers.cpp:352-680 with one rank): lines over (j,k,d). */
#pragma omp parallel for schedule(static)
  for (long long jk = 0; jk < (long long)ny * nz; ++jk) {
    for (int d = 0; d < S; ++d) {
      double* q = p + (size_t)jk * S + d;
      q[0] /= dnx[d];
      for (int i = 1; i < nx; ++i) {
        q[i * jx] = fma(c1[d], q[(i - 1) * jx], q[i * jx]);
        q[i * jx] /= dnx[(size_t)i * S + d];
      }
      for (int i = nx - 2; i >= 0; --i) q[i * jx] = fma(-cx[(size_t)i * S + d], q[(i + 1) * jx], q[i * jx]);
    }
  }
  orc_apply_dirichlet(p, nx, ny, nz, S, active, dv);

  /* y sweep (:684-729): lines over (i,k,d). */
#pragma omp parallel for schedule(static)
  for (long long ik = 0; ik < (long long)nx * nz; ++ik) {
    const size_t i = (size_t)(ik / nz), k = (size_t)(ik % nz);
    for (int d = 0; d < S; ++d) {
      double* q = p + i * jx + k * jz + d;
      q[0] /= dny[d];
      for (int j = 1; j < ny; ++j) {
        q[j * jy] = fma(c1[d], q[(j - 1) * jy], q[j * jy]);
        q[j * jy] /= dny[(size_t)j * S + d];
      }
      for (int j = ny - 2; j >= 0; --j) q[j * jy] = fma(-cy[(size_t)j * S + d], q[(j + 1) * jy], q[j * jy]);
    }
  }
  orc_apply_dirichlet(p, nx, ny, nz, S, active, dv);

  /* z sweep (:733-777): lines over (i,j,d). */
#pragma omp parallel for schedule(static)
  for (long long ij = 0; ij < (long long)nx * ny; ++ij) {
    for (int d = 0; d < S; ++d) {
      double* q = p + (size_t)ij * (size_t)nz * S + d;
      q[0] /= dnz[d];
      for (int k = 1; k < nz; ++k) {
        q[k * jz] = fma(c1[d], q[(k - 1) * jz], q[k * jz]);
        q[k * jz] /= dnz[(size_t)k * S + d];
      }
      for (int k = nz - 2; k >= 0; --k) q[k * jz] = fma(-cz[(size_t)k * S + d], q[(k + 1) * jz], q[k * jz]);
    }
  }
  orc_apply_dirichlet(p, nx, ny, nz, S, active, dv);
  free(coef);
}

void orc_agent_constants(int S, double dt, double V, double Vvox, const double* sec, const double* upt,
                         const double* sat, const double* exp_, double* c1, double* c2, double* e2) {
  /* BioFVM_basic_agent.cpp:238: dt * volume / voxel_volume, left to right. */
  double k = dt * V / Vvox;
  for (int d = 0; d < S; ++d) {
    /* temp1 = 0; += S; *= T; *= k  (:241-244) */
    double t1 = 0.0;
    t1 += sec[d];
    t1 *= sat[d];
    t1 *= k;
    /* temp2 = 1; axpy(temp2, k, S); axpy(temp2, k, U)  (:249-251) */
    double t2 = 1.0;
    t2 = fma(k, sec[d], t2);
    t2 = fma(k, upt[d], t2);
    /* export1 = E * dt; export2 = export1 / voxel_volume  (:258-262) */
    double x1 = exp_[d];
    x1 *= dt;
    double x2 = x1;
    x2 /= Vvox;
    c1[d] = t1;
    c2[d] = t2;
    e2[d] = x2;
  }
}

void orc_sources(double* field, int S, int n, const int* voxel, const unsigned char* active, const double* c1,
                 const double* c2, const double* e2) {
  for (int a = 0; a < n; ++a) {
    if ((active && !active[a]) || voxel[a] < 0) continue;
    double* rho = field + (size_t)voxel[a] * S;
    /* BioFVM_basic_agent.cpp:538-552: += c1; /= c2; += e2 */
    for (int d = 0; d < S; ++d) rho[d] += c1[(size_t)a * S + d];
    for (int d = 0; d < S; ++d) rho[d] /= c2[(size_t)a * S + d];
    for (int d = 0; d < S; ++d) rho[d] += e2[(size_t)a * S + d];
  }
}

int orc_nearest_voxel(double x, double y, double z, double x0, double y0, double z0, double dx, int nx,
                      int ny, int nz) {
  /* Positions outside [x0, x0+n*dx] are rejected by the reference before
     indexing (General_Mesh::is_position_valid, BioFVM_mesh.cpp:242-251). */
  if (x < x0 || x > x0 + nx * dx || y < y0 || y > y0 + ny * dx || z < z0 || z > z0 + nz * dx) return -1;
  long long i = (long long)floor((x - x0) / dx);
  long long j = (long long)floor((y - y0) / dx);
  long long k = (long long)floor((z - z0) / dx);
  if (i >= nx) i = nx - 1;
  if (j >= ny) j = ny - 1;
  if (k >= nz) k = nz - 1;
  if (i < 0) i = 0;
  if (j < 0) j = 0;
  if (k < 0) k = 0;
  return (int)((i * ny + j) * nz + k);
}

/* BioFVM/BioFVM_microenvironment.cpp:1454-1616.  The three passes of the
 * reference write disjoint components, so they are restated as one loop per
 * component with the same expressions: value = a; value -= b; value /= h. */
void orc_gradients(const double* field, int nx, int ny, int nz, int S, double dx, double* out) {
  const double two_dx = dx * 2.0;
  const long jump[3] = {(long)ny * nz * S, (long)nz * S, (long)S};
  const int len[3] = {nx, ny, nz};
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int pos[3] = {i, j, k};
        const long n = ((long)i * ny + j) * nz + k;
        for (int d = 0; d < S; ++d) {
          const long idx = n * S + d;
          for (int ax = 0; ax < 3; ++ax) {
            double g = 0.0;
            if (len[ax] > 1) {
              if (pos[ax] == 0) {
                g = field[idx + jump[ax]];
                g -= field[idx];
                g /= dx;
              } else if (pos[ax] == len[ax] - 1) {
                g = field[idx];
                g -= field[idx - jump[ax]];
                g /= dx;
              } else {
                g = field[idx + jump[ax]];
                g -= field[idx - jump[ax]];
                g /= two_dx;
              }
            }
            out[idx * 3 + ax] = g;
          }
        }
      }
}

/* BioFVM/BioFVM_microenvironment.cpp:1327-1368, one value at a time in the
 * order of the reference's loops:
 *   temp2 = T; temp2 *= S;                (:1346-1347)
 *   rho += dt * temp2;     contracted to one fma by the reference build (:1349-1351)
 *   temp3 = U; temp3 += S; temp3 *= dt; temp3 += 1;   (:1353-1360)
 *   rho /= temp3;                                       (:1362-1363) */
void orc_bulk_sources(double* field, long n_values, double dt, const double* supply, const double* target,
                      const double* uptake) {
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n_values; ++q) {
    double t2 = target[q];
    t2 *= supply[q];
    double r = fma(dt, t2, field[q]);
    double t3 = uptake[q];
    t3 += supply[q];
    t3 *= dt;
    t3 += 1.0;
    r /= t3;
    field[q] = r;
  }
}

/* BioFVM/BioFVM_microenvironment.cpp:1222-1249, BioFVM/BioFVM_matlab.cpp:536-578,
 * centres from BioFVM/BioFVM_mesh.cpp:1436-1560 (one rank: the local start is
 * start + 0.0). */
int orc_write_matlab(const char* path, const double* field, int nx, int ny, int nz, int S, double x0, double y0,
                     double z0, double dx) {
  FILE* fp = fopen(path, "wb");
  if (!fp) return -1;
  static const char name[] = "multiscale_microenvironment";
  const unsigned int hdr[5] = {0u, (unsigned int)(4 + S), (unsigned int)((long)nx * ny * nz), 0u,
                               (unsigned int)(sizeof(name) - 1)};
  fwrite(hdr, sizeof(unsigned int), 5, fp);
  fwrite(name, 1, sizeof(name) - 1, fp);
  double dv = dx * dx;
  dv *= dx;
  const double xs = x0 + 0.0, ys = y0 + 0.0, zs = z0 + 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const double col[4] = {fma(i + 0.5, dx, xs), fma(j + 0.5, dx, ys), fma(k + 0.5, dx, zs), dv};
        fwrite(col, sizeof(double), 4, fp);
        fwrite(field + (((long)i * ny + j) * nz + k) * S, sizeof(double), (size_t)S, fp);
      }
  return fclose(fp) == 0 ? 0 : -1;
}

/* BioFVM/BioFVM_basic_agent.cpp:509-559 with tracking on, in its operation
 * order (no contractions: the steps run in separate loops and vector
 * operators). */
void orc_sources_tracked(double* field, int S, int n, const int* voxel, const unsigned char* active, const double* c1,
                         const double* c2, const double* e2, const double* e1, double vvox, double* internal) {
  for (int a = 0; a < n; ++a) {
    if ((active && !active[a]) || voxel[a] < 0) continue;
    double* rho = field + (size_t)voxel[a] * S;
    for (int d = 0; d < S; ++d) {
      const size_t q = (size_t)a * S + d;
      double tec = 1.0;
      tec -= c2[q];
      tec *= rho[d];
      tec += c1[q];
      tec /= c2[q];
      tec *= vvox;
      internal[q] -= tec;
    }
    for (int d = 0; d < S; ++d) rho[d] += c1[(size_t)a * S + d];
    for (int d = 0; d < S; ++d) rho[d] /= c2[(size_t)a * S + d];
    for (int d = 0; d < S; ++d) rho[d] += e2[(size_t)a * S + d];
    for (int d = 0; d < S; ++d) internal[(size_t)a * S + d] -= e1[(size_t)a * S + d];
  }
}

/* BioFVM/BioFVM_basic_agent.cpp:310-333 for agents[0..count) in that order:
 * internal /= vvox; internal *= fraction; rho += internal; internal = 0.
 * Agents without a voxel (voxel < 0) are skipped. */
void orc_release_internalized(double* field, int S, int count, const int* agents, const int* voxel,
                              const double* fraction, double vvox, double* internal) {
  for (int q = 0; q < count; ++q) {
    const int a = agents[q];
    if (voxel[a] < 0) continue;
    double* rho = field + (size_t)voxel[a] * S;
    double* in = internal + (size_t)a * S;
    for (int d = 0; d < S; ++d) in[d] /= vvox;
    for (int d = 0; d < S; ++d) in[d] *= fraction[(size_t)q * S + d];
    for (int d = 0; d < S; ++d) rho[d] += in[d];
    for (int d = 0; d < S; ++d) in[d] = 0.0;
  }
}

/* Microenvironment::apply_dirichlet_conditions (BioFVM/BioFVM_microenvironment.cpp:
 * 303-323) over a node list: for node q, every substrate d with act[q][d]
 * set takes values[q][d].  act NULL: all set.  Nodes hold distinct voxels. */
void orc_dirichlet_nodes(double* field, int S, int count, const int* voxel, const double* values,
                         const unsigned char* act) {
  for (int q = 0; q < count; ++q)
    for (int d = 0; d < S; ++d)
      if (!act || act[(size_t)q * S + d]) field[(size_t)voxel[q] * S + d] = values[(size_t)q * S + d];
}

/* One step of the 2-D LOD solver, diffusion_decay_solver__constant_coefficients_LOD_2D
 * (BioFVM/BioFVM_solvers.cpp:1668-1832) as its commented-out vector forms
 * state it: nodes pinned; x sweep; nodes pinned; y sweep; nodes pinned.
 * Field in the reference layout with nz = 1: (i*ny + j)*S + d.  The x lines
 * step by ny*S values and the y lines by S (the reference's loops in this
 * tree step by S and by nx, which walk other lines or past the array for
 * most shapes, and add the y upper-diagonal term where the commented naxpy
 * subtracts it; they agree with this restatement when ny == 1). */
void orc_lod2d_step(double* p, int nx, int ny, int S, const double* D, const double* decay, double dt, double dx,
                    int count, const int* voxel, const double* values, const unsigned char* act) {
  double* coef = (double*)malloc(sizeof(double) * (2 * ((size_t)nx + ny) * S + S));
  double *dnx = coef, *cx = dnx + (size_t)nx * S, *dny = cx + (size_t)nx * S, *cy = dny + (size_t)ny * S;
  double* c1 = cy + (size_t)ny * S;
  thomas_axis_k(nx, S, D, decay, dt, dx, dnx, cx, c1, 1);
  thomas_axis_k(ny, S, D, decay, dt, dx, dny, cy, c1, 1);
  const size_t jx = (size_t)ny * S, jy = (size_t)S;
  orc_dirichlet_nodes(p, S, count, voxel, values, act);
  for (int j = 0; j < ny; ++j)
    for (int d = 0; d < S; ++d) {
      double* q = p + (size_t)j * S + d;
      q[0] /= dnx[d];
      for (int i = 1; i < nx; ++i) {
        q[i * jx] = fma(c1[d], q[(i - 1) * jx], q[i * jx]);
        q[i * jx] /= dnx[(size_t)i * S + d];
      }
      for (int i = nx - 2; i >= 0; --i) q[i * jx] = fma(-cx[(size_t)i * S + d], q[(i + 1) * jx], q[i * jx]);
    }
  orc_dirichlet_nodes(p, S, count, voxel, values, act);
  for (int i = 0; i < nx; ++i)
    for (int d = 0; d < S; ++d) {
      double* q = p + (size_t)i * jx + d;
      q[0] /= dny[d];
      for (int j = 1; j < ny; ++j) {
        q[j * jy] = fma(c1[d], q[(j - 1) * jy], q[j * jy]);
        q[j * jy] /= dny[(size_t)j * S + d];
      }
      for (int j = ny - 2; j >= 0; --j) q[j * jy] = fma(-cy[(size_t)j * S + d], q[(j + 1) * jy], q[j * jy]);
    }
  orc_dirichlet_nodes(p, S, count, voxel, values, act);
  free(coef);
}
