/* Test infrastructure only (the oracle).  Plain-C restatement of BioFVM
 * 1.0.4's transport step; see bfvm_oracle.h for scope and conventions.
 * Every loop below names the reference statements it restates. */
#include "bfvm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

int or_nodes_from_spacing(double start, double end, double d) {
  /* BioFVM_mesh.cpp:802-805 */
  double eps = 1e-16;
  return (int)ceil(eps + (end - start) / d);
}

int64_t or_nearest_voxel(const double* box_min, double dx, double dy, double dz, int nx,
                         int ny, int nz, double x, double y, double z) {
  /* BioFVM_mesh.cpp:932-947 */
  int i = (int)floor((x - box_min[0]) / dx);
  int j = (int)floor((y - box_min[1]) / dy);
  int k = (int)floor((z - box_min[2]) / dz);
  if (i >= nx) i = nx - 1;
  if (i < 0) i = 0;
  if (j >= ny) j = ny - 1;
  if (j < 0) j = 0;
  if (k >= nz) k = nz - 1;
  if (k < 0) k = 0;
  return ((int64_t)k * ny + j) * nx + i;
}

static void thomas_setup_split(int n, int S, double dx, double dt, const double* D,
                               const double* decay, double* c1, double* denom, double* cx,
                               int dims) {
  for (int s = 0; s < S; ++s) {
    /* BioFVM_solvers.cpp:105-126: each constant built by the same sequence
     * of elementwise vector operations. */
    double k1 = D[s];
    k1 *= dt;
    k1 /= dx;
    k1 /= dx;
    double k1a = k1;
    k1a *= -1.0;
    double k2 = decay[s];
    k2 *= dt;
    if (dims == 2)
      k2 *= 0.5; /* :311-312 */
    else
      k2 /= 3.0;
    double k3 = 1.0;
    k3 += k1;
    k3 += k1;
    k3 += k2;
    double k3a = 1.0;
    k3a += k1;
    k3a += k2;
    c1[s] = k1;
    /* :130-135 */
    for (int i = 0; i < n; ++i) {
      cx[(size_t)i * S + s] = k1a;
      denom[(size_t)i * S + s] = k3;
    }
    denom[s] = k3a;
    denom[(size_t)(n - 1) * S + s] = k3a;
    if (n == 1) {
      denom[s] = 1.0;
      denom[s] += k2;
    }
    /* :137-142 */
    cx[s] /= denom[s];
    for (int i = 1; i <= n - 1; ++i) {
      denom[(size_t)i * S + s] += k1 * cx[(size_t)(i - 1) * S + s];
      cx[(size_t)i * S + s] /= denom[(size_t)i * S + s];
    }
  }
}

void or_thomas_setup(int n, int S, double dx, double dt, const double* D, const double* decay,
                     double* c1, double* denom, double* cx) {
  thomas_setup_split(n, S, dx, dt, D, decay, c1, denom, cx, 3);
}

void or_thomas_setup_2d(int n, int S, double dx, double dt, const double* D,
                        const double* decay, double* c1, double* denom, double* cx) {
  thomas_setup_split(n, S, dx, dt, D, decay, c1, denom, cx, 2);
}

void or_apply_dirichlet(int S, double* p, int ndir, const int64_t* idx, const double* val) {
  /* BioFVM_microenvironment.cpp:194-196 */
  for (int d = 0; d < ndir; ++d)
    memcpy(p + (size_t)idx[d] * S, val + (size_t)d * S, sizeof(double) * (size_t)S);
}

/* One axis of the LOD solve for every line: forward elimination then back
 * substitution, the exact statement sequence of BioFVM_solvers.cpp:186-200
 * (x), :217-234 (y) and :252-271 (z).  A line starts at base, its points are
 * jump apart. */
static void thomas_line(double* p, int64_t base, int64_t jump, int n, int S, const double* c1,
                        const double* den, const double* cx) {
  double* v = p + base * S;
  for (int s = 0; s < S; ++s) v[s] /= den[s];
  for (int i = 1; i < n; ++i) {
    double* cur = p + (base + (int64_t)i * jump) * S;
    const double* prev = cur - jump * S;
    for (int s = 0; s < S; ++s) cur[s] += c1[s] * prev[s];
    for (int s = 0; s < S; ++s) cur[s] /= den[(size_t)i * S + s];
  }
  for (int i = n - 2; i >= 0; --i) {
    double* cur = p + (base + (int64_t)i * jump) * S;
    const double* next = cur + jump * S;
    for (int s = 0; s < S; ++s) cur[s] -= cx[(size_t)i * S + s] * next[s];
  }
}

void or_lod3d(int nx, int ny, int nz, int S, double* p, const double* c1, const double* denx,
              const double* cxx, const double* deny, const double* cxy, const double* denz,
              const double* cxz, int ndir, const int64_t* dir_idx, const double* dir_val) {
  const int64_t ij = 1, jj = nx, kj = (int64_t)nx * ny;
  /* x-diffusion, :177-203 */
  or_apply_dirichlet(S, p, ndir, dir_idx, dir_val);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j) thomas_line(p, ((int64_t)k * ny + j) * nx, ij, nx, S, c1, denx, cxx);
  /* y-diffusion, :207-237 */
  or_apply_dirichlet(S, p, ndir, dir_idx, dir_val);
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) thomas_line(p, (int64_t)k * ny * nx + i, jj, ny, S, c1, deny, cxy);
  /* z-diffusion, :241-273 */
  or_apply_dirichlet(S, p, ndir, dir_idx, dir_val);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) thomas_line(p, (int64_t)j * nx + i, kj, nz, S, c1, denz, cxz);
}

void or_lod2d(int nx, int ny, int S, double* p, const double* c1, const double* denx,
              const double* cxx, const double* deny, const double* cxy, int ndir,
              const int64_t* dir_idx, const double* dir_val) {
  /* :367-392 x-diffusion of the rows of the z = 0 plane */
  or_apply_dirichlet(S, p, ndir, dir_idx, dir_val);
  for (int j = 0; j < ny; ++j) thomas_line(p, (int64_t)j * nx, 1, nx, S, c1, denx, cxx);
  /* :394-425 y-diffusion */
  or_apply_dirichlet(S, p, ndir, dir_idx, dir_val);
  for (int i = 0; i < nx; ++i) thomas_line(p, i, nx, ny, S, c1, deny, cxy);
}

void or_bulk(int64_t N, int S, double* p, const double* supply, const double* target,
             const double* uptake, double dt) {
  /* BioFVM_microenvironment.cpp:598-609; temp1 = S, temp2 = T, temp3 = U. */
  for (int64_t n = 0; n < N; ++n) {
    for (int s = 0; s < S; ++s) {
      size_t q = (size_t)n * S + s;
      double t1 = supply ? supply[q] : 0.0;
      double t2 = target ? target[q] : 0.0;
      double t3 = uptake ? uptake[q] : 0.0;
      t2 *= t1;           /* :603 temp2 = S*T        */
      p[q] += dt * t2;    /* :604 axpy               */
      t3 += t1;           /* :605 temp3 = U+S        */
      t3 *= dt;           /* :606                    */
      t3 += 1.0;          /* :607                    */
      p[q] /= t3;         /* :609                    */
    }
  }
}

void or_agent_constants(int S, double dt, double volume, double voxel_volume,
                        const double* secretion, const double* saturation, const double* uptake,
                        double* temp1, double* temp2) {
  /* BioFVM_basic_agent.cpp:122 */
  double c = dt * volume / voxel_volume;
  for (int s = 0; s < S; ++s) {
    /* :139-142 */
    double a = 0.0;
    a += secretion[s];
    a *= saturation[s];
    a *= c;
    /* :145-147 */
    double b = 1.0;
    b += c * secretion[s];
    b += c * uptake[s];
    temp1[s] = a;
    temp2[s] = b;
  }
}

void or_cells(int64_t A, int S, double* p, const int64_t* voxel, const double* temp1,
              const double* temp2) {
  /* BioFVM_basic_agent.cpp:234-235, agents in list order */
  for (int64_t a = 0; a < A; ++a) {
    double* v = p + (size_t)voxel[a] * S;
    for (int s = 0; s < S; ++s) v[s] += temp1[(size_t)a * S + s];
    for (int s = 0; s < S; ++s) v[s] /= temp2[(size_t)a * S + s];
  }
}

void or_run(int nx, int ny, int nz, int S, double dx, double dt, int nsteps, int flags,
            double* p, const double* D, const double* decay, const double* supply,
            const double* target, const double* uptake, int64_t A, const int64_t* agent_voxel,
            const double* temp1, const double* temp2, int ndir, const int64_t* dir_idx,
            const double* dir_val) {
  const int64_t N = (int64_t)nx * ny * nz;
  double* c1 = (double*)malloc(sizeof(double) * (size_t)S);
  double* denx = (double*)malloc(sizeof(double) * (size_t)nx * S);
  double* cxx = (double*)malloc(sizeof(double) * (size_t)nx * S);
  double* deny = (double*)malloc(sizeof(double) * (size_t)ny * S);
  double* cxy = (double*)malloc(sizeof(double) * (size_t)ny * S);
  double* denz = (double*)malloc(sizeof(double) * (size_t)nz * S);
  double* cxz = (double*)malloc(sizeof(double) * (size_t)nz * S);
  /* Thomas setup once, from the first call's dt (BioFVM_solvers.cpp:87,172). */
  or_thomas_setup(nx, S, dx, dt, D, decay, c1, denx, cxx);
  or_thomas_setup(ny, S, dx, dt, D, decay, c1, deny, cxy);
  or_thomas_setup(nz, S, dx, dt, D, decay, c1, denz, cxz);
  for (int it = 0; it < nsteps; ++it) {
    if (flags & 1) or_bulk(N, S, p, supply, target, uptake, dt);
    if (flags & 2) or_cells(A, S, p, agent_voxel, temp1, temp2);
    if (flags & 4)
      or_lod3d(nx, ny, nz, S, p, c1, denx, cxx, deny, cxy, denz, cxz, ndir, dir_idx, dir_val);
  }
  free(c1);
  free(denx);
  free(cxx);
  free(deny);
  free(cxy);
  free(denz);
  free(cxz);
}

void or_gradients(int nx, int ny, int nz, int S, const double* p, double dx, double dy,
                  double dz, double* g) {
  /* BioFVM_microenvironment.cpp:702-787; two_d = d; two_d *= 2.0 (:704-713) */
  const double two_dx = dx * 2.0, two_dy = dy * 2.0, two_dz = dz * 2.0;
  const int64_t jx = S, jy = (int64_t)nx * S, jz = (int64_t)nx * ny * S;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        for (int s = 0; s < S; ++s) {
          const int64_t q = (((int64_t)k * ny + j) * nx + i) * S + s;
          double* o = g + 3 * q;
          if (i > 0 && i < nx - 1) { /* :728-730 */
            o[0] = p[q + jx];
            o[0] -= p[q - jx];
            o[0] /= two_dx;
          }
          if (j > 0 && j < ny - 1) { /* :751-753 */
            o[1] = p[q + jy];
            o[1] -= p[q - jy];
            o[1] /= two_dy;
          }
          if (k > 0 && k < nz - 1) { /* :774-776 */
            o[2] = p[q + jz];
            o[2] -= p[q - jz];
            o[2] /= two_dz;
          }
        }
}
