/* Test infrastructure only (the oracle): a plain-C, single-threaded CPU
 * restatement of BioFVM 1.0.4's per-step transport path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as
 * the checker; the product library never links or calls it.
 *
 * Every function follows the reference statement by statement (same
 * operations, same order, IEEE double, no FMA contraction: build with
 * -ffp-contract=off), so on the same inputs it reproduces the reference's
 * shipped core2 build.  The file:line citations are relative to the BioFVM
 * source tree.
 *
 * Layout: densities are [voxel][substrate] with voxel n = (k*ny + j)*nx + i
 * (BioFVM_mesh.cpp:641-644), the reference's own logical order. */
#ifndef BFVM_ORACLE_H
#define BFVM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Node count along one axis for resize_space(..., dx, dy, dz):
 * (int) ceil(1e-16 + (end - start)/d)   (BioFVM_mesh.cpp:802-805). */
int or_nodes_from_spacing(double start, double end, double d);

/* nearest_voxel_index (BioFVM_mesh.cpp:930-948): floor((x - min)/d),
 * clamped to [0, n-1] on each axis. */
int64_t or_nearest_voxel(const double* box_min, double dx, double dy, double dz, int nx,
                         int ny, int nz, double x, double y, double z);

/* Thomas coefficients of one axis for the 2-D LOD solver
 * (BioFVM_solvers.cpp:293-336): as or_thomas_setup with the decay split in
 * halves (constant2 *= 0.5). */
void or_thomas_setup_2d(int n, int S, double dx, double dt, const double* D,
                        const double* decay, double* c1, double* denom, double* cx);

/* diffusion_decay_solver__constant_coefficients_LOD_2D (BioFVM_solvers.cpp:
 * 339-426): Dirichlet, x-Thomas on the z = 0 plane, Dirichlet, y-Thomas. */
void or_lod2d(int nx, int ny, int S, double* p, const double* c1, const double* denx,
              const double* cxx, const double* deny, const double* cxy, int ndir,
              const int64_t* dir_idx, const double* dir_val);

/* Thomas coefficients of one axis (BioFVM_solvers.cpp:105-170).
 * c1[S] = dt*D/dx^2, denom[n*S], cx[n*S] ([point][substrate]).  The
 * reference uses mesh.dx for all three axes (BioFVM_solvers.cpp:112-113). */
void or_thomas_setup(int n, int S, double dx, double dt, const double* D, const double* decay,
                     double* c1, double* denom, double* cx);

/* apply_dirichlet_conditions (BioFVM_microenvironment.cpp:192-197): copies
 * each node's whole value vector, nodes applied in list order. */
void or_apply_dirichlet(int S, double* p, int ndir, const int64_t* idx, const double* val);

/* diffusion_decay_solver__constant_coefficients_LOD_3D
 * (BioFVM_solvers.cpp:175-273): Dirichlet, x-Thomas, Dirichlet, y-Thomas,
 * Dirichlet, z-Thomas. */
void or_lod3d(int nx, int ny, int nz, int S, double* p, const double* c1, const double* denx,
              const double* cxx, const double* deny, const double* cxy, const double* denz,
              const double* cxz, int ndir, const int64_t* dir_idx, const double* dir_val);

/* simulate_bulk_sources_and_sinks (BioFVM_microenvironment.cpp:595-610).
 * supply/target/uptake are the callback outputs [N][S]; NULL = zero. */
void or_bulk(int64_t N, int S, double* p, const double* supply, const double* target,
             const double* uptake, double dt);

/* Basic_Agent::set_internal_uptake_constants (BioFVM_basic_agent.cpp:114-148). */
void or_agent_constants(int S, double dt, double volume, double voxel_volume,
                        const double* secretion, const double* saturation, const double* uptake,
                        double* temp1, double* temp2);

/* simulate_cell_sources_and_sinks -> Basic_Agent::simulate_secretion_and_uptake
 * (BioFVM_microenvironment.cpp:615-633, BioFVM_basic_agent.cpp:229-238), in
 * agent-list order. */
void or_cells(int64_t A, int S, double* p, const int64_t* voxel, const double* temp1,
              const double* temp2);

/* nsteps of bulk -> cells -> LOD_3D (flags: 1 bulk, 2 cells, 4 diffusion),
 * with the Thomas setup done once from dt (BioFVM_solvers.cpp:87-173). */
void or_run(int nx, int ny, int nz, int S, double dx, double dt, int nsteps, int flags,
            double* p, const double* D, const double* decay, const double* supply,
            const double* target, const double* uptake, int64_t A, const int64_t* agent_voxel,
            const double* temp1, const double* temp2, int ndir, const int64_t* dir_idx,
            const double* dir_val);

/* compute_all_gradient_vectors (BioFVM_microenvironment.cpp:702-787): central
 * differences at points with both neighbours along an axis, into g
 * [N][S][3]; other components are left as they are. */
void or_gradients(int nx, int ny, int nz, int S, const double* p, double dx, double dy,
                  double dz, double* g);

#ifdef __cplusplus
}
#endif
#endif
