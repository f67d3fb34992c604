#pragma once

namespace bfvm {

// (int) ceil(1e-16 + (end - start)/d)  (BioFVM_mesh.cpp:802-805)
int nodes_from_spacing(double start, double end, double d);

// Thomas coefficients of one axis, [n][S] (BioFVM_solvers.cpp:105-170 for
// the 3-D LOD solver, dims = 3; :293-336 for the 2-D one, dims = 2, which
// splits the decay in halves instead of thirds).
void thomas_axis(int n, int S, double dx, double dt, const double* D, const double* decay,
                 double* c1, double* denom, double* cx, int dims = 3);

// Per-voxel bulk coefficients st = T*S and su = U+S
// (BioFVM_microenvironment.cpp:603,605); NULL rate arrays are zero.
void bulk_coefficients(int S, const double* supply, const double* target, const double* uptake,
                       double* st, double* su);

}  // namespace bfvm

namespace bfvm {

// Tables of the chunked sweep for one axis (n points, S densities, chunks of
// ch points), from the Thomas coefficients denom/cx [n][S] and c1 [S], all
// interleaved [point][density] like the field itself (k1, kg sized
// nc*ch*S*2 so that every chunk has a full block; entries past n are 0):
//   k1[k][s] = {1/d_k, a_k}   a_k = c1/d_k = -cx_k (the same value: the
//                             reference builds cx_k = -c1/d_k), so
//                             forward:  q_k = a_k q_{k-1} + p_k/d_k
//                             backward: x_k = a_k x_{k+1} + q_k
//   kg[k][s] = {G_k, R_k}     x_k = x'_k + cf*G_k + cb*R_k, where x' is the
//                             chunk-local solve with zero carries, cf/cb the
//                             forward/backward carries into the chunk,
//                             R_k = prod_{j=k}^{end} a_j and G the chunk-local
//                             back substitution of P_k = prod_{j=start}^{k} a_j
//   kc[c][s] = {P_end, G_start, R_start, 0}   per-chunk transfer constants
void chunk_tables(int n, int S, int ch, const double* c1, const double* denom, const double* cx,
                  double* k1, double* kg, double* kc);

// FP32 Thomas tables of one axis whose roundings keep a constant field's
// decay rate.  Rounded to nearest one by one, every interior point of a line
// gets the same rounded coefficients, so every sweep scales the field by the
// same slightly wrong factor and the bias grows linearly with the step count
// (up to ~2e-5 relative after 150 sweeps of a 512-point line at
// c1 = dt D / dx^2 = 10).  Here each coefficient is rounded down or up
// (one of the two floats around it), greedily along the line, so that the
// solve of a unit right-hand side carried out with the FP32 coefficients
// stays closest to the exact one (error diffusion).  Where the exact
// coefficients repeat with period 8 (the converged interior of a line, in
// whole 32-point blocks) the choices of the first 8 points there repeat, so
// chunks of 8, 16 or 32 points inside keep identical tables.
//   register form (lod_sweep_kernel): q_k = (p_k + c1 q_{k-1}) inv_k,
//     x_k = q_k + bwd_k x_{k+1}; fwd_k = c1 inv_k (the carry products);
//     out: inv, fwd, bwd [n][S], c1f [S];
//   tile form (line and row kernels): q_k = a_k q_{k-1} + p_k inv'_k,
//     x_k = a_k x_{k+1} + q_k with a_k = bwd_k; out as FP64 arrays
//     den' = 1 / inv'_k and cx' = -a_k [n][S], from which chunk_tables
//     builds tables that round back to exactly these floats.
void fp32_tables(int n, int S, const double* c1, const double* denom, const double* cx,
                 float* inv, float* fwd, float* bwd, float* c1f, double* tile_den,
                 double* tile_cx);

}  // namespace bfvm
