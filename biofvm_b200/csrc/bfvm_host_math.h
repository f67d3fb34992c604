#pragma once

namespace bfvm {

// (int) ceil(1e-16 + (end - start)/d)  (BioFVM_mesh.cpp:802-805)
int nodes_from_spacing(double start, double end, double d);

// Thomas coefficients of one axis, [n][S] (BioFVM_solvers.cpp:105-170).
void thomas_axis(int n, int S, double dx, double dt, const double* D, const double* decay,
                 double* c1, double* denom, double* cx);

// Per-voxel bulk coefficients st = T*S and su = U+S
// (BioFVM_microenvironment.cpp:603,605); NULL rate arrays are zero.
void bulk_coefficients(int S, const double* supply, const double* target, const double* uptake,
                       double* st, double* su);

}  // namespace bfvm
