// Host-side numerics that must reproduce the reference bit for bit.  This
// file is compiled with -ffp-contract=off so that no multiply-add is fused,
// matching the reference's shipped x86-64 build (-march=core2, no FMA).
#include "bfvm_host_math.h"

#include <cmath>
#include <vector>

namespace bfvm {

int nodes_from_spacing(double start, double end, double d) {
  // Cartesian_Mesh::resize(..., dx, dy, dz), BioFVM_mesh.cpp:802-805
  double eps = 1e-16;
  return (int)std::ceil(eps + (end - start) / d);
}

void thomas_axis(int n, int S, double dx, double dt, const double* D, const double* decay,
                 double* c1, double* denom, double* cx, int dims) {
  for (int s = 0; s < S; ++s) {
    // BioFVM_solvers.cpp:105-126: the constants are built by the same
    // sequence of elementwise operations.
    double k1 = D[s];
    k1 *= dt;
    k1 /= dx;
    k1 /= dx;
    double k1a = k1;
    k1a *= -1.0;
    double k2 = decay[s];
    k2 *= dt;
    if (dims == 2)
      k2 *= 0.5;  // LOD_2D splits the decay over two sweeps (BioFVM_solvers.cpp:311-312)
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
    // :130-135 boundary rows carry 1 + c1 + c2 (Neumann); a single point 1 + c2
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
    // :137-142 forward elimination of the constant matrix
    cx[s] /= denom[s];
    for (int i = 1; i <= n - 1; ++i) {
      denom[(size_t)i * S + s] += k1 * cx[(size_t)(i - 1) * S + s];
      cx[(size_t)i * S + s] /= denom[(size_t)i * S + s];
    }
  }
}

void bulk_coefficients(int S, const double* supply, const double* target, const double* uptake,
                       double* st, double* su) {
  // BioFVM_microenvironment.cpp:603,605: temp2 = T*S, temp3 = U+S
  for (int s = 0; s < S; ++s) {
    double t1 = supply ? supply[s] : 0.0;
    double t2 = target ? target[s] : 0.0;
    double t3 = uptake ? uptake[s] : 0.0;
    t2 *= t1;
    t3 += t1;
    st[s] = t2;
    su[s] = t3;
  }
}

}  // namespace bfvm

namespace bfvm {

void chunk_tables(int n, int S, int ch, const double* c1, const double* denom, const double* cx,
                  double* k1, double* kg, double* kc) {
  const int nc = (n + ch - 1) / ch;
  for (size_t i = 0; i < (size_t)nc * ch * S * 2; ++i) k1[i] = kg[i] = 0.0;
  for (int s = 0; s < S; ++s) {
    for (int c = 0; c < nc; ++c) {
      const int k0 = c * ch, k1e = (k0 + ch < n) ? k0 + ch : n;
      double P = 1.0;
      for (int k = k0; k < k1e; ++k) {
        const size_t q = (size_t)k * S + s;
        const double a = -cx[q];  // == c1[s] / denom[q], see the header
        P *= a;
        k1[q * 2 + 0] = 1.0 / denom[q];
        k1[q * 2 + 1] = a;
        kg[q * 2 + 0] = P;  // P_k for now, turned into G_k below
      }
      double R = 1.0, G = 0.0;
      for (int k = k1e - 1; k >= k0; --k) {
        const size_t q = (size_t)k * S + s;
        const double a = k1[q * 2 + 1];
        G = kg[q * 2 + 0] + a * G;
        R *= a;
        kg[q * 2 + 0] = G;
        kg[q * 2 + 1] = R;
      }
      double* t = kc + ((size_t)c * S + s) * 4;
      t[0] = P;
      t[1] = kg[((size_t)k0 * S + s) * 2 + 0];
      t[2] = kg[((size_t)k0 * S + s) * 2 + 1];
      t[3] = 0.0;
    }
  }
  (void)c1;
}


namespace {

// The float nearest v first, then the float on v's other side (if v is not
// a float itself).
int float_candidates(double v, float out[2]) {
  const float r = (float)v;
  out[0] = r;
  if ((double)r == v) return 1;
  out[1] = std::nextafter(r, (double)r < v ? INFINITY : -INFINITY);
  return 2;
}

}  // namespace

void fp32_tables(int n, int S, const double* c1, const double* denom, const double* cx,
                 float* inv, float* fwd, float* bwd, float* c1f, double* tile_den,
                 double* tile_cx) {
  constexpr int kPeriod = 8, kBlock = 32;
  std::vector<double> qe(n), xe(n);
  std::vector<float> tinv(n);
  std::vector<char> per((size_t)(n + kBlock - 1) / kBlock, 0);
  // nearest float first, then the one on the other side of v
  auto pick = [](double v, auto err) {
    float cand[2];
    const int nc = float_candidates(v, cand);
    float best = cand[0];
    double best_e = err(cand[0]);
    for (int j = 1; j < nc; ++j) {
      const double e = err(cand[j]);
      if (std::fabs(e) < std::fabs(best_e)) {
        best = cand[j];
        best_e = e;
      }
    }
    return best;
  };
  for (int s = 0; s < S; ++s) {
    auto at = [&](const double* a, int k) { return a[(size_t)k * S + s]; };
    c1f[s] = (float)c1[s];
    const double c1r = (double)c1f[s];
    // exact solve of a unit right-hand side (the reference's elimination)
    double q = 0.0;
    for (int k = 0; k < n; ++k) {
      q = (1.0 + c1[s] * q) / at(denom, k);
      qe[k] = q;
    }
    double x = 0.0;
    for (int k = n - 1; k >= 0; --k) {
      x = qe[k] - at(cx, k) * x;
      xe[k] = x;
    }
    // Whole 32-point blocks whose exact coefficients repeat with period 8
    // (the converged interior of a long line): there the roundings repeat
    // too, so that every chunk of 8, 16 or 32 points inside keeps identical
    // tables (the tile kernels share the tables of identical chunks).  The
    // greedy choices of the 8 points where such a region is entered (its
    // last 8 points backward, its first 8 forward) are the repeated period.
    for (size_t j = 0; j < per.size(); ++j) {
      bool ok = j > 0 && (int)((j + 1) * kBlock) <= n;
      for (int k = (int)j * kBlock; ok && k < (int)(j + 1) * kBlock; ++k)
        ok = at(denom, k) == at(denom, k - kPeriod) && at(cx, k) == at(cx, k - kPeriod);
      per[j] = ok;
    }
    auto periodic = [&](int k) { return k >= 0 && k < n && per[k / kBlock]; };
    // backward coefficients (shared by both forms): x_k = q_k + b_k x_{k+1}
    double xc = 0.0;
    for (int k = n - 1; k >= 0; --k) {
      const size_t i = (size_t)k * S + s;
      float b;
      if (periodic(k) && periodic(k + kPeriod))
        b = bwd[i + (size_t)kPeriod * S];
      else
        b = pick(-cx[i], [&](float c) { return qe[k] + (double)c * xc - xe[k]; });
      bwd[i] = b;
      tile_cx[i] = -(double)b;
      xc = qe[k] + (double)b * xc;
    }
    // forward: register form q_k = (1 + c1 q_{k-1}) inv_k, every point chosen
    // (its tables are not shared between chunks); tile form
    // q_k = a_k q_{k-1} + inv'_k with a_k = b_k
    double qr = 0.0, qt = 0.0;
    for (int k = 0; k < n; ++k) {
      const size_t i = (size_t)k * S + s;
      const double v = 1.0 / denom[i];
      const float r = pick(v, [&](float c) { return (1.0 + c1r * qr) * (double)c - qe[k]; });
      inv[i] = r;
      fwd[i] = (float)(c1r * (double)r);
      qr = (1.0 + c1r * qr) * (double)r;
      float t;
      if (periodic(k) && periodic(k - kPeriod))
        t = tinv[k - kPeriod];
      else
        t = pick(v, [&](float c) { return (double)bwd[i] * qt + (double)c - qe[k]; });
      tinv[k] = t;
      tile_den[i] = 1.0 / (double)t;
      qt = (double)bwd[i] * qt + (double)t;
    }
  }
}

}  // namespace bfvm
