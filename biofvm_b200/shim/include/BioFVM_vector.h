// Elementwise std::vector<double> arithmetic with BioFVM's names and
// semantics (BioFVM_vector.h): products and quotients are elementwise,
// axpy is y += a*x, naxpy is y -= a*x.
#ifndef __BioFVM_vector_h__
#define __BioFVM_vector_h__

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

namespace BioFVM {
std::vector<double> operator-(const std::vector<double>& v1, const std::vector<double>& v2);
std::vector<double> operator+(const std::vector<double>& v1, const std::vector<double>& v2);
std::vector<double> operator*(const std::vector<double>& v1, const std::vector<double>& v2);
std::vector<double> operator/(const std::vector<double>& v1, const std::vector<double>& v2);
std::vector<double> operator*(double d, const std::vector<double>& v1);
std::vector<double> operator+(double d, const std::vector<double>& v1);
std::vector<double> operator+(const std::vector<double>& v1, double d);
std::vector<double> operator-(double d, const std::vector<double>& v1);
std::vector<double> operator-(const std::vector<double>& v1, double d);
void operator+=(std::vector<double>& v1, const std::vector<double>& v2);
void operator-=(std::vector<double>& v1, const std::vector<double>& v2);
void operator/=(std::vector<double>& v1, const std::vector<double>& v2);
void operator*=(std::vector<double>& v1, const double& a);
void operator*=(std::vector<double>& v1, const std::vector<double>& v2);
void operator/=(std::vector<double>& v1, const double& a);

std::ostream& operator<<(std::ostream& os, const std::vector<double>& v);
std::vector<double> normalize(std::vector<double>& v);
void normalize(std::vector<double>* v);
double norm_squared(const std::vector<double>& v);
double norm(const std::vector<double>& v);
double maxabs(const std::vector<double>& v);
double max_abs_difference(const std::vector<double>& v1, const std::vector<double>& v2);
std::vector<double> exponentiate(const std::vector<double>& exponent);
void randomize(std::vector<double>* v);

void axpy(std::vector<double>* y, double& a, std::vector<double>& x);
void axpy(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x);
void naxpy(std::vector<double>* y, double& a, std::vector<double>& x);
void naxpy(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x);

// y = (y + a.*x) ./ d
void axpy_div(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x,
              std::vector<double>& d);
// y = y + a1.*x1 + a2.*x2
void double_axpy(std::vector<double>* y, std::vector<double>& a1, std::vector<double>& a2,
                 std::vector<double>& x1, std::vector<double>& x2);
// y = y + a.*(x1 + x2)
void double_axpy(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x1,
                 std::vector<double>& x2);
// y = (y + a.*(x1 + x2)) ./ d
void double_axpy_div(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x1,
                     std::vector<double>& x2, std::vector<double>& d);
// y = (y + a1.*x1 + a2.*x2) ./ d
void double_axpy_div(std::vector<double>* y, std::vector<double>& a1, std::vector<double>& a2,
                     std::vector<double>& x1, std::vector<double>& x2, std::vector<double>& d);

// Comma-separated values, each printed as %.7e.  vector_to_csv returns a new
// char[] buffer (release with delete[]); vector_to_csv_safe replaces the
// caller's buffer (delete[] of the old one) with a new one; the two-argument
// vector_to_csv writes into the caller's buffer, which must hold 16 chars
// per value plus one.
void csv_to_vector(const char* buffer, std::vector<double>& vect);
char* vector_to_csv(const std::vector<double>& vect);
void vector_to_csv_safe(const std::vector<double>& vect, char*& buffer);
void vector_to_csv(const std::vector<double>& vect, char*& buffer);
}  // namespace BioFVM

#endif
