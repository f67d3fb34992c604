// Vector arithmetic, stopwatch and MATLAB v4 I/O of the drop-in headers.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <random>
#include <sstream>

#include "BioFVM.h"

namespace BioFVM {

std::string BioFVM_Version = "1.0.4";
std::string BioFVM_URL = "http://BioFVM.MathCancer.org";

// ---- vectors (elementwise, like BioFVM_vector.cpp) ------------------------

namespace {
template <typename F>
std::vector<double> zip(const std::vector<double>& a, const std::vector<double>& b, F f) {
  std::vector<double> r(a.size());
  for (size_t i = 0; i < a.size(); ++i) r[i] = f(a[i], b[i]);
  return r;
}
template <typename F>
std::vector<double> each(const std::vector<double>& a, F f) {
  std::vector<double> r(a.size());
  for (size_t i = 0; i < a.size(); ++i) r[i] = f(a[i]);
  return r;
}
}  // namespace

std::vector<double> operator-(const std::vector<double>& v1, const std::vector<double>& v2) {
  return zip(v1, v2, [](double a, double b) { return a - b; });
}
std::vector<double> operator+(const std::vector<double>& v1, const std::vector<double>& v2) {
  return zip(v1, v2, [](double a, double b) { return a + b; });
}
std::vector<double> operator*(const std::vector<double>& v1, const std::vector<double>& v2) {
  return zip(v1, v2, [](double a, double b) { return a * b; });
}
std::vector<double> operator/(const std::vector<double>& v1, const std::vector<double>& v2) {
  return zip(v1, v2, [](double a, double b) { return a / b; });
}
std::vector<double> operator*(double d, const std::vector<double>& v1) {
  return each(v1, [d](double a) { return d * a; });
}
std::vector<double> operator+(double d, const std::vector<double>& v1) {
  return each(v1, [d](double a) { return d + a; });
}
std::vector<double> operator+(const std::vector<double>& v1, double d) {
  return each(v1, [d](double a) { return a + d; });
}
std::vector<double> operator-(double d, const std::vector<double>& v1) {
  return each(v1, [d](double a) { return d - a; });
}
std::vector<double> operator-(const std::vector<double>& v1, double d) {
  return each(v1, [d](double a) { return a - d; });
}
void operator+=(std::vector<double>& v1, const std::vector<double>& v2) {
  for (size_t i = 0; i < v1.size(); ++i) v1[i] += v2[i];
}
void operator-=(std::vector<double>& v1, const std::vector<double>& v2) {
  for (size_t i = 0; i < v1.size(); ++i) v1[i] -= v2[i];
}
void operator/=(std::vector<double>& v1, const std::vector<double>& v2) {
  for (size_t i = 0; i < v1.size(); ++i) v1[i] /= v2[i];
}
void operator*=(std::vector<double>& v1, const double& a) {
  for (double& x : v1) x *= a;
}
void operator*=(std::vector<double>& v1, const std::vector<double>& v2) {
  for (size_t i = 0; i < v1.size(); ++i) v1[i] *= v2[i];
}
void operator/=(std::vector<double>& v1, const double& a) {
  for (double& x : v1) x /= a;
}

std::ostream& operator<<(std::ostream& os, const std::vector<double>& v) {
  for (size_t i = 0; i < v.size(); ++i) os << v[i] << (i + 1 < v.size() ? " " : "");
  return os;
}

double norm_squared(const std::vector<double>& v) {
  double s = 0.0;
  for (double x : v) s += x * x;
  return s;
}
double norm(const std::vector<double>& v) { return std::sqrt(norm_squared(v)); }
void normalize(std::vector<double>* v) {
  const double n = norm(*v);
  if (n > 1e-16) *v /= n;
}
std::vector<double> normalize(std::vector<double>& v) {
  std::vector<double> r = v;
  normalize(&r);
  return r;
}
double maxabs(const std::vector<double>& v) {
  double m = 0.0;
  for (double x : v) m = std::max(m, std::fabs(x));
  return m;
}
double max_abs_difference(const std::vector<double>& v1, const std::vector<double>& v2) {
  double m = 0.0;
  for (size_t i = 0; i < v1.size(); ++i) m = std::max(m, std::fabs(v1[i] - v2[i]));
  return m;
}
std::vector<double> exponentiate(const std::vector<double>& e) {
  return each(e, [](double a) { return std::exp(a); });
}
void randomize(std::vector<double>* v) {
  static std::mt19937_64 gen(0);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  for (double& x : *v) x = u(gen);
}

void axpy(std::vector<double>* y, double& a, std::vector<double>& x) {
  for (size_t i = 0; i < y->size(); ++i) (*y)[i] += a * x[i];
}
void axpy(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x) {
  for (size_t i = 0; i < y->size(); ++i) (*y)[i] += a[i] * x[i];
}
void naxpy(std::vector<double>* y, double& a, std::vector<double>& x) {
  for (size_t i = 0; i < y->size(); ++i) (*y)[i] -= a * x[i];
}
void naxpy(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x) {
  for (size_t i = 0; i < y->size(); ++i) (*y)[i] -= a[i] * x[i];
}

void csv_to_vector(const char* buffer, std::vector<double>& vect) {
  vect.clear();
  const char* p = buffer;
  while (*p) {
    char* end = nullptr;
    const double d = std::strtod(p, &end);
    if (end == p) {
      ++p;
      continue;
    }
    vect.push_back(d);
    p = end;
  }
}
// The values as "%.7e" separated by commas (BioFVM_vector.cpp:313-364).
namespace {
size_t csv_write(const std::vector<double>& vect, char* out) {
  size_t pos = 0;
  for (size_t i = 0; i < vect.size(); ++i)
    pos += (size_t)std::sprintf(out + pos, i + 1 < vect.size() ? "%.7e," : "%.7e", vect[i]);
  out[pos] = '\0';
  return pos;
}
// room for one "%.7e," value: sign, digit, point, 7 digits, e, sign, up to 3
// exponent digits, comma
constexpr size_t kCsvDatum = 16;
}  // namespace

char* vector_to_csv(const std::vector<double>& vect) {
  char* out = new char[kCsvDatum * vect.size() + 1];
  csv_write(vect, out);
  return out;
}

void vector_to_csv_safe(const std::vector<double>& vect, char*& buffer) {
  delete[] buffer;
  buffer = new char[kCsvDatum * vect.size() + 1];
  csv_write(vect, buffer);
}

void vector_to_csv(const std::vector<double>& vect, char*& buffer) { csv_write(vect, buffer); }

// ---- fused elementwise updates (declared by BioFVM_vector.h:97-106) -------

void axpy_div(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x,
              std::vector<double>& d) {
  std::vector<double>& Y = *y;
  for (size_t i = 0; i < Y.size(); ++i) {
    Y[i] += a[i] * x[i];
    Y[i] /= d[i];
  }
}

void double_axpy(std::vector<double>* y, std::vector<double>& a1, std::vector<double>& a2,
                 std::vector<double>& x1, std::vector<double>& x2) {
  std::vector<double>& Y = *y;
  for (size_t i = 0; i < Y.size(); ++i) {
    Y[i] += a1[i] * x1[i];
    Y[i] += a2[i] * x2[i];
  }
}

void double_axpy(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x1,
                 std::vector<double>& x2) {
  std::vector<double>& Y = *y;
  for (size_t i = 0; i < Y.size(); ++i) Y[i] += a[i] * (x1[i] + x2[i]);
}

void double_axpy_div(std::vector<double>* y, std::vector<double>& a, std::vector<double>& x1,
                     std::vector<double>& x2, std::vector<double>& d) {
  double_axpy(y, a, x1, x2);
  std::vector<double>& Y = *y;
  for (size_t i = 0; i < Y.size(); ++i) Y[i] /= d[i];
}

void double_axpy_div(std::vector<double>* y, std::vector<double>& a1, std::vector<double>& a2,
                     std::vector<double>& x1, std::vector<double>& x2, std::vector<double>& d) {
  double_axpy(y, a1, a2, x1, x2);
  std::vector<double>& Y = *y;
  for (size_t i = 0; i < Y.size(); ++i) Y[i] /= d[i];
}

// ---- stopwatch (wall time) ----------------------------------------------

namespace {
using clk = std::chrono::steady_clock;
clk::time_point t_tic, t_toc, t_run0, t_run1;
double t_total = 0.0;
}  // namespace

void TIC(void) { t_tic = clk::now(); }
void TOC(void) {
  t_toc = clk::now();
  t_total += std::chrono::duration<double>(t_toc - t_tic).count();
}
void RUNTIME_TIC(void) { t_run0 = clk::now(); }
void RUNTIME_TOC(void) { t_run1 = clk::now(); }
double stopwatch_value(void) { return std::chrono::duration<double>(t_toc - t_tic).count(); }
double runtime_stopwatch_value(void) {
  return std::chrono::duration<double>(t_run1 - t_run0).count();
}
double total_stopwatch_time(void) { return t_total; }
std::string format_stopwatch_value(double d) {
  const int days = (int)(d / 86400.0);
  d -= days * 86400.0;
  const int hours = (int)(d / 3600.0);
  d -= hours * 3600.0;
  const int minutes = (int)(d / 60.0);
  d -= minutes * 60.0;
  std::ostringstream os;
  os << days << " days, " << hours << " hours, " << minutes << " minutes, and " << d
     << " seconds ";
  return os.str();
}
void display_stopwatch_value(std::ostream& os, double dIn) { os << format_stopwatch_value(dIn); }

// ---- MATLAB Level 4 (column-major doubles, 20-byte header) ---------------

namespace {
struct Mat4Header {
  int32_t type;  // 0: little-endian, double, full, real
  int32_t rows;
  int32_t cols;
  int32_t imag;
  int32_t name_len;
};
}  // namespace

FILE* write_matlab_header(int rows, int cols, std::string filename, std::string variable_name) {
  FILE* fp = std::fopen(filename.c_str(), "wb");
  if (!fp) {
    std::cout << "Error: could not open file " << filename << "!" << std::endl;
    return nullptr;
  }
  Mat4Header h{0, rows, cols, 0, (int32_t)variable_name.size() + 1};
  std::fwrite(&h, sizeof(h), 1, fp);
  std::fwrite(variable_name.c_str(), 1, variable_name.size() + 1, fp);
  return fp;
}

FILE* read_matlab_header(int* rows, int* cols, std::string filename) {
  FILE* fp = std::fopen(filename.c_str(), "rb");
  if (!fp) {
    std::cout << "Error: could not open file " << filename << "!" << std::endl;
    return nullptr;
  }
  Mat4Header h;
  if (std::fread(&h, sizeof(h), 1, fp) != 1 || h.type != 0 || h.name_len <= 0) {
    std::fclose(fp);
    return nullptr;
  }
  std::vector<char> name(h.name_len);
  if (std::fread(name.data(), 1, name.size(), fp) != name.size()) {
    std::fclose(fp);
    return nullptr;
  }
  *rows = h.rows;
  *cols = h.cols;
  return fp;
}

std::vector<std::vector<double> > read_matlab(std::string filename) {
  int rows = 0, cols = 0;
  std::vector<std::vector<double> > out;
  FILE* fp = read_matlab_header(&rows, &cols, filename);
  if (!fp) return out;
  // stored column-major: one entry per column of `rows` values
  out.assign(cols, std::vector<double>(rows));
  for (int c = 0; c < cols; ++c)
    if (std::fread(out[c].data(), sizeof(double), rows, fp) != (size_t)rows) {
      out.clear();
      break;
    }
  std::fclose(fp);
  return out;
}

bool write_matlab(std::vector<std::vector<double> >& input, std::string filename) {
  const int cols = (int)input.size();
  const int rows = cols ? (int)input[0].size() : 0;
  FILE* fp = write_matlab_header(rows, cols, filename, "input");
  if (!fp) return false;
  for (auto& col : input) std::fwrite(col.data(), sizeof(double), col.size(), fp);
  std::fclose(fp);
  return true;
}

}  // namespace BioFVM
