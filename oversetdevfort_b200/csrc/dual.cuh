// Forward-mode dual number (value + one tangent) for the adjoint of the
// element residual: the element routines of assemble.cu are instantiated on
// it, so one evaluation gives the residual rows and their derivative along
// one seeded input.  Comparisons and branches use the value, as the FP64
// routine does; conversion to double (explicit) drops the tangent.
#pragma once

struct Dual {
  double v, d;
  __host__ __device__ Dual() : v(0.0), d(0.0) {}
  __host__ __device__ Dual(double x) : v(x), d(0.0) {}
  __host__ __device__ Dual(double x, double t) : v(x), d(t) {}
  __host__ __device__ explicit operator double() const { return v; }
  __host__ __device__ explicit operator float() const { return (float)v; }
  __host__ __device__ Dual& operator+=(const Dual& b) { v += b.v; d += b.d; return *this; }
  __host__ __device__ Dual& operator-=(const Dual& b) { v -= b.v; d -= b.d; return *this; }
  __host__ __device__ Dual& operator*=(const Dual& b) { d = d * b.v + v * b.d; v *= b.v; return *this; }
  __host__ __device__ Dual& operator/=(const Dual& b) {
    const double q = v / b.v;
    d = (d - q * b.d) / b.v;
    v = q;
    return *this;
  }
};

__host__ __device__ inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
__host__ __device__ inline Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
__host__ __device__ inline Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
__host__ __device__ inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__host__ __device__ inline Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__host__ __device__ inline Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
__host__ __device__ inline Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
__host__ __device__ inline Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
__host__ __device__ inline Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
__host__ __device__ inline Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
__host__ __device__ inline Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
__host__ __device__ inline Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
__host__ __device__ inline Dual operator/(double a, const Dual& b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}

__host__ __device__ inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
__host__ __device__ inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
__host__ __device__ inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
__host__ __device__ inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
__host__ __device__ inline bool operator<(const Dual& a, double b) { return a.v < b; }
__host__ __device__ inline bool operator>(const Dual& a, double b) { return a.v > b; }
__host__ __device__ inline bool operator<=(const Dual& a, double b) { return a.v <= b; }
__host__ __device__ inline bool operator>=(const Dual& a, double b) { return a.v >= b; }

// d sqrt(x) = dx / (2 sqrt(x)); d |x| = sign(x) dx (0 at 0)
__device__ inline Dual sqrt(const Dual& a) {
  const double s = ::sqrt(a.v);
  return Dual(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
}
__device__ inline Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : (a.v > 0.0 ? a : Dual(0.0, 0.0)); }
__device__ inline bool isfinite(const Dual& a) { return ::isfinite(a.v) && ::isfinite(a.d); }
