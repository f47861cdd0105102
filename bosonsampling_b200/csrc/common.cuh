// Shared device helpers for libbsmpo: FP64 complex arithmetic and launch checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define BSMPO_DEV __device__ __forceinline__

struct cplx {
  double x, y;
};

BSMPO_DEV cplx cmake(double r, double i) { return cplx{r, i}; }
BSMPO_DEV cplx cadd(cplx a, cplx b) { return cplx{a.x + b.x, a.y + b.y}; }
BSMPO_DEV cplx csub(cplx a, cplx b) { return cplx{a.x - b.x, a.y - b.y}; }
BSMPO_DEV cplx cmul(cplx a, cplx b) { return cplx{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
// a * conj(b)
BSMPO_DEV cplx cmulc(cplx a, cplx b) { return cplx{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y}; }
// conj(a) * b
BSMPO_DEV cplx ccmul(cplx a, cplx b) { return cplx{a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x}; }
BSMPO_DEV cplx cconj(cplx a) { return cplx{a.x, -a.y}; }
BSMPO_DEV cplx cscale(cplx a, double s) { return cplx{a.x * s, a.y * s}; }
BSMPO_DEV double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }
// acc += a * b (4 FMA)
BSMPO_DEV void cfma(cplx& acc, cplx a, cplx b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
BSMPO_DEV void ccfma(cplx& acc, cplx a, cplx b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}

BSMPO_DEV cplx ldc(const cplx* p) {
  double2 v = *reinterpret_cast<const double2*>(p);
  return cplx{v.x, v.y};
}
BSMPO_DEV void stc(cplx* p, cplx v) { *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y); }

static inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
