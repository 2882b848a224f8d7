// complex_t of the reference (src/wrapper/complex.h:22-26): a plain struct of
// two doubles, with the same free functions, so code written against the
// reference's scalar type compiles unchanged.  Layout-compatible with the
// interleaved complex128 the C ABI takes.
#pragma once

#include <iostream>

typedef struct complex_t {
  double re;
  double im;
} complex_t;

complex_t operator+(complex_t a, complex_t b);
complex_t& operator+=(complex_t& a, complex_t b);
complex_t operator-(complex_t a);
complex_t operator-(complex_t a, complex_t b);
complex_t operator*(complex_t a, complex_t b);
complex_t& operator*=(complex_t& a, complex_t b);
complex_t operator*(double x, complex_t a);
complex_t operator*(complex_t a, double x);
complex_t operator/(complex_t a, complex_t b);
complex_t operator/(complex_t a, double x);
complex_t conjugate(complex_t a);
bool operator==(complex_t a, complex_t b);
bool operator!=(complex_t a, complex_t b);
std::ostream& operator<<(std::ostream& os, complex_t c);
double abs(complex_t c);
double phase(complex_t c);
double real(complex_t c);
double imag(complex_t c);
complex_t sqrt(complex_t c);
complex_t exp(complex_t c);

static const complex_t ONE_c = {1., 0.};
static const complex_t ZERO_c = {0., 0.};
static const complex_t I_c = {0., 1.};
