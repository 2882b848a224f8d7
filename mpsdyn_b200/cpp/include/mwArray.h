// mwArray of the reference (src/wrapper/mwArray.h:23): a dense complex array,
// column-major, with the reference's dimension bookkeeping.  In this
// library the arrays live on the host and are only the exchange format of
// the drop-in API (MPO and MPS tensors in and out); the contractions of the
// sweep run on the device behind the C ABI (include/mpsgpu.h).
#pragma once

#include <cmath>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "Indices.h"
#include "complex_t.h"

// The reference's headers open namespace std for the programs that include
// them (src/core/headers/Site.h:27 and others); programs written against
// them rely on it.
using namespace std;

class mwArray {
 public:
  mwArray() {}
  explicit mwArray(const shrt::Indices& dims);                        // zero filled
  mwArray(const shrt::Indices& dims, const complex_t* values);        // column-major copy
  mwArray(const shrt::Indices& dims, const double* values);           // interleaved re, im
  mwArray(complex_t scalar);

  int getRank() const { return (int)dims_.size(); }
  int getDimension(int k) const { return dims_[k]; }
  const shrt::Indices& getDimensions() const { return dims_; }
  int getNrComponents() const { return (int)data_.size(); }
  bool isScalar() const { return data_.size() == 1; }
  bool isEmpty() const { return data_.empty(); }

  complex_t getElement(int idx) const { return data_[idx]; }
  complex_t getElement(const shrt::Indices& idx) const { return data_[offset(idx)]; }
  void setElement(complex_t v, int idx) { data_[idx] = v; }
  void setElement(complex_t v, const shrt::Indices& idx) { data_[offset(idx)] = v; }
  void setElement(double re, double im, const shrt::Indices& idx) { data_[offset(idx)] = complex_t{re, im}; }

  // Same number of elements; one entry may be -1 (inferred).
  void reshape(const shrt::Indices& dims);
  // New dimensions; entries inside both boxes are kept, the rest is zero.
  void resize(const shrt::Indices& dims);
  // order is 1-based like the reference's Indices(2,1,3); optional conjugation.
  void permute(const shrt::Indices& order, bool conjugate = false);
  void conjugate();
  void transpose(bool conjugate = false);  // rank 2
  void Hconjugate() { transpose(true); }
  void fillWithZero();
  void clear() { dims_.clear(); data_.clear(); }
  // *this = *this . rhs and lhs . *this (rank 2 matrix products)
  void multiplyRight(const mwArray& rhs);
  void multiplyLeft(const mwArray& lhs);

  mwArray operator*(const mwArray& rhs) const;  // matrix product (scalar operands scale)
  mwArray operator+(const mwArray& rhs) const;
  mwArray operator-(const mwArray& rhs) const;
  mwArray& operator*=(complex_t c);

  // Binary form of mwArray::save/load (src/wrapper/mwArray.cpp:382-442):
  // int rank, int dims[rank], then re, im of every element, column-major.
  void save(std::ostream& os) const;
  void load(std::istream& is);

  const complex_t* components() const { return data_.data(); }
  complex_t* components() { return data_.data(); }

  friend std::ostream& operator<<(std::ostream& os, const mwArray& a);

 private:
  long long offset(const shrt::Indices& idx) const;
  shrt::Indices dims_;
  std::vector<complex_t> data_;
};

mwArray operator*(complex_t c, const mwArray& a);
mwArray reshape(const mwArray& a, const shrt::Indices& dims);
mwArray permute(const mwArray& a, const shrt::Indices& order);
mwArray conjugate(const mwArray& a);
mwArray identityMatrix(int d);
