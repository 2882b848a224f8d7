// Operator of the reference (src/core/headers/Operator.h:24): one MPO
// tensor W(du, Dl, dd, Dr), column-major.
#pragma once

#include "mwArray.h"

class Operator {
 public:
  explicit Operator(const mwArray& data) : data_(data) {}
  const mwArray& getFullData() const { return data_; }
  const shrt::Indices& getDimensions() const { return data_.getDimensions(); }
  int getDimension(int k) const { return data_.getDimension(k); }

 private:
  mwArray data_;
};
