// Site of the reference (src/core/headers/Site.h:49): one MPS tensor
// A(d, Dl, Dr), column-major.  Here a host snapshot of a device-resident
// tensor, returned by MPS::getA.
#pragma once

#include "mwArray.h"

class Site {
 public:
  Site() {}
  explicit Site(const mwArray& A) : A_(A) {}
  const mwArray& getA() const { return A_; }
  int getd() const { return A_.getDimension(0); }
  int getDl() const { return A_.getDimension(1); }
  int getDr() const { return A_.getDimension(2); }
  const shrt::Indices& getDimensions() const { return A_.getDimensions(); }

 private:
  mwArray A_;
};

typedef Site Site_t;
