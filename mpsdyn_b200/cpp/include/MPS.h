// MPS of the reference (src/core/headers/MPS.h:62), kept on the device.
// The tensors live in the library (mpsgpu_mps); getA returns host snapshots
// and setA writes through.  Copies are device copies.
#pragma once

#include <cstdint>
#include <iostream>
#include <ostream>
#include <vector>

#include "MPO.h"
#include "Site.h"
#include "mwArray.h"

struct mpsgpu_mps;

enum Gauge { gNone, gLeft, gRight, gBoth };

class MPS {
 public:
  MPS() {}
  // product state |0...0> with bonds (1, D, ..., D, 1) (MPS.cpp:15-35)
  MPS(int length, int bond, int d);
  MPS(const MPS& aMPS);
  // a copy cut to bond dimension `bond` (MPS.cpp:761-772)
  MPS(const MPS& aMPS, int bond);
  // ops applied to aMPS and cut to `bond` (MPS::approximate)
  MPS(const MPO& ops, const MPS& aMPS, int bond, char dir = 'D', char gauge = 'L');
  MPS& operator=(const MPS& aMPS);
  ~MPS();

  int getLength() const { return length_; }
  int getBond() const;
  bool isEmpty() const { return length_ == 0; }
  bool isGaugeL() const;
  bool isGaugeR() const;
  double getNormFact() const;
  void setNormFact(double value);

  const Site_t& getA(int k) const;
  void setA(int pos, const mwArray& data);

  // random sites, each right-gauged in turn (MPS.cpp:282-294); seeded by
  // setRandomSeed (default 0) for reproducible runs
  void setRandomState();
  static void setRandomSeed(uint64_t seed);
  void gaugeCond(char dir, bool normalize = false, int cutD = 0);
  void increaseBondDimension(int D);
  void applyExactly(const MPO& ops, bool dagger = false, char gaugedir = 'L');
  void approximate(const MPO& ops, const MPS& aMPS, int D, char dir = 'D', char gaugeDir = 'L');

  // binary formats of MPS::exportMPS / importMPS (MPS.cpp:442-509)
  void exportMPS(const char* filename) const;
  void importMPS(const char* filename);

  friend std::ostream& operator<<(std::ostream& os, const MPS& mps);

  // library handle, for the Contractor
  mpsgpu_mps* device() const { return h_; }
  void adopt(mpsgpu_mps* h);           // replace the tensors by h (owned from now on)
  void changed() const { cache_ok_ = false; }  // the device tensors were modified

 private:
  void release();
  void sync_cache() const;
  int length_ = 0;
  mpsgpu_mps* h_ = nullptr;
  mutable std::vector<Site> cache_;
  mutable bool cache_ok_ = false;
};
