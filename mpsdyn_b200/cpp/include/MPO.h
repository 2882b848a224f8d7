// MPO of the reference (src/core/headers/MPO.h:33): a row of Operators,
// stored by pointer with per-slot ownership (setOp(pos, op, myop)).  The
// device copy that the sweep uses is uploaded on first use and again after
// any setOp.
#pragma once

#include <vector>

#include "Operator.h"

struct mpsgpu_mpo;

class MPO {
 public:
  MPO() {}
  explicit MPO(int length) { initLength(length); }
  MPO(const MPO& other);
  MPO& operator=(const MPO& other);
  virtual ~MPO();

  void initLength(int len);
  void clear();
  int getLength() const { return length_; }
  const Operator& getOp(int pos) const;
  const mwArray getOpData(int pos) const { return getOp(pos).getFullData(); }
  bool isEmpty(int pos) const { return ops_[pos] == nullptr; }
  void setOp(int pos, const Operator* op, bool myop = false);
  // physical (output) dimension of every site
  const std::vector<int> getDimensions() const;
  // binary MPO file of the reference (MPO.cpp:214-231, 291-312)
  void saveMPO(const char* filename) const;
  void loadMPO(const char* filename);

  // The device copy (uploaded on demand), for the Contractor and MPS.
  mpsgpu_mpo* device() const;
  // Take over an MPO built by the library: host Operators are downloaded
  // from it and the handle becomes this MPO's device copy.
  void setFromDevice(mpsgpu_mpo* h);

 private:
  void drop_device() const;
  int length_ = 0;
  std::vector<const Operator*> ops_;
  std::vector<bool> own_;
  mutable mpsgpu_mpo* dev_ = nullptr;
};
