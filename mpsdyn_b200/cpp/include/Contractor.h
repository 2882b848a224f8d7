// Contractor of the reference (src/core/headers/Contractor.h:46): the
// singleton that runs the sweeps.  Every call forwards to the C ABI of
// libmpsgpu on one device (MPSGPU_DEVICE, default 0); the MPS and MPO
// arguments stay on the device between calls.
//
// Errors: the reference prints a message and calls exit(code).  This
// facade throws MpsgpuException (with the library's status code and
// message) unless MPSDYN_STRICT_EXIT is defined when facade.cpp is built,
// in which case it prints the message and exits with 212 (energy increase,
// non-finite values, shapes) like the reference.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "MPO.h"
#include "MPS.h"
#include "mwArray.h"

struct mpsgpu_context;

enum EigenSolver { arpack = 0, fulleig, primme };

class MpsgpuException : public std::runtime_error {
 public:
  MpsgpuException(int status, const std::string& msg) : std::runtime_error(msg), status(status) {}
  int status;
};

class Contractor {
 public:
  static Contractor& theContractor();

  void setSVDTol(double value) { svdtol = value; }
  void setConvTol(double value) { convtol = value; }
  void setExcOrthTol(double value) { excorthtol = value; }
  void setEigTol(double value) { eigtol = value; }
  // every solver maps to the library's thick-restart Lanczos
  void setEigenSolver(EigenSolver solver_ = arpack) { solver = solver_; }
  double getConvTol() const { return convtol; }
  double getEigTol() const { return eigtol; }
  // Extension without a counterpart in the reference: 0 = complex FP64
  // throughout (default), 1 = mixed precision for findGroundState and
  // findNextExcitedState (split-precision products on the tensor cores until
  // the half-sweep energy settles, then FP64 to the convergence tolerance).
  void setPrecision(int value) { precision = value; }
  int getPrecision() const { return precision; }

  void findGroundState(const MPO& ops, int D, double* lambda, MPS& resultMPS, double offset = 0.,
                       int nrLocalEig = 1, const std::string& tmpfile = "", int freqSv = 200, bool useLM = false);
  void findNextExcitedState(const MPO& ops, int D, const std::vector<MPS*>& computedLevels, double* lambdak,
                            MPS& init, double offset = 0., int nrLocalEig = 1, const std::string& tmpfile = "",
                            int maxTime = 0, bool useLM = false);
  void optimize(const MPO& ops, const MPS& ket, MPS& init, int D = 0, double* errN = 0, double* errT = 0);
  // Contractor.h:133-140 of the reference
  void optimizeSum(std::vector<const MPS*> kets, std::vector<complex_t> beta, MPS& init, int D = 0);
  void optimizeMPS(const MPS& ket, MPS& init, int D = 0, double* err = 0);

  complex_t contract(const MPS& ket, const MPS& bra, char dir = 'L');
  complex_t contract(const MPS& ket, const MPO& ops, const MPS& bra);
  complex_t contract2(const MPO& ops, const MPS& ket);
  complex_t contract2(const MPS& bra, const MPO& ops, const MPS& ket);
  double getEntropy(const MPS& state, int len = 0);
  void getSchmidtValues(const MPS& state, std::vector<complex_t>& lambdas, int len = 0);

  // the library context used by every facade object
  mpsgpu_context* context();
  // status check used by the facade classes: throws (or exits, see above)
  static void check(int status, const char* what);

 private:
  Contractor();
  Contractor(const Contractor&) = delete;
  Contractor& operator=(const Contractor&) = delete;
  double svdtol = 1e-8, convtol = 1e-5, eigtol = 0., excorthtol = 0.;
  int precision = 0;
  EigenSolver solver = primme;
  mpsgpu_context* ctx_ = nullptr;
};
