// IsingHamiltonian of the reference (src/models/headers/IsingHamiltonian.h:26):
// H = J sum sz sz + g sum sx + h sum sz on an open chain, its MPO (bond 3)
// and the second-order Trotter evolution MPO.  Built by the library
// (mpsgpu_mpo_ising / mpsgpu_mpo_ising_evolution) with the reference's
// coefficient tables; d = 2 and K = 0 only.
#pragma once

#include "MPO.h"
#include "mwArray.h"

class IsingHamiltonian {
 public:
  IsingHamiltonian(int N, int d, double J0, double g0, double h0 = 0., double K = 0.);
  virtual ~IsingHamiltonian() {}
  const MPO& getHMPO(double t);
  const MPO& getHMPO() const { return hamil; }
  // exp(-i delta H) (imag: exp(-delta H)); second order only (orderT = 2)
  void getUMPO(MPO& mpo, double delta, double t, bool imag = false, int orderT = 2, int nrOp = 0);

 private:
  int N, d;
  double J, g, h;
  MPO hamil;
};
