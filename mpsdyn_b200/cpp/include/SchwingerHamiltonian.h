// SchwingerHamiltonian of the reference
// (src/models/headers/SchwingerHamiltonian.h:13): spin formulation of the
// lattice Schwinger model, MPO bond 5, built by the library
// (mpsgpu_mpo_schwinger) with the reference's tables.  offset = nu = 0 and
// y = 1 only.
#pragma once

#include "MPO.h"
#include "mwArray.h"

class SchwingerHamiltonian {
 public:
  SchwingerHamiltonian(int N, double mu, double x, double l0, double alpha, double offset = 0, double nu = 0.,
                       double y = 1.);
  ~SchwingerHamiltonian() {}
  const MPO& getHMPO() const { return hamil; }

 private:
  MPO hamil;
};
