// HeisenbergHamiltonian of the reference
// (src/models/headers/HeisenbergHamiltonian.h:39-60): the spin-1/2 XYZ chain
// H = sum (Jx Sx Sx + Jy Sy Sy + Jz Sz Sz) + sum (hx Sx + hy Sy + hz Sz) +
// offset, MPO bond 5, built by the library (mpsgpu_mpo_heisenberg) with the
// reference's tables.  Uniform couplings, d = 2, no Sz-target penalty.
#pragma once

#include "MPO.h"
#include "mwArray.h"

class HeisenbergHamiltonian {
 public:
  HeisenbergHamiltonian(int L, double Jx, double Jy, double Jz, double h, int d = 2, double offset = 0.,
                        int Star = 0, double penalty = 0.);
  HeisenbergHamiltonian(int L, double Jx, double Jy, double Jz, double hx, double hy, double hz, int d = 2,
                        double offset = 0., int Star = 0, double penalty = 0.);
  ~HeisenbergHamiltonian() {}
  const MPO& getHMPO() const { return hamil; }

 private:
  void build(int L, double Jx, double Jy, double Jz, double hx, double hy, double hz, int d, double offset,
             double penalty);
  MPO hamil;
};
