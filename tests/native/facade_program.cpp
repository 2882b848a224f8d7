// A program written against the reference's C++ API (Contractor, MPS, MPO,
// IsingHamiltonian, SchwingerHamiltonian), linked to the facade in
// mpsdyn_b200/cpp: the same calls as programs/ising/testIsing.cpp and
// schwingerExc-style runs, on seeded inputs written by the test.  Prints
// one JSON line with the results.
//
//   facade_program <gs_init.mps> <exc_init0.mps> <exc_init1.mps> <trunc.mps> <tmpdir>
#include <cstdio>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "Contractor.h"
#include "IsingHamiltonian.h"
#include "MPS.h"
#include "SchwingerHamiltonian.h"
#include "mwArray.h"

static std::string num(double x) {
  std::ostringstream os;
  os << std::setprecision(17) << x;
  return os.str();
}

int main(int argc, const char* argv[]) {
  if (argc < 6) return 2;
  Contractor& contractor = Contractor::theContractor();
  contractor.setConvTol(1e-10);
  std::vector<std::string> out;

  // ground state: Ising L=10, D=8, seed-0 initial state (file)
  {
    IsingHamiltonian hamI(10, 2, 1., 1., 0.);
    const MPO& hamil = hamI.getHMPO(0.);
    MPS gs;
    gs.importMPS(argv[1]);
    double E0 = 0.;
    contractor.findGroundState(hamil, 8, &E0, gs);
    out.push_back("\"gs_E0\": " + num(E0));
    out.push_back("\"gs_norm\": " + num(real(contractor.contract(gs, gs))));
    out.push_back("\"gs_H\": " + num(real(contractor.contract(gs, hamil, gs))));
    out.push_back("\"gs_H2\": " + num(real(contractor.contract2(hamil, gs))));
    out.push_back("\"gs_entropy\": " + num(contractor.getEntropy(gs, 5)));
    // export / import round trip keeps the state
    std::string fn = std::string(argv[5]) + "/gs_out.mps";
    gs.exportMPS(fn.c_str());
    MPS back;
    back.importMPS(fn.c_str());
    out.push_back("\"roundtrip_overlap\": " + num(abs(contractor.contract(back, gs))));
    out.push_back("\"site3_dims\": [" + std::to_string(gs.getA(3).getd()) + ", " +
                  std::to_string(gs.getA(3).getDl()) + ", " + std::to_string(gs.getA(3).getDr()) + "]");
  }

  // imaginary-time evolution as in testIsing.cpp: MPS(L, D, d), getUMPO,
  // optimize, gaugeCond('R', true), energy
  {
    const int L = 10, D = 6;
    IsingHamiltonian hamI(L, 2, 1., 1., 0.);
    const MPO& hamil = hamI.getHMPO(0.);
    MPO evol(L);
    hamI.getUMPO(evol, 0.05, 0., true, 2);
    MPS imaGS(L, D, 2);
    std::string es;
    for (int cnt = 0; cnt < 20; cnt++) {
      MPS aux(imaGS);
      contractor.optimize(evol, aux, imaGS, D);
      imaGS.gaugeCond('R', true);
      es += (cnt ? ", " : "") + num(real(contractor.contract(imaGS, hamil, imaGS)));
    }
    out.push_back("\"imag_energies\": [" + es + "]");
  }

  // excited state: Ising L=10, D=16, seeds 1 and 11 (files)
  {
    IsingHamiltonian hamI(10, 2, 1., 1., 0.);
    const MPO& hamil = hamI.getHMPO(0.);
    MPS g0, g1;
    g0.importMPS(argv[2]);
    g1.importMPS(argv[3]);
    double E0 = 0., E1 = 0.;
    contractor.findGroundState(hamil, 16, &E0, g0);
    std::vector<MPS*> levels(1, &g0);
    contractor.findNextExcitedState(hamil, 16, levels, &E1, g1);
    out.push_back("\"exc_E0\": " + num(E0));
    out.push_back("\"exc_E1\": " + num(E1));
  }

  // SVD cut MPS(mps, D) of a bond-16 state to D=5 (file); the norm is kept
  {
    MPS big;
    big.importMPS(argv[4]);
    MPS cut(big, 5);
    out.push_back("\"trunc_bond\": " + std::to_string(cut.getBond()));
    out.push_back("\"trunc_overlap\": " + num(real(contractor.contract(cut, big))));
    out.push_back("\"trunc_norm\": " + num(real(contractor.contract(cut, cut))));
  }

  // the same ground state in mixed precision (facade extension setPrecision)
  {
    IsingHamiltonian hamI(10, 2, 1., 1., 0.);
    const MPO& hamil = hamI.getHMPO(0.);
    MPS gs;
    gs.importMPS(argv[1]);
    double E0 = 0.;
    contractor.setPrecision(1);
    contractor.findGroundState(hamil, 8, &E0, gs);
    contractor.setPrecision(0);
    out.push_back("\"mixed_gs_E0\": " + num(E0));
  }

  // Schwinger MPO built by the library: energy of the product state
  {
    SchwingerHamiltonian hs(16, 2.5, 100., 0., 0.);
    MPS p(16, 1, 2);
    out.push_back("\"schwinger_product_energy\": " + num(real(contractor.contract(p, hs.getHMPO(), p))));
  }

  std::string line = "{";
  for (size_t i = 0; i < out.size(); i++) line += (i ? ", " : "") + out[i];
  line += "}";
  std::printf("%s\n", line.c_str());
  return 0;
}
