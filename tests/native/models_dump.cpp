// Prints the library's host-side Bose-Hubbard MPO (mpsdyn_b200/csrc/models.cpp)
// for the CPU tests: one line per site, "du Dl dd Dr" then the column-major
// entries as re im pairs with 17 significant digits.
//   models_dump L N t U Ntarget penN V
#include <cstdio>
#include <cstdlib>

#include "models.h"

int main(int argc, char** argv) {
  if (argc != 8) return 2;
  const mpsgpu::HostMPO m =
      mpsgpu::bosehubbard_hmpo(std::atoi(argv[1]), std::atoi(argv[2]), std::atof(argv[3]), std::atof(argv[4]),
                               std::atoi(argv[5]), std::atof(argv[6]), std::atof(argv[7]));
  for (size_t k = 0; k < m.W.size(); k++) {
    std::printf("%d %d %d %d", m.dims[k][0], m.dims[k][1], m.dims[k][2], m.dims[k][3]);
    for (const auto& z : m.W[k]) std::printf(" %.17g %.17g", z.real(), z.imag());
    std::printf("\n");
  }
  return 0;
}
