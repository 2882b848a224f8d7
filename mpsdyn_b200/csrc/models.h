// MPO builders of the two model families on the hot path, producing host
// tensors in the reference Operator layout W(du, Dl, dd, Dr), column-major
// complex128.  They are the inputs of the sweeps (built once, uploaded).
#pragma once

#include <array>
#include <complex>
#include <vector>

namespace mpsgpu {

struct HostMPO {
  std::vector<std::array<int, 4>> dims;             // (du, Dl, dd, Dr) per site
  std::vector<std::vector<std::complex<double>>> W;  // column-major tensors
};

// IsingHamiltonian::setHMPO (models/cpp/IsingHamiltonian.cpp:70-121):
// H = J sum sz_i sz_i+1 + g sum sx_i + h sum sz_i (+ K, spread over the chain).
HostMPO ising_hmpo(int L, double J, double g, double h, double K = 0.0);
// IsingHamiltonian::getUMPO with orderT = 2 (IsingHamiltonian.cpp:131-148,
// 169-244): second-order Trotter exp(eps H) with eps = -delta (imaginary
// time) or -i delta (real time); MPO bond 2.
HostMPO ising_umpo(int L, double J, double g, double h, double delta, bool imag);
// SchwingerHamiltonian::initHMPO (models/cpp/SchwingerHamiltonian.cpp:43-121):
// spin formulation, staggered fermions, gauge field integrated out, MPO bond 5.
HostMPO schwinger_hmpo(int N, double mu, double x, double l0, double alpha, double offset = 0.0,
                       double nu = 0.0, double y = 1.0);
// HeisenbergHamiltonian::initHMPO (models/cpp/HeisenbergHamiltonian.cpp:266-331)
// with uniform couplings, d = 2 and no Sz penalty: H = sum (Jx SxSx + Jy SySy
// + Jz SzSz) + sum (hx Sx + hy Sy + hz Sz) + offset, S = sigma / 2, bond 5.
HostMPO heisenberg_hmpo(int L, double Jx, double Jy, double Jz, double hx, double hy, double hz,
                        double offset = 0.0);
// BoseHubbardHamiltonian(L, N, t, U, Ntarget, penaltyN, V) and its initZ /
// initHMPO (models/cpp/BoseHubbardHamiltonian.cpp:7-17, 73-160): occupation
// cut at N (d = N + 1), H = -t sum (b+_i b_i+1 + h.c.) + U/2 sum n_i (n_i - 1)
// + V sum n_i + penaltyN (sum n_i - Ntarget)^2, bond 5.  t >= 0 (the
// reference's uniform-coupling form takes sqrt(t) on both sides of a hop).
HostMPO bosehubbard_hmpo(int L, int N, double t, double U, int Ntarget, double penN, double V = 0.0);

}  // namespace mpsgpu
