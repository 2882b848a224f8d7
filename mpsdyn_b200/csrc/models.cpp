// MPO builders (host side).  Each operator is assembled exactly as the
// reference assembles it: a coefficient tensor C(Dl, Dr, nops) contracted
// with the stack of single-site operators Z(nops, d, d), then reordered to
// W(du, Dl, dd, Dr) (IsingHamiltonian.cpp:111-116, SchwingerHamiltonian.cpp:114-118).
// Identical operators of the reference's shared middle sites are built once
// and copied.
#include "models.h"

#include <cmath>
#include <stdexcept>

namespace mpsgpu {

namespace {

typedef std::complex<double> cd;

// W[s', l, s, r] = sum_op C[l, r, op] Z[op][s', s]
std::vector<cd> contract_coeffs(const std::vector<cd>& C, int Dl, int Dr, int nops,
                                const std::vector<std::array<cd, 4>>& Z) {
  const int d = 2;
  std::vector<cd> W((size_t)d * Dl * d * Dr, cd(0, 0));
  for (int l = 0; l < Dl; l++)
    for (int r = 0; r < Dr; r++)
      for (int op = 0; op < nops; op++) {
        const cd c = C[l + Dl * (r + Dr * op)];
        if (c == cd(0, 0)) continue;
        for (int sp = 0; sp < d; sp++)
          for (int s = 0; s < d; s++)
            W[sp + d * (l + Dl * (s + d * r))] += c * Z[op][sp + d * s];
      }
  return W;
}

// column-major 2x2 matrices
const std::array<cd, 4> SIG0 = {cd(1, 0), cd(0, 0), cd(0, 0), cd(1, 0)};
const std::array<cd, 4> SIGX = {cd(0, 0), cd(1, 0), cd(1, 0), cd(0, 0)};
const std::array<cd, 4> SIGZ = {cd(1, 0), cd(0, 0), cd(0, 0), cd(-1, 0)};
// The Schwinger builder fills its sigma_y column-major from {0, -i, i, 0}
// (SchwingerHamiltonian.cpp:30-31), i.e. [[0, i], [-i, 0]].
const std::array<cd, 4> SIGY_SCHW = {cd(0, 0), cd(0, -1), cd(0, 1), cd(0, 0)};

}  // namespace

HostMPO ising_hmpo(int L, double J, double g, double h, double K) {
  if (L < 2) throw std::invalid_argument("ising_hmpo: L < 2");
  const std::vector<std::array<cd, 4>> Z = {SIG0, SIGZ, SIGX};
  const int D = 3;
  HostMPO m;
  for (int k = 0; k < L; k++) {
    if (k > 1 && k < L - 1) {
      m.dims.push_back(m.dims[k - 1]);
      m.W.push_back(m.W[k - 1]);
      continue;
    }
    const int Dl = k == 0 ? 1 : D, Dr = k == L - 1 ? 1 : D;
    std::vector<cd> C((size_t)Dl * Dr * 3, cd(0, 0));
    auto at = [&](int l, int r, int op) -> cd& { return C[l + Dl * (r + Dr * op)]; };
    const cd effJ = J < 0 ? cd(0, std::sqrt(std::fabs(J))) : cd(std::sqrt(J), 0);
    if (k != L - 1) at(0, 0, 0) = 1.0;
    if (k != 0) at(Dl - 1, Dr - 1, 0) = 1.0;
    at(0, Dr - 1, 2) = g;
    at(0, Dr - 1, 1) = h;
    at(0, Dr - 1, 0) = K / L;
    if (k != L - 1) at(0, 1, 1) = effJ;
    if (k != 0) at(1, Dr - 1, 1) = effJ;
    m.dims.push_back({2, Dl, 2, Dr});
    m.W.push_back(contract_coeffs(C, Dl, Dr, 3, Z));
  }
  return m;
}

namespace {

// isingU1MPO (IsingHamiltonian.cpp:203-218): exp(eps (g sx + h sz)) as a 2x2
std::array<cd, 4> ising_u1(cd eps, double g, double h) {
  const double nrm = std::sqrt(g * g + h * h);
  std::array<cd, 4> r;
  for (int i = 0; i < 4; i++) r[i] = std::cosh(nrm * eps) * SIG0[i];
  if (nrm != 0)
    for (int i = 0; i < 4; i++)
      r[i] += (h / nrm) * std::sinh(nrm * eps) * SIGZ[i] + (g / nrm) * std::sinh(nrm * eps) * SIGX[i];
  return r;
}

// isingU2MPO (IsingHamiltonian.cpp:169-201): exp(eps sz sz) split over bond 2
std::vector<cd> ising_u2(cd eps, int pos, int L, int& Dl, int& Dr) {
  const std::vector<std::array<cd, 4>> Z = {SIG0, SIGZ, SIGX};
  if (eps == cd(0, 0)) {
    Dl = Dr = 1;
    return std::vector<cd>(SIG0.begin(), SIG0.end());
  }
  const int D = 2;
  if (pos != 0 && pos != L - 1) {
    Dl = Dr = D;
    std::vector<cd> C((size_t)D * D * 3, cd(0, 0));
    auto at = [&](int l, int r, int op) -> cd& { return C[l + D * (r + D * op)]; };
    at(0, 0, 0) = std::cosh(eps);
    at(1, 1, 0) = std::sinh(eps);
    at(0, 1, 1) = std::sqrt(std::cosh(eps) * std::sinh(eps));
    at(1, 0, 1) = std::sqrt(std::cosh(eps) * std::sinh(eps));
    return contract_coeffs(C, Dl, Dr, 3, Z);
  }
  // edge: C(1, D, 3) reinterpreted as (Dl, Dr) = (1, D) or (D, 1)
  std::vector<cd> C((size_t)D * 3, cd(0, 0));
  C[0 + D * 0] = std::sqrt(std::cosh(eps));
  C[1 + D * 1] = std::sqrt(std::sinh(eps));
  if (pos == 0) { Dl = 1; Dr = D; }
  else { Dl = D; Dr = 1; }
  return contract_coeffs(C, Dl, Dr, 3, Z);
}

}  // namespace

HostMPO ising_umpo(int L, double J, double g, double h, double delta, bool imag) {
  if (L < 2) throw std::invalid_argument("ising_umpo: L < 2");
  const cd eps = imag ? cd(-delta, 0) : cd(0, -delta);
  HostMPO m;
  for (int k = 0; k < L; k++) {
    if (k > 1 && k < L - 1) {
      m.dims.push_back(m.dims[k - 1]);
      m.W.push_back(m.W[k - 1]);
      continue;
    }
    // constructU2T (IsingHamiltonian.cpp:220-244): U1(eps/2) . U2(J eps) . U1(eps/2)
    const std::array<cd, 4> U1 = ising_u1(0.5 * eps, g, h);
    int Dl, Dr;
    const std::vector<cd> U2 = ising_u2(J * eps, k, L, Dl, Dr);
    const int d = 2;
    std::vector<cd> W((size_t)d * Dl * d * Dr, cd(0, 0));
    for (int sp = 0; sp < d; sp++)
      for (int l = 0; l < Dl; l++)
        for (int s = 0; s < d; s++)
          for (int r = 0; r < Dr; r++) {
            cd acc(0, 0);
            for (int a = 0; a < d; a++)
              for (int b = 0; b < d; b++)
                acc += U1[sp + d * a] * U2[a + d * (l + Dl * (b + d * r))] * U1[b + d * s];
            W[sp + d * (l + Dl * (s + d * r))] = acc;
          }
    m.dims.push_back({d, Dl, d, Dr});
    m.W.push_back(W);
  }
  return m;
}

HostMPO schwinger_hmpo(int N, double mu, double x, double l0, double alpha, double offset, double nu,
                       double y) {
  if (N < 3) throw std::invalid_argument("schwinger_hmpo: N < 3");
  const std::vector<std::array<cd, 4>> Z = {SIG0, SIGX, SIGY_SCHW, SIGZ};
  const int D = 5;
  const double alpha_ = alpha + l0;
  std::vector<double> alphas(N), sumA(N, 0.0);
  for (int k = 0; k < N; k++) {
    const double signo = (k + 1) % 2 == 0 ? 1.0 : -1.0;
    alphas[k] = alpha_ - 0.25 * (1.0 - signo);
  }
  double tot = 0.0;
  for (int k = N - 2; k >= 0; k--) {
    tot += alphas[k];
    sumA[k] = tot;
  }
  const double gw = y;
  const double sx = std::sqrt(x / 2);
  HostMPO m;
  for (int k = 0; k < N; k++) {
    const int Dl = k == 0 ? 1 : D, Dr = k == N - 1 ? 1 : D;
    std::vector<cd> C((size_t)Dl * Dr * 4, cd(0, 0));
    auto at = [&](int l, int r, int op) -> cd& { return C[l + Dl * (r + Dr * op)]; };
    if (k != N - 1) at(0, 0, 0) = 1.0;
    if (k != 0) at(D - 1, Dr - 1, 0) = 1.0;
    if (k > 0 && k < N - 2) at(3, 3, 0) = 1.0;
    const double ak = alphas[k];
    const double signok = (k + 1) % 2 == 0 ? 1.0 : -1.0;
    if (k != N - 1) {
      at(0, Dr - 1, 0) = gw * ak * ak + (gw * (k + 1) / 4.0 + mu / 2.0 + nu / 2.0 + offset / N);
      at(0, Dr - 1, 3) = (signok * mu / 2.0 + nu / 2.0) + gw * sumA[k];
    } else {
      at(0, Dr - 1, 0) = mu / 2.0 + nu / 2.0 + offset / N;
      at(0, Dr - 1, 3) = signok * mu / 2.0 + nu / 2.0;
    }
    if (k != N - 1) {
      at(0, 1, 1) = sx;
      at(0, 2, 2) = sx;
      if (k < N - 2) at(0, 3, 3) = gw;
      if (k != 0) {
        at(1, 4, 1) = sx;
        at(2, 4, 2) = sx;
        at(3, 4, 3) = (N - k - 1) / 2.0;
      }
    } else {
      at(1, 0, 1) = sx;
      at(2, 0, 2) = sx;
    }
    m.dims.push_back({2, Dl, 2, Dr});
    m.W.push_back(contract_coeffs(C, Dl, Dr, 4, Z));
  }
  return m;
}

HostMPO heisenberg_hmpo(int L, double Jx, double Jy, double Jz, double hx, double hy, double hz, double offset) {
  if (L < 2) throw std::invalid_argument("heisenberg_hmpo: L < 2");
  // spin-1/2 operators: identity, S_x, S_y = [[0, -i/2], [i/2, 0]], S_z
  // (HeisenbergHamiltonian.cpp:266-284 fills them column-major)
  const std::array<cd, 4> S0 = SIG0;
  const std::array<cd, 4> SX = {cd(0, 0), cd(0.5, 0), cd(0.5, 0), cd(0, 0)};
  const std::array<cd, 4> SY = {cd(0, 0), cd(0, 0.5), cd(0, -0.5), cd(0, 0)};
  const std::array<cd, 4> SZ = {cd(0.5, 0), cd(0, 0), cd(0, 0), cd(-0.5, 0)};
  const std::vector<std::array<cd, 4>> Z = {S0, SX, SY, SZ};
  const int D = 5;
  HostMPO m;
  for (int k = 0; k < L; k++) {
    const int Dl = k == 0 ? 1 : D, Dr = k == L - 1 ? 1 : D;
    std::vector<cd> C((size_t)Dl * Dr * 4, cd(0, 0));
    auto at = [&](int l, int r, int op) -> cd& { return C[l + Dl * (r + Dr * op)]; };
    if (k != L - 1) {
      at(0, 0, 0) = 1.0;
      at(0, 1, 1) = Jx;
      at(0, 2, 2) = Jy;
      at(0, 3, 3) = Jz;
    }
    if (k != 0) {
      at(Dl - 1, Dr - 1, 0) = 1.0;
      at(1, Dr - 1, 1) = 1.0;
      at(2, Dr - 1, 2) = 1.0;
      at(3, Dr - 1, 3) = 1.0;
    }
    at(0, Dr - 1, 3) = hz;
    if (hx != 0) at(0, Dr - 1, 1) = hx;
    if (hy != 0) at(0, Dr - 1, 2) = hy;
    if (offset != 0) at(0, Dr - 1, 0) = offset / L;
    m.dims.push_back({2, Dl, 2, Dr});
    m.W.push_back(contract_coeffs(C, Dl, Dr, 4, Z));
  }
  return m;
}

namespace {

// W[s', l, s, r] = sum_op C[l, r, op] Z[op][s', s] for a physical dimension d
// (Z[op] column-major d x d); the ops are summed in order, as the
// reference's C * Z product does.
std::vector<cd> contract_coeffs_d(const std::vector<cd>& C, int Dl, int Dr, int nops,
                                  const std::vector<std::vector<cd>>& Z, int d) {
  std::vector<cd> W((size_t)d * Dl * d * Dr, cd(0, 0));
  for (int l = 0; l < Dl; l++)
    for (int r = 0; r < Dr; r++)
      for (int op = 0; op < nops; op++) {
        const cd c = C[l + Dl * (r + Dr * op)];
        if (c == cd(0, 0)) continue;
        for (int sp = 0; sp < d; sp++)
          for (int s = 0; s < d; s++) W[sp + d * (l + Dl * (s + d * r))] += c * Z[op][sp + d * s];
      }
  return W;
}

}  // namespace

HostMPO bosehubbard_hmpo(int L, int N, double t, double U, int Ntarget, double penN, double V) {
  if (L < 2) throw std::invalid_argument("bosehubbard_hmpo: L < 2");
  if (N < 1) throw std::invalid_argument("bosehubbard_hmpo: N < 1");
  if (!(t >= 0)) throw std::invalid_argument("bosehubbard_hmpo: t < 0");
  const int d = N + 1;
  // local operators (initZ): 1, n(n-1), b+, b, n, n^2; entry (i1, i2) = <i1|op|i2>
  std::vector<std::vector<cd>> Z(6, std::vector<cd>((size_t)d * d, cd(0, 0)));
  for (int i = 0; i < d; i++) {
    Z[0][i + d * i] = 1.0;
    Z[1][i + d * i] = (double)(i * (i - 1));
    if (i > 0) Z[2][i + d * (i - 1)] = std::sqrt((double)i);
    if (i < N) Z[3][i + d * (i + 1)] = std::sqrt((double)(i + 1));
    Z[4][i + d * i] = (double)i;
    Z[5][i + d * i] = (double)(i * i);
  }
  const double half_u = 0.5 * U;  // the reference keeps U/2
  const cd hop(0.0, std::sqrt(t));  // i sqrt(t) on each side of a hop
  const int D = 5;
  HostMPO m;
  for (int k = 0; k < L; k++) {
    const int Dl = k == 0 ? 1 : D, Dr = k == L - 1 ? 1 : D;
    std::vector<cd> C((size_t)Dl * Dr * 6, cd(0, 0));
    auto at = [&](int l, int r, int op) -> cd& { return C[l + Dl * (r + Dr * op)]; };
    if (k != L - 1) {
      at(0, 0, 0) = 1.0;
      at(0, 1, 2) = hop;
      at(0, 2, 3) = hop;
      at(0, 3, 4) = 2 * penN;  // first half of the 2 pen n_i n_j pair term
    }
    if (k != 0 && k != L - 1) at(3, 3, 0) = 1.0;
    at(0, Dr - 1, 1) = half_u;
    at(0, Dr - 1, 4) = V - 2 * Ntarget * penN;
    at(0, Dr - 1, 5) = penN;
    at(0, Dr - 1, 0) = penN * Ntarget * Ntarget / L;  // constant share of pen Ntarget^2
    if (k != 0) {
      at(1, Dr - 1, 3) = hop;
      at(2, Dr - 1, 2) = hop;
      at(3, Dr - 1, 4) = 1.0;
      at(Dl - 1, Dr - 1, 0) = 1.0;
    }
    m.dims.push_back({d, Dl, d, Dr});
    m.W.push_back(contract_coeffs_d(C, Dl, Dr, 6, Z, d));
  }
  return m;
}

}  // namespace mpsgpu
