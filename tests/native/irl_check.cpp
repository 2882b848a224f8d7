// Host check of the thick-restart compression used by the device Lanczos
// (mpsdyn_b200/csrc/tridiag.h).  Reads m, keep, fnorm, a[m], b[m] from stdin
// and prints r, the compressed a and b, the m x r matrix G and the
// eigenvalues of the compressed tridiagonal by bisection.
#include <cstdio>
#include <vector>

#include "../../mpsdyn_b200/csrc/tridiag.h"

int main() {
  int m = 0, keep = 0;
  double fnorm = 0.0;
  if (std::scanf("%d %d %lf", &m, &keep, &fnorm) != 3) return 2;
  std::vector<double> a(m), b(m);
  for (auto& v : a) if (std::scanf("%lf", &v) != 1) return 2;
  for (auto& v : b) if (std::scanf("%lf", &v) != 1) return 2;
  mpsgpu::ThickRestart tr;
  std::vector<double> G;
  const int r = tr.compress(a, b, m, keep, fnorm, G);
  std::printf("%d\n", r);
  for (int i = 0; i < r; i++) std::printf("%.17g ", a[i]);
  std::printf("\n");
  for (int i = 0; i < r; i++) std::printf("%.17g ", b[i]);
  std::printf("\n");
  for (double v : G) std::printf("%.17g ", v);
  std::printf("\n");
  for (int i = 0; i < r; i++) std::printf("%.17g ", mpsgpu::tridiag_eigenvalue(a, b, r, i));
  std::printf("\n");
  return 0;
}
