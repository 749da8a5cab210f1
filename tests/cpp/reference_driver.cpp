// A driver written against the reference's C++ entry points (the class
// templates of gemm_opt.cpp, include/sme_syrk.hpp and include/sme_trp_3d.hpp),
// compiled against include/skgemm.hpp and linked with libskgemm.so only.
// It replays the reference's own known-answer inputs and checks them with a
// naive loop, in the way the reference's drivers do (gemm_opt.cpp:432-505,
// syrk_crsp.cpp:469-527, trp_3d_test.cpp:113-159). Exit status 0 = all pass.
#include <cmath>
#include <cstdio>
#include <vector>

#include "skgemm.hpp"

static int check_gemm(int M, int N, int K, double alpha, double gamma) {
  std::vector<double> A(M * K), B(K * N), D(M * N, 0.0);
  for (int j = 0; j < K; ++j)
    for (int i = 0; i < M; ++i) A[i + j * M] = (i + 1) * 0.01 + (j + 1) * 0.001;
  for (int i = 0; i < K; ++i)
    for (int j = 0; j < N; ++j) B[i * N + j] = (i + 1) * 0.001 + (j + 1) * 0.01;
  gemm<double>::compute_test(M, N, K, A.data(), B.data(), D.data(), alpha, gamma);
  double worst = 0;
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0;
      for (int k = 0; k < K; ++k) s += A[i + k * M] * B[k * N + j];
      double ref = alpha * s + gamma;
      worst = std::fmax(worst, std::fabs(D[i * N + j] - ref) / (std::fabs(ref) + 1e-10));
    }
  std::printf("gemm %d %d %d: max rel err %.2e\n", M, N, K, worst);
  return worst < 1e-12 ? 0 : 1;
}

static int check_syrk(int K, int M) {
  const int tiles = (M + 15) / 16;
  std::vector<double> Ap(tiles * K * 16, 0.0), C(M * M, 0.1);
  for (int tm = 0; tm < tiles; ++tm)
    for (int k = 0; k < K; ++k)
      for (int ml = 0; ml < 16; ++ml)
        if (tm * 16 + ml < M) Ap[(tm * K + k) * 16 + ml] = std::sin(0.001 * (tm * 16 + ml) + 0.01 * k);
  sme_syrk<double>::compute(K, M, Ap.data(), C.data(), 1.0, 0.0);
  double worst = 0;
  for (int m1 = 0; m1 < M; ++m1)
    for (int m2 = m1; m2 < M; ++m2) {
      double s = 0;
      for (int k = 0; k < K; ++k)
        s += Ap[(m1 / 16) * K * 16 + k * 16 + m1 % 16] * Ap[(m2 / 16) * K * 16 + k * 16 + m2 % 16];
      worst = std::fmax(worst, std::fabs(C[m1 + m2 * M] - s) / std::fmax(1.0, std::fabs(s)));
    }
  std::printf("syrk %d %d: max rel err %.2e\n", K, M, worst);
  return worst < 1e-12 ? 0 : 1;
}

static int check_rot(int Nd, int nb) {
  std::vector<double> A(Nd * nb), Q(nb * nb), D(Nd * nb, 0.0);
  for (int g = 0; g < Nd; ++g)
    for (int b = 0; b < nb; ++b) A[(g / 16) * nb * 16 + b * 16 + g % 16] = (g + 1) * 0.001 + (b + 1) * 0.01;
  for (int b = 0; b < nb; ++b)
    for (int bp = 0; bp < nb; ++bp) Q[b * nb + bp] = (b + 1) * 0.01 + (bp + 1) * 0.001;
  sme_gemm_trp<double>::compute(Nd, nb, A.data(), Q.data(), D.data());
  double worst = 0;
  for (int g = 0; g < Nd; ++g)
    for (int bp = 0; bp < nb; ++bp) {
      double s = 0;
      for (int b = 0; b < nb; ++b) s += A[(g / 16) * nb * 16 + b * 16 + g % 16] * Q[b * nb + bp];
      double got = D[(bp / 16) * Nd * 16 + g * 16 + bp % 16];
      worst = std::fmax(worst, std::fabs(got - s) / (std::fabs(s) + 1e-10));
    }
  std::printf("rot %d %d: max rel err %.2e\n", Nd, nb, worst);
  return worst < 1e-12 ? 0 : 1;
}

int main() {
  int fails = 0;
  fails += check_gemm(32, 64, 128, 1.0, 0.0);
  fails += check_gemm(32, 64, 4096, 1.0, 0.0);
  fails += check_gemm(32, 64, 4096, 2.0, 0.5);
  fails += check_gemm(64, 128, 2048, 1.0, 0.0);
  fails += check_gemm(1000, 1000, 1000, 1.0, 0.0);
  fails += check_syrk(2048, 256);
  fails += check_syrk(1000, 100);
  fails += check_rot(4096, 128);
  fails += check_rot(1024, 256);
  try {
    gemm<double>::compute_test(-1, 2, 2, nullptr, nullptr, nullptr, 1.0, 0.0);
    fails += 1;  // must have thrown
  } catch (const skgemm::error& e) {
    std::printf("bad shape rejected: %d\n", e.code);
  }
  std::printf("%s\n", fails ? "FAILED" : "PASSED");
  return fails ? 1 : 0;
}
