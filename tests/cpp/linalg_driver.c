/* A C caller of the reference's converter names, declared exactly as in the
 * reference (include/sme_pack.hpp:319-329) and linked against libskgemm.so
 * alone: pack and unpack a column-major [Nd, nb] block, check the grid-packed
 * index map [(g/16)*nb*16 + b*16 + g%16] and the round trip, including a
 * ragged Nd whose last Nd % 16 grid points the reference leaves alone. */
#include <stdio.h>
#include <stdlib.h>

void linalg_pack_c16_f64(const int Nd, const int nb, const double* src, double* dst);
void linalg_pack_r16_f64(const int Nd, const int nb, const double* src, double* dst);
void linalg_unpack_c16_f64(const int Nd, const int nb, const double* src, double* dst);
void linalg_unpack_r16_f64(const int Nd, const int nb, const double* src, double* dst);

static int run(int Nd, int nb) {
  const int R = Nd / 16 * 16;
  double* X = malloc(sizeof(double) * Nd * nb);
  double* P = malloc(sizeof(double) * R * nb);
  double* P2 = malloc(sizeof(double) * R * nb);
  double* Y = malloc(sizeof(double) * Nd * nb);
  int fails = 0;
  for (int b = 0; b < nb; ++b)
    for (int g = 0; g < Nd; ++g) X[g + b * Nd] = g * 4096.0 + b + 0.5;
  for (int i = 0; i < Nd * nb; ++i) Y[i] = -1.0;
  linalg_pack_c16_f64(Nd, nb, X, P);
  for (int g = 0; g < R; ++g)
    for (int b = 0; b < nb; ++b)
      fails += P[(g / 16) * nb * 16 + b * 16 + g % 16] != X[g + b * Nd];
  linalg_pack_r16_f64(Nd, nb, X, P2); /* row-major [nb, Nd]: the same bytes */
  for (int i = 0; i < R * nb; ++i) fails += P2[i] != P[i];
  linalg_unpack_c16_f64(Nd, nb, P, Y);
  for (int b = 0; b < nb; ++b)
    for (int g = 0; g < Nd; ++g) fails += Y[g + b * Nd] != (g < R ? X[g + b * Nd] : -1.0);
  for (int i = 0; i < Nd * nb; ++i) Y[i] = -1.0;
  linalg_unpack_r16_f64(Nd, nb, P, Y);
  for (int b = 0; b < nb; ++b)
    for (int g = 0; g < Nd; ++g) fails += Y[g + b * Nd] != (g < R ? X[g + b * Nd] : -1.0);
  free(X);
  free(P);
  free(P2);
  free(Y);
  return fails;
}

int main(void) {
  int fails = run(4096, 96) + run(1000, 48) + run(16, 1) + run(110592, 64);
  printf("%s (%d mismatches)\n", fails ? "FAILED" : "PASSED", fails);
  return fails ? 1 : 0;
}
