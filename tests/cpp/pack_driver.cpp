// The host-side sme_pack<double> of include/skgemm.hpp against the index
// maps of the reference's layouts (include/sme_pack.hpp:30-313); needs no GPU.
#include <cstdio>
#include <vector>

#include "skgemm.hpp"

int main() {
  const int Nd = 48, nb = 32;
  int fails = 0;
  std::vector<double> X(Nd * nb), P(Nd * nb), B(Nd * nb), P2(Nd * nb), X2(Nd * nb);
  for (int g = 0; g < Nd; ++g)
    for (int b = 0; b < nb; ++b) X[g + b * Nd] = g * 1000.0 + b;  // column-major [Nd, nb]
  sme_pack<double>::pack_c16(Nd, nb, X.data(), P.data());
  for (int g = 0; g < Nd; ++g)
    for (int b = 0; b < nb; ++b) fails += P[(g / 16) * nb * 16 + b * 16 + g % 16] != g * 1000.0 + b;
  sme_pack<double>::pack_r16(Nd, nb, X.data(), P2.data());
  fails += P2 != P;
  sme_pack<double>::grid_to_band_tile(Nd, nb, P.data(), B.data());
  for (int g = 0; g < Nd; ++g)
    for (int b = 0; b < nb; ++b) fails += B[(b / 16) * Nd * 16 + g * 16 + b % 16] != g * 1000.0 + b;
  sme_pack<double>::band_to_grid_tile(Nd, nb, B.data(), P2.data());
  fails += P2 != P;
  sme_pack<double>::unpack_c16(Nd, nb, P.data(), X2.data());
  fails += X2 != X;
  sme_pack<double>::unpack_r16(Nd, nb, P.data(), X2.data());
  fails += X2 != X;
  try {
    sme_pack<double>::pack_c16(Nd + 8, nb, X.data(), P.data());
    fails += 1;
  } catch (const skgemm::error& e) {
    fails += e.code != SKGEMM_ERR_INVALID_ARG;
  }
  std::printf("%s\n", fails ? "FAILED" : "PASSED");
  return fails ? 1 : 0;
}
