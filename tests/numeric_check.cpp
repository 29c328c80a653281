// Exhaustive check of the division-free byte rounding in rdb_numeric.h
// against the oracle's restatement of ScaleQuantumToChar (q / 257.0f + 0.5f).
// Built and run by tests/test_numeric.py; prints "mismatches N checked M".
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "rdb_numeric.h"

extern "C" unsigned char orc_scale_quantum_to_char(float q);

int main() {
  uint32_t lim;
  const float top = 65535.0f;
  std::memcpy(&lim, &top, 4);
  uint64_t bad = 0, n = 0;
  for (uint32_t u = 0; u <= lim; ++u) {
    float q;
    std::memcpy(&q, &u, 4);
    ++n;
    const unsigned want = orc_scale_quantum_to_char(q);
    if (rdb::scale_char(q) != want || rdb::key6(q) != (want >> 2)) ++bad;
  }
  // The clamp never yields -0 or NaN here, but both must map to 0.
  const float specials[] = {-0.0f, __builtin_nanf("")};
  for (float q : specials) {
    ++n;
    if (rdb::scale_char(q) != orc_scale_quantum_to_char(q)) ++bad;
  }
  std::printf("mismatches %llu checked %llu\n", static_cast<unsigned long long>(bad),
              static_cast<unsigned long long>(n));
  return bad == 0 ? 0 : 1;
}
