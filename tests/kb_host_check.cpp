// Test harness (not product code): compiles the product's field header for the
// host and prints results of its arithmetic for inputs read from stdin, so the
// CPU test suite can check the Montgomery and extension arithmetic exactly.
// Input lines: "mul a b", "ef a0 a1 a2 a3 b0 b1 b2 b3", "red t", "shoup a w" (canonical
// values for mul/ef; a raw 64-bit value for red; any 32-bit a and canonical w for shoup).
#include <cstdio>
#include <cstring>

#include "kb.cuh"

int main() {
  char op[16];
  while (std::scanf("%15s", op) == 1) {
    if (!std::strcmp(op, "mul")) {
      unsigned a, b;
      std::scanf("%u %u", &a, &b);
      std::printf("%u\n", kb::from_mont(kb::mul(kb::to_mont(a), kb::to_mont(b))));
    } else if (!std::strcmp(op, "ef")) {
      kb::ef x, y;
      for (int i = 0; i < 4; i++) { unsigned v; std::scanf("%u", &v); x.c[i] = kb::to_mont(v); }
      for (int i = 0; i < 4; i++) { unsigned v; std::scanf("%u", &v); y.c[i] = kb::to_mont(v); }
      kb::ef z = kb::ef_mul(x, y);
      std::printf("%u %u %u %u\n", kb::from_mont(z.c[0]), kb::from_mont(z.c[1]), kb::from_mont(z.c[2]),
                  kb::from_mont(z.c[3]));
    } else if (!std::strcmp(op, "shoup")) {
      unsigned a, w;
      std::scanf("%u %u", &a, &w);
      std::printf("%u\n", kb::mul_shoup(a, w, kb::shoup_const(w)));
    } else if (!std::strcmp(op, "red")) {
      unsigned long long t;
      std::scanf("%llu", &t);
      std::printf("%u\n", kb::reduce_wide(t));
    }
  }
  return 0;
}
