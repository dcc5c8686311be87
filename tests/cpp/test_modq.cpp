// Checks the modular arithmetic of altopir-public_b200/csrc/modq.cuh (shared by the host and the kernels) against
// 128-bit reference arithmetic: add, subtract, multiply, the 64-bit reduction and the inverse powers of two, on
// edge values and on seeded random inputs.  Prints OK and exits 0 when every case agrees.
#include <cstdint>
#include <cstdio>
#include "../../altopir-public_b200/csrc/modq.cuh"

namespace {
constexpr uint64_t Q = 4294955009ull;
uint64_t state = 0x243f6a8885a308d3ull;
uint64_t next() {  // splitmix64
  uint64_t z = (state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
int bad = 0;
void expect(const char *what, uint64_t got, uint64_t want, uint64_t a, uint64_t b) {
  if (got != want && bad++ < 10)
    printf("%s(%llu, %llu) = %llu, want %llu\n", what, (unsigned long long)a, (unsigned long long)b,
           (unsigned long long)got, (unsigned long long)want);
}
void check_pair(uint32_t a, uint32_t b) {  // a, b residues in [0, Q)
  expect("add_q", alto::add_q(a, b), ((uint64_t)a + b) % Q, a, b);
  expect("sub_q", alto::sub_q(a, b), ((uint64_t)a + Q - b) % Q, a, b);
}
}  // namespace

int main() {
  const uint32_t edges[] = {0u, 1u, 2u, 12286u, 12287u, 12288u, (uint32_t)(Q / 2), (uint32_t)(Q / 2 + 1),
                            (uint32_t)(Q - 12288), (uint32_t)(Q - 2), (uint32_t)(Q - 1)};
  for (uint32_t a : edges)
    for (uint32_t b : edges) check_pair(a, b);
  const uint32_t any[] = {0u, 1u, 12287u, (uint32_t)(Q - 1), (uint32_t)Q, (uint32_t)(Q + 1), 0xfffffffeu, 0xffffffffu};
  for (uint32_t a : any)
    for (uint32_t b : any) expect("mul_q", alto::mul_q(a, b), (uint64_t)((unsigned __int128)a * b % Q), a, b);
  for (int i = 0; i < 20000000; ++i) {
    const uint64_t r = next();
    const uint32_t a = (uint32_t)(r % Q), b = (uint32_t)((r >> 32) * 4294967291ull % Q);
    check_pair(a, b);
    const uint32_t x = (uint32_t)r, y = (uint32_t)(r >> 32);  // any 32-bit operands
    expect("mul_q", alto::mul_q(x, y), (uint64_t)((unsigned __int128)x * y % Q), x, y);
    const uint64_t w = next();
    expect("red_q64", alto::red_q64(w), w % Q, w, 0);
  }
  const uint64_t w_edges[] = {0ull, Q - 1, Q, Q + 1, 0xffffffffull, 0x100000000ull, 0xffffffffffffffffull,
                              0xffffffff00000000ull, (Q << 32) - 1};
  for (uint64_t w : w_edges) expect("red_q64", alto::red_q64(w), w % Q, w, 0);
  for (int l = 0; l <= 12; ++l)
    expect("inv_pow2_q * 2^l", (uint64_t)((unsigned __int128)alto::inv_pow2_q(l) * (1ull << l) % Q), 1, l, 0);
  if (bad) {
    printf("%d mismatches\n", bad);
    return 1;
  }
  printf("OK\n");
  return 0;
}
