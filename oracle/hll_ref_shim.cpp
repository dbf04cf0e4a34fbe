// TEST INFRASTRUCTURE ONLY: a C-ABI shim over the reference's own
// HyperLogLog and hash headers, compiled from where they lie in the
// reference tree (plato/util/hyperloglog.hpp, plato/util/hash.hpp) into
// oracle/_ref/libhll_ref.so by oracle/build.py (build_ref).  It is used only
// by tests/golden/make_golden.py to generate the committed HLL golden
// vectors that pin oracle/hll.py; nothing on the GPU box loads it.
#include <cstdint>
#include <cstring>

#include "plato/util/hyperloglog.hpp"

namespace {

template <uint32_t P>
void add_ids(uint8_t* regs, const uint32_t* ids, uint64_t n) {
  plato::hyperloglog_t<P> h;
  std::memcpy(h.registers_, regs, sizeof(h.registers_));
  for (uint64_t i = 0; i < n; ++i) h.add(&ids[i], sizeof(uint32_t));
  std::memcpy(regs, h.registers_, sizeof(h.registers_));
}

template <uint32_t P>
double estimate(const uint8_t* regs) {
  plato::hyperloglog_t<P> h;
  std::memcpy(h.registers_, regs, sizeof(h.registers_));
  return h.estimate();
}

template <uint32_t P>
int merge(uint8_t* dst, const uint8_t* src) {
  plato::hyperloglog_t<P> a, b;
  std::memcpy(a.registers_, dst, sizeof(a.registers_));
  std::memcpy(b.registers_, src, sizeof(b.registers_));
  const int c = a.merge(b);
  std::memcpy(dst, a.registers_, sizeof(a.registers_));
  return c;
}

#define PLATO_HLL_SWITCH(P, CALL) \
  switch (P) {                    \
    case 4: CALL(4);              \
    case 5: CALL(5);              \
    case 6: CALL(6);              \
    case 7: CALL(7);              \
    case 8: CALL(8);              \
    case 9: CALL(9);              \
    case 10: CALL(10);            \
    case 11: CALL(11);            \
    case 12: CALL(12);            \
    case 13: CALL(13);            \
    case 14: CALL(14);            \
    case 15: CALL(15);            \
    case 16: CALL(16);            \
    default: break;               \
  }

}  // namespace

extern "C" {

// plato::murmurhash3(&id, 4, seed) as hyperloglog_t::add calls it.
uint32_t ref_murmur3_u32(uint32_t id, uint32_t seed) { return plato::murmurhash3(&id, 4u, seed); }

// hyperloglog_t<P>::add of every id, applied to regs [1 << P].
int ref_hll_add(uint32_t P, uint8_t* regs, const uint32_t* ids, uint64_t n) {
#define PLATO_CALL(p) add_ids<p>(regs, ids, n); return 0;
  PLATO_HLL_SWITCH(P, PLATO_CALL)
#undef PLATO_CALL
  return -1;
}

// hyperloglog_t<P>::estimate of regs [1 << P].
double ref_hll_estimate(uint32_t P, const uint8_t* regs) {
#define PLATO_CALL(p) return estimate<p>(regs);
  PLATO_HLL_SWITCH(P, PLATO_CALL)
#undef PLATO_CALL
  return -1.0;
}

// hyperloglog_t<P>::merge(src) into dst; returns the changed-register count.
int ref_hll_merge(uint32_t P, uint8_t* dst, const uint8_t* src) {
#define PLATO_CALL(p) return merge<p>(dst, src);
  PLATO_HLL_SWITCH(P, PLATO_CALL)
#undef PLATO_CALL
  return -1;
}

}  // extern "C"
