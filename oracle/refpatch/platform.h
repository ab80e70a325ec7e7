/*
 * Carry primitives used when the reference C (lib/cbits) is compiled as a TEST ORACLE.
 *
 * This header is placed ahead of the reference's own lib/cbits/platform.h on the
 * include path by oracle/Makefile. The reference header cannot be used as shipped:
 *   - x86 branch (lib/cbits/platform.h:13,17,22-23) passes the *value* `*tgt` where
 *     `_addcarry_u64` expects a pointer, so any build with -DARCH_X86_64 crashes;
 *   - portable branch (lib/cbits/platform.h:52) stores an uninitialised local into
 *     the high word, so every bigint multiplication is wrong.
 * The functions below give the semantics the rest of the generated C relies on
 * (64-bit add/sub with carry/borrow in and out, 128-bit in-place add), written
 * independently. Nothing in the product library includes this file.
 */
#ifndef ZKB200_ORACLE_REF_PLATFORM_H
#define ZKB200_ORACLE_REF_PLATFORM_H

#include <stdint.h>

#if defined(ARCH_X86_64)
#include <x86intrin.h>

static inline uint8_t addcarry_u64(uint8_t carry, uint64_t arg1, uint64_t arg2, uint64_t *tgt) {
  unsigned long long out;
  uint8_t c = _addcarry_u64(carry, arg1, arg2, &out);
  *tgt = (uint64_t)out;
  return c;
}

static inline uint8_t subborrow_u64(uint8_t borrow, uint64_t arg1, uint64_t arg2, uint64_t *tgt) {
  unsigned long long out;
  uint8_t b = _subborrow_u64(borrow, arg1, arg2, &out);
  *tgt = (uint64_t)out;
  return b;
}

#else

static inline uint8_t addcarry_u64(uint8_t carry, uint64_t arg1, uint64_t arg2, uint64_t *tgt) {
  unsigned __int128 s = (unsigned __int128)arg1 + arg2 + carry;
  *tgt = (uint64_t)s;
  return (uint8_t)(s >> 64);
}

static inline uint8_t subborrow_u64(uint8_t borrow, uint64_t arg1, uint64_t arg2, uint64_t *tgt) {
  unsigned __int128 d = (unsigned __int128)arg1 - arg2 - borrow;
  *tgt = (uint64_t)d;
  return (uint8_t)((d >> 64) & 1);
}

#endif

/* (hi:lo) += (arg_hi:arg_lo); returns the carry out of the high word */
static inline uint8_t addcarry_u128_inplace(uint64_t *tgt_lo, uint64_t *tgt_hi, uint64_t arg_lo, uint64_t arg_hi) {
  uint8_t c = addcarry_u64(0, *tgt_lo, arg_lo, tgt_lo);
  return addcarry_u64(c, *tgt_hi, arg_hi, tgt_hi);
}

#endif
