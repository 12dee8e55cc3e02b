// Chunk and node digests on the device.
//
// Murmur3: the reference's MurmurHash3_x64_128 (include/kokkos_murmur3.hpp:213-292, seed 0
// at :436) declares rotl64 to return uint32_t (:30-31), so every 64-bit rotate keeps only
// its low 32 bits.  The functions below reproduce that exactly.  Because the rotated value
// fits in 32 bits, the following multiply is a 32x64 product, which the compiler emits as
// two IMADs instead of three.
// MD5: standard RFC 1321 digest (include/kokkos_md5.hpp:287-323 is a plain MD5).
#pragma once
#include "common.cuh"

namespace b2d {

// ---------------------------------------------------------------- Murmur3 (reference variant)
__host__ __device__ __forceinline__ uint64_t mm3_rotl_trunc(uint64_t x, int r) {
  return (uint64_t)(uint32_t)((x << r) | (x >> (64 - r)));
}
__host__ __device__ __forceinline__ uint64_t mm3_fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}
struct Murmur3 {
  uint64_t h1, h2;
  __host__ __device__ __forceinline__ void init() { h1 = 0; h2 = 0; }
  __host__ __device__ __forceinline__ void block(uint64_t k1, uint64_t k2) {
    const uint64_t c1 = 0x87c37b91114253d5ULL, c2 = 0x4cf5ad432745937fULL;
    k1 *= c1; k1 = mm3_rotl_trunc(k1, 31); k1 *= c2; h1 ^= k1;
    h1 = mm3_rotl_trunc(h1, 27); h1 += h2; h1 = h1 * 5 + 0x52dce729ULL;
    k2 *= c2; k2 = mm3_rotl_trunc(k2, 33); k2 *= c1; h2 ^= k2;
    h2 = mm3_rotl_trunc(h2, 31); h2 += h1; h2 = h2 * 5 + 0x38495ab5ULL;
  }
  __host__ __device__ __forceinline__ void block_words(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    block((uint64_t)a | ((uint64_t)b << 32), (uint64_t)c | ((uint64_t)d << 32));
  }
  // tail: 0..15 remaining bytes, given as two little-endian words (bytes beyond rem are 0)
  __host__ __device__ __forceinline__ void tail(uint64_t t1, uint64_t t2, unsigned rem) {
    const uint64_t c1 = 0x87c37b91114253d5ULL, c2 = 0x4cf5ad432745937fULL;
    if (rem > 8) {
      uint64_t k2 = t2;
      k2 *= c2; k2 = mm3_rotl_trunc(k2, 33); k2 *= c1; h2 ^= k2;
    }
    if (rem > 0) {
      uint64_t k1 = t1;
      k1 *= c1; k1 = mm3_rotl_trunc(k1, 31); k1 *= c2; h1 ^= k1;
    }
  }
  __host__ __device__ __forceinline__ Digest finish(uint64_t len) {
    h1 ^= len; h2 ^= len;
    h1 += h2; h2 += h1;
    h1 = mm3_fmix64(h1); h2 = mm3_fmix64(h2);
    h1 += h2; h2 += h1;
    Digest d;
    d.w[0] = (uint32_t)h1; d.w[1] = (uint32_t)(h1 >> 32);
    d.w[2] = (uint32_t)h2; d.w[3] = (uint32_t)(h2 >> 32);
    return d;
  }
};

// ---------------------------------------------------------------- MD5 (RFC 1321)
#define B2D_MD5_F(x, y, z) ((z) ^ ((x) & ((y) ^ (z))))
#define B2D_MD5_G(x, y, z) ((y) ^ ((z) & ((x) ^ (y))))
#define B2D_MD5_H(x, y, z) ((x) ^ (y) ^ (z))
#define B2D_MD5_I(x, y, z) ((y) ^ ((x) | ~(z)))
// One step: a = b + rotl(a + f(b, c, d) + x + t, s).  Only b is the previous step's output, so
// the chain runs through f, one three-input add, the rotate and the add of b; `a` is four steps
// old, and a + x can be formed off the chain.
#define B2D_MD5_STEP(f, a, b, c, d, x, t, s) \
  a = md5_pre_add<SPLIT>(a, (x), one);       \
  a += f(b, c, d) + (t);                     \
  a = ((a << (s)) | (a >> (32 - (s))));      \
  a += b;

// The staged hashing kernels are bound by the integer ALU pipe on MD5 (its logic ops, adds and
// funnel shifts).  With SPLIT, a + x, which does not wait for the previous step, is written as a
// multiply-add by `one`, a 1 the kernel reads from its launch arguments so the compiler cannot
// fold it back into an add (a 1 from constant memory can be folded).  Measured on the 8 GiB
// float32 series (256 B chunks): 2.89 against 2.97 ms per hashing launch, with the same
// instruction count and the ALU pipe at 73.6 % and the FMA pipe at 12.7 % of their peaks either
// way.  Two other splits were slower: also the on-chain add of b as a multiply-add (4.34 against
// 3.23 ms per step), and also the rotate as a 32x32->64 multiply by 2^s whose two halves add up
// to the rotated word (3.59 against 2.95 ms per hashing launch).
template <int SPLIT>
__host__ __device__ __forceinline__ uint32_t md5_pre_add(uint32_t a, uint32_t x, uint32_t one) {
#ifdef __CUDA_ARCH__
  if constexpr (SPLIT != 0) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(one), "r"(a));
    return r;
  }
#endif
  (void)one;
  return a + x;
}

template <int SPLIT>
__host__ __device__ __forceinline__ void md5_compress_t(uint32_t st[4], const uint32_t m[16], uint32_t one = 1u) {
  uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
  B2D_MD5_STEP(B2D_MD5_F, a, b, c, d, m[0], 0xd76aa478u, 7)
  B2D_MD5_STEP(B2D_MD5_F, d, a, b, c, m[1], 0xe8c7b756u, 12)
  B2D_MD5_STEP(B2D_MD5_F, c, d, a, b, m[2], 0x242070dbu, 17)
  B2D_MD5_STEP(B2D_MD5_F, b, c, d, a, m[3], 0xc1bdceeeu, 22)
  B2D_MD5_STEP(B2D_MD5_F, a, b, c, d, m[4], 0xf57c0fafu, 7)
  B2D_MD5_STEP(B2D_MD5_F, d, a, b, c, m[5], 0x4787c62au, 12)
  B2D_MD5_STEP(B2D_MD5_F, c, d, a, b, m[6], 0xa8304613u, 17)
  B2D_MD5_STEP(B2D_MD5_F, b, c, d, a, m[7], 0xfd469501u, 22)
  B2D_MD5_STEP(B2D_MD5_F, a, b, c, d, m[8], 0x698098d8u, 7)
  B2D_MD5_STEP(B2D_MD5_F, d, a, b, c, m[9], 0x8b44f7afu, 12)
  B2D_MD5_STEP(B2D_MD5_F, c, d, a, b, m[10], 0xffff5bb1u, 17)
  B2D_MD5_STEP(B2D_MD5_F, b, c, d, a, m[11], 0x895cd7beu, 22)
  B2D_MD5_STEP(B2D_MD5_F, a, b, c, d, m[12], 0x6b901122u, 7)
  B2D_MD5_STEP(B2D_MD5_F, d, a, b, c, m[13], 0xfd987193u, 12)
  B2D_MD5_STEP(B2D_MD5_F, c, d, a, b, m[14], 0xa679438eu, 17)
  B2D_MD5_STEP(B2D_MD5_F, b, c, d, a, m[15], 0x49b40821u, 22)
  B2D_MD5_STEP(B2D_MD5_G, a, b, c, d, m[1], 0xf61e2562u, 5)
  B2D_MD5_STEP(B2D_MD5_G, d, a, b, c, m[6], 0xc040b340u, 9)
  B2D_MD5_STEP(B2D_MD5_G, c, d, a, b, m[11], 0x265e5a51u, 14)
  B2D_MD5_STEP(B2D_MD5_G, b, c, d, a, m[0], 0xe9b6c7aau, 20)
  B2D_MD5_STEP(B2D_MD5_G, a, b, c, d, m[5], 0xd62f105du, 5)
  B2D_MD5_STEP(B2D_MD5_G, d, a, b, c, m[10], 0x02441453u, 9)
  B2D_MD5_STEP(B2D_MD5_G, c, d, a, b, m[15], 0xd8a1e681u, 14)
  B2D_MD5_STEP(B2D_MD5_G, b, c, d, a, m[4], 0xe7d3fbc8u, 20)
  B2D_MD5_STEP(B2D_MD5_G, a, b, c, d, m[9], 0x21e1cde6u, 5)
  B2D_MD5_STEP(B2D_MD5_G, d, a, b, c, m[14], 0xc33707d6u, 9)
  B2D_MD5_STEP(B2D_MD5_G, c, d, a, b, m[3], 0xf4d50d87u, 14)
  B2D_MD5_STEP(B2D_MD5_G, b, c, d, a, m[8], 0x455a14edu, 20)
  B2D_MD5_STEP(B2D_MD5_G, a, b, c, d, m[13], 0xa9e3e905u, 5)
  B2D_MD5_STEP(B2D_MD5_G, d, a, b, c, m[2], 0xfcefa3f8u, 9)
  B2D_MD5_STEP(B2D_MD5_G, c, d, a, b, m[7], 0x676f02d9u, 14)
  B2D_MD5_STEP(B2D_MD5_G, b, c, d, a, m[12], 0x8d2a4c8au, 20)
  B2D_MD5_STEP(B2D_MD5_H, a, b, c, d, m[5], 0xfffa3942u, 4)
  B2D_MD5_STEP(B2D_MD5_H, d, a, b, c, m[8], 0x8771f681u, 11)
  B2D_MD5_STEP(B2D_MD5_H, c, d, a, b, m[11], 0x6d9d6122u, 16)
  B2D_MD5_STEP(B2D_MD5_H, b, c, d, a, m[14], 0xfde5380cu, 23)
  B2D_MD5_STEP(B2D_MD5_H, a, b, c, d, m[1], 0xa4beea44u, 4)
  B2D_MD5_STEP(B2D_MD5_H, d, a, b, c, m[4], 0x4bdecfa9u, 11)
  B2D_MD5_STEP(B2D_MD5_H, c, d, a, b, m[7], 0xf6bb4b60u, 16)
  B2D_MD5_STEP(B2D_MD5_H, b, c, d, a, m[10], 0xbebfbc70u, 23)
  B2D_MD5_STEP(B2D_MD5_H, a, b, c, d, m[13], 0x289b7ec6u, 4)
  B2D_MD5_STEP(B2D_MD5_H, d, a, b, c, m[0], 0xeaa127fau, 11)
  B2D_MD5_STEP(B2D_MD5_H, c, d, a, b, m[3], 0xd4ef3085u, 16)
  B2D_MD5_STEP(B2D_MD5_H, b, c, d, a, m[6], 0x04881d05u, 23)
  B2D_MD5_STEP(B2D_MD5_H, a, b, c, d, m[9], 0xd9d4d039u, 4)
  B2D_MD5_STEP(B2D_MD5_H, d, a, b, c, m[12], 0xe6db99e5u, 11)
  B2D_MD5_STEP(B2D_MD5_H, c, d, a, b, m[15], 0x1fa27cf8u, 16)
  B2D_MD5_STEP(B2D_MD5_H, b, c, d, a, m[2], 0xc4ac5665u, 23)
  B2D_MD5_STEP(B2D_MD5_I, a, b, c, d, m[0], 0xf4292244u, 6)
  B2D_MD5_STEP(B2D_MD5_I, d, a, b, c, m[7], 0x432aff97u, 10)
  B2D_MD5_STEP(B2D_MD5_I, c, d, a, b, m[14], 0xab9423a7u, 15)
  B2D_MD5_STEP(B2D_MD5_I, b, c, d, a, m[5], 0xfc93a039u, 21)
  B2D_MD5_STEP(B2D_MD5_I, a, b, c, d, m[12], 0x655b59c3u, 6)
  B2D_MD5_STEP(B2D_MD5_I, d, a, b, c, m[3], 0x8f0ccc92u, 10)
  B2D_MD5_STEP(B2D_MD5_I, c, d, a, b, m[10], 0xffeff47du, 15)
  B2D_MD5_STEP(B2D_MD5_I, b, c, d, a, m[1], 0x85845dd1u, 21)
  B2D_MD5_STEP(B2D_MD5_I, a, b, c, d, m[8], 0x6fa87e4fu, 6)
  B2D_MD5_STEP(B2D_MD5_I, d, a, b, c, m[15], 0xfe2ce6e0u, 10)
  B2D_MD5_STEP(B2D_MD5_I, c, d, a, b, m[6], 0xa3014314u, 15)
  B2D_MD5_STEP(B2D_MD5_I, b, c, d, a, m[13], 0x4e0811a1u, 21)
  B2D_MD5_STEP(B2D_MD5_I, a, b, c, d, m[4], 0xf7537e82u, 6)
  B2D_MD5_STEP(B2D_MD5_I, d, a, b, c, m[11], 0xbd3af235u, 10)
  B2D_MD5_STEP(B2D_MD5_I, c, d, a, b, m[2], 0x2ad7d2bbu, 15)
  B2D_MD5_STEP(B2D_MD5_I, b, c, d, a, m[9], 0xeb86d391u, 21)
  st[0] += a; st[1] += b; st[2] += c; st[3] += d;
}
__host__ __device__ __forceinline__ void md5_compress(uint32_t st[4], const uint32_t m[16]) {
  md5_compress_t<0>(st, m, 1u);
}


__host__ __device__ __forceinline__ void md5_init(uint32_t st[4]) {
  st[0] = 0x67452301u; st[1] = 0xefcdab89u; st[2] = 0x98badcfeu; st[3] = 0x10325476u;
}
// final block for a message whose length is a multiple of 64 bytes
__host__ __device__ __forceinline__ void md5_pad_block64(uint32_t st[4], uint64_t len) {
  uint32_t m[16];
#pragma unroll
  for (int i = 0; i < 16; i++) m[i] = 0;
  m[0] = 0x80u;
  m[14] = (uint32_t)(len << 3);
  m[15] = (uint32_t)(len >> 29);
  md5_compress(st, m);
}
__host__ __device__ __forceinline__ Digest md5_digest(const uint32_t st[4]) {
  Digest d;
  d.w[0] = st[0]; d.w[1] = st[1]; d.w[2] = st[2]; d.w[3] = st[3];
  return d;
}

// ---------------------------------------------------------------- byte-granular hashing
// Used for chunk sizes or alignments the staged kernels do not cover and for the short
// last chunk.  Reads bytes, so it works for any address and length.
__host__ __device__ __forceinline__ uint32_t ld_le32_bytes(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
__host__ __device__ __forceinline__ uint32_t ld_le32_partial(const uint8_t* p, uint64_t avail) {
  uint32_t v = 0;
  for (unsigned i = 0; i < 4 && i < avail; i++) v |= (uint32_t)p[i] << (8 * i);
  return v;
}

__host__ __device__ inline Digest hash_bytes_murmur3(const uint8_t* p, uint64_t len) {
  Murmur3 h;
  h.init();
  const uint64_t nb = len / 16;
  const bool al4 = (((uintptr_t)p) & 3u) == 0;
  for (uint64_t i = 0; i < nb; i++) {
    const uint8_t* q = p + 16 * i;
    uint32_t a, b, c, d;
    if (al4) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(q);
      a = w[0]; b = w[1]; c = w[2]; d = w[3];
    } else {
      a = ld_le32_bytes(q); b = ld_le32_bytes(q + 4); c = ld_le32_bytes(q + 8); d = ld_le32_bytes(q + 12);
    }
    h.block_words(a, b, c, d);
  }
  const unsigned rem = (unsigned)(len & 15u);
  const uint8_t* t = p + 16 * nb;
  uint64_t t1 = 0, t2 = 0;
  for (unsigned i = 0; i < rem; i++) {
    if (i < 8) t1 |= (uint64_t)t[i] << (8 * i);
    else t2 |= (uint64_t)t[i] << (8 * (i - 8));
  }
  h.tail(t1, t2, rem);
  return h.finish(len);
}

__host__ __device__ inline Digest hash_bytes_md5(const uint8_t* p, uint64_t len) {
  uint32_t st[4];
  md5_init(st);
  const uint64_t nb = len / 64;
  uint32_t m[16];
  for (uint64_t i = 0; i < nb; i++) {
    const uint8_t* q = p + 64 * i;
#pragma unroll
    for (int k = 0; k < 16; k++) m[k] = ld_le32_bytes(q + 4 * k);
    md5_compress(st, m);
  }
  const unsigned rem = (unsigned)(len - nb * 64);
  const uint8_t* t = p + 64 * nb;
  // message tail + 0x80 + zero pad + 64-bit bit length, one or two blocks
#pragma unroll
  for (int k = 0; k < 16; k++) {
    uint32_t v = 0;
    for (unsigned b = 0; b < 4; b++) {
      unsigned idx = 4u * k + b;
      uint32_t byte = idx < rem ? t[idx] : (idx == rem ? 0x80u : 0u);
      v |= byte << (8 * b);
    }
    m[k] = v;
  }
  if (rem < 56) {
    m[14] = (uint32_t)(len << 3);
    m[15] = (uint32_t)(len >> 29);
    md5_compress(st, m);
  } else {
    md5_compress(st, m);
#pragma unroll
    for (int k = 0; k < 16; k++) m[k] = 0;
    m[14] = (uint32_t)(len << 3);
    m[15] = (uint32_t)(len >> 29);
    md5_compress(st, m);
  }
  return md5_digest(st);
}

__host__ __device__ __forceinline__ Digest hash_bytes(int kind, const uint8_t* p, uint64_t len) {
  return kind == HASH_MD5 ? hash_bytes_md5(p, len) : hash_bytes_murmur3(p, len);
}

// Inner node digest: hash of the 32 bytes left-child digest || right-child digest
// (src/tree_approach.cpp:131,221,389,459 of the reference).
__device__ __forceinline__ Digest hash_pair(int kind, const Digest& l, const Digest& r) {
  if (kind == HASH_MD5) {
    uint32_t st[4];
    md5_init(st);
    uint32_t m[16] = {l.w[0], l.w[1], l.w[2], l.w[3], r.w[0], r.w[1], r.w[2], r.w[3],
                      0x80u, 0u, 0u, 0u, 0u, 0u, 256u, 0u};
    md5_compress(st, m);
    return md5_digest(st);
  }
  Murmur3 h;
  h.init();
  h.block_words(l.w[0], l.w[1], l.w[2], l.w[3]);
  h.block_words(r.w[0], r.w[1], r.w[2], r.w[3]);
  return h.finish(32);
}

}  // namespace b2d
