// Counter-based random stream for the production tracing mode.
//
// Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
// multiplies with the round multipliers and Weyl key increments given there.
//
// Counter layout used by the tracer (key = the 64-bit seed):
//   x = ray index, y = slot | purpose << 24, z/w = low/high 32 bits of the
//   stream key (scene identity).  Slot 0 is the initial-direction jitter,
//   slot b+1 the diffuse decision of bounce b.  Purpose 1 is synthesis noise.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define AC_HD __host__ __device__ __forceinline__
#else
#define AC_HD inline
#endif

namespace ac {

struct u32x4 {
    uint32_t x, y, z, w;
};

AC_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

AC_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t hi0 = mulhi32(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = mulhi32(M1, c.z), lo1 = M1 * c.z;
        c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// 53-bit uniform double in [0, 1) from two 32-bit words.
AC_HD double u01_53(uint32_t hi, uint32_t lo) {
    const uint64_t bits = (static_cast<uint64_t>(hi >> 5) << 26) | static_cast<uint64_t>(lo >> 6);
    return static_cast<double>(bits) * (1.0 / 9007199254740992.0);
}

// Uniform integer in [0, n) by multiply-high.
AC_HD uint32_t below(uint32_t word, uint32_t n) { return mulhi32(word, n); }

enum : uint32_t { kPurposeTrace = 0u, kPurposeNoise = 1u };

AC_HD u32x4 trace_draw(uint64_t seed, uint64_t stream_key, uint32_t ray, uint32_t slot) {
    return philox4x32_10(
        u32x4{ray, (slot & 0xFFFFFFu) | (kPurposeTrace << 24), static_cast<uint32_t>(stream_key),
              static_cast<uint32_t>(stream_key >> 32)},
        static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
}

AC_HD u32x4 noise_draw(uint64_t seed, uint32_t pair_index) {
    return philox4x32_10(u32x4{pair_index, kPurposeNoise << 24, 0u, 0u}, static_cast<uint32_t>(seed),
                         static_cast<uint32_t>(seed >> 32));
}

// pi * (3 - sqrt(5)) as Python evaluates it (steam_rt.py:3965 golden-angle step),
// and the same step in turns, (3 - sqrt(5)) / 2.
constexpr double kGoldenAngle = 2.399963229728653;
constexpr double kGoldenTurns = 0.3819660112501051;
constexpr double kInvTwoPi = 0.15915494309189535;

}  // namespace ac
