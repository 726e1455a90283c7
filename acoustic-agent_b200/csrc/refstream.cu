// The reference's random workspace drawn on the device (ac_reference_stream).
//
// Acoustic Agent draws, per trace, `num_bounces` rows of uniforms and diffuse
// bank indices from one numpy Generator (steam_rt.py:4009-4044
// `_diffuse_random_sequence`): for each bounce, `rng.random(R)` then
// `rng.integers(0, n, R, dtype=int32)`, with `rng = default_rng(seed + 1)`.
// Generated on the host and uploaded, that is 12 bytes per ray-bounce (240 MB
// for 200,000 rays x 100 bounces).  Here every draw is computed where it is
// stored, bit for bit as numpy makes it.
//
// numpy's default generator is PCG64 (O'Neill, "PCG: A family of simple fast
// space-efficient statistically good algorithms for random number
// generation", 2014): a 128-bit LCG s <- a*s + c, a =
// 0x2360ED051FC65DA44385DF649FCCF645, stepped before each output, the output
// being the XSL-RR permutation of the new state (the xor of its halves
// rotated right by its top six bits).  `random()` is (x >> 11) * 2^-53 of one
// output.  `integers(0, n)` for int32 takes 32-bit words, two per output (low
// half first, the high half kept for the next call, across calls), and maps
// each with Lemire's multiply-shift ((w * n) >> 32); for n a power of two
// that never rejects a word, and for n = 1 no word is drawn at all.
//
// So the draw of every (bounce b, ray r) has a fixed position in the output
// sequence (u = 1 word per integer, 0 when n = 1):
//   uniform: b*R + ceil(b*R*u / 2) + r
//   integer: word k = b*R + r, from output (floor(2p/R) + 1)*R + p, p = k/2,
//            its low half when k is even, else its high half
// and the LCG jumps to any position in O(log position) steps (Brown,
// "Random number generation with arbitrary strides", 1994): a^d and
// c*(a^(d-1) + ... + 1) are composed from precomputed squarings.  Each thread
// jumps once to the start of a run of 32 draws of one row and steps from
// there.  Bank sizes that are not powers of two can reject a word (numpy then
// draws another, shifting every later draw); the entry point refuses them and
// the caller draws those workspaces on the host.
#include <cstdint>

#include <cuda_runtime.h>

#include "common.h"

namespace ac {
namespace {

typedef unsigned __int128 u128;

constexpr int kJumpBits = 48;    // positions below 2^48
constexpr int kRun = 32;         // draws per thread

struct PcgArgs {
    uint64_t state_lo, state_hi;
    uint64_t mult_lo[kJumpBits], mult_hi[kJumpBits];   // a^(2^k)
    uint64_t plus_lo[kJumpBits], plus_hi[kJumpBits];   // c * (a^(2^k) - 1) / (a - 1)
    uint64_t inc_lo, inc_hi;
    int64_t rays;
    int32_t bounces;
    int32_t words_per_draw;   // 1, or 0 when the bank has a single entry
    int32_t bank_shift;       // log2(bank size)
};

__device__ __forceinline__ u128 make128(uint64_t hi, uint64_t lo) { return (static_cast<u128>(hi) << 64) | lo; }

// The state after `steps` LCG steps from the initial one.
__device__ __forceinline__ u128 jump(const PcgArgs &a, uint64_t steps) {
    u128 am = 1, ap = 0;
    for (int k = 0; steps; ++k, steps >>= 1) {
        if (steps & 1u) {
            const u128 m = make128(a.mult_hi[k], a.mult_lo[k]);
            am = am * m;
            ap = ap * m + make128(a.plus_hi[k], a.plus_lo[k]);
        }
    }
    return am * make128(a.state_hi, a.state_lo) + ap;
}

__device__ __forceinline__ uint64_t xsl_rr(u128 s) {
    const uint64_t hi = static_cast<uint64_t>(s >> 64), lo = static_cast<uint64_t>(s);
    const unsigned rot = static_cast<unsigned>(hi >> 58);
    const uint64_t x = hi ^ lo;
    return (x >> rot) | (x << ((64u - rot) & 63u));
}

template <typename T>
__global__ void __launch_bounds__(256) reference_stream_kernel(const __grid_constant__ PcgArgs a, T *random,
                                                               int32_t *indices) {
    const u128 mult = make128(a.mult_hi[0], a.mult_lo[0]);
    const u128 inc = make128(a.inc_hi, a.inc_lo);
    const int64_t R = a.rays;
    const int64_t runs_per_row = (R + kRun - 1) / kRun;
    const int64_t rows = static_cast<int64_t>(a.bounces);
    const int64_t total = (a.words_per_draw ? 2 : 1) * rows * runs_per_row;
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const bool ints = t >= rows * runs_per_row;
        const int64_t run = ints ? t - rows * runs_per_row : t;
        const int64_t b = run / runs_per_row;
        const int64_t r0 = (run % runs_per_row) * kRun;
        const int n = static_cast<int>(R - r0 < kRun ? R - r0 : kRun);
        if (!ints) {
            const int64_t words_before = b * R * a.words_per_draw;
            const uint64_t first = static_cast<uint64_t>(b * R + (words_before + 1) / 2 + r0);
            u128 s = jump(a, first + 1);
            T *out = random + b * R + r0;
            for (int i = 0; i < n; ++i) {
                out[i] = static_cast<T>(static_cast<double>(xsl_rr(s) >> 11) * 0x1.0p-53);
                s = s * mult + inc;
            }
        } else {
            int32_t *out = indices + b * R + r0;
            uint64_t at = ~uint64_t{0};     // output position `s` produces next
            uint64_t have = ~uint64_t{0};   // output position held in `x`
            uint64_t x = 0;
            u128 s = 0;
            for (int i = 0; i < n; ++i) {
                const int64_t k = b * R + r0 + i;
                const int64_t p = k >> 1;
                const uint64_t pos = static_cast<uint64_t>(((2 * p) / R + 1) * R + p);
                if (pos != have) {   // the two words of one output are consecutive draws
                    if (pos != at) s = jump(a, pos + 1);
                    x = xsl_rr(s);
                    s = s * mult + inc;
                    at = pos + 1;
                    have = pos;
                }
                const uint32_t word = (k & 1) ? static_cast<uint32_t>(x >> 32) : static_cast<uint32_t>(x);
                out[i] = static_cast<int32_t>(word >> (32 - a.bank_shift));   // (word * 2^shift) >> 32
            }
        }
    }
}

__global__ void zero_indices_kernel(int32_t *indices, int64_t count) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        indices[i] = 0;
}

}  // namespace
}  // namespace ac

extern "C" int ac_reference_stream(uint64_t state_hi, uint64_t state_lo, uint64_t inc_hi, uint64_t inc_lo,
                                   int64_t num_rays, int32_t num_bounces, int32_t num_bank, int32_t precision,
                                   void *random, int32_t *indices, void *stream_ptr) {
    ac::NvtxRange nvtx_range("ac_reference_stream");
    using ac::u128;
    if (num_rays < 1 || num_bounces < 0 || num_bank < 1 || (num_bounces > 0 && (!random || !indices)))
        return ac::fail(AC_ERR_INVALID, "ac_reference_stream: bad argument");
    if ((inc_lo & 1u) == 0) return ac::fail(AC_ERR_INVALID, "ac_reference_stream: a PCG64 increment is odd");
    if (num_bank & (num_bank - 1))
        return ac::fail(AC_ERR_UNSUPPORTED,
                        "ac_reference_stream: a bank of %d entries can make numpy redraw a word; draw this "
                        "workspace on the host", num_bank);
    // highest output position used: the last integer pair of the last bounce
    const long double last = static_cast<long double>(num_bounces) * num_rays * 2.0L + 2.0L;
    if (last >= static_cast<long double>(uint64_t{1} << ac::kJumpBits))
        return ac::fail(AC_ERR_CAPACITY, "ac_reference_stream: %lld rays x %d bounces is too many draws",
                        (long long)num_rays, num_bounces);
    if (num_bounces == 0) return AC_OK;
    ac::PcgArgs a{};
    a.state_lo = state_lo;
    a.state_hi = state_hi;
    a.inc_lo = inc_lo;
    a.inc_hi = inc_hi;
    a.rays = num_rays;
    a.bounces = num_bounces;
    a.words_per_draw = num_bank > 1 ? 1 : 0;
    int shift = 0;
    while ((1 << shift) < num_bank) ++shift;
    a.bank_shift = shift;
    u128 m = (static_cast<u128>(0x2360ED051FC65DA4ull) << 64) | 0x4385DF649FCCF645ull;
    u128 c = (static_cast<u128>(inc_hi) << 64) | inc_lo;
    for (int k = 0; k < ac::kJumpBits; ++k) {
        a.mult_lo[k] = static_cast<uint64_t>(m);
        a.mult_hi[k] = static_cast<uint64_t>(m >> 64);
        a.plus_lo[k] = static_cast<uint64_t>(c);
        a.plus_hi[k] = static_cast<uint64_t>(c >> 64);
        c = (m + 1) * c;   // 2^k steps twice over: c_{2d} = (a^d + 1) c_d
        m = m * m;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const int64_t runs = ((num_rays + ac::kRun - 1) / ac::kRun) * num_bounces * (a.words_per_draw ? 2 : 1);
    int device = 0, sms = 148;
    AC_CUDA_TRY(cudaGetDevice(&device));
    AC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = static_cast<int>(runs / 256 + 1 < 8LL * sms ? runs / 256 + 1 : 8LL * sms);
    if (precision == AC_PRECISION_FP64)
        ac::reference_stream_kernel<double><<<grid, 256, 0, stream>>>(a, static_cast<double *>(random), indices);
    else
        ac::reference_stream_kernel<float><<<grid, 256, 0, stream>>>(a, static_cast<float *>(random), indices);
    AC_CUDA_TRY(cudaGetLastError());
    if (!a.words_per_draw) {
        const int64_t count = static_cast<int64_t>(num_bounces) * num_rays;
        ac::zero_indices_kernel<<<static_cast<int>(count / 256 + 1 < 4LL * sms ? count / 256 + 1 : 4LL * sms), 256, 0,
                                  stream>>>(indices, count);
        AC_CUDA_TRY(cudaGetLastError());
    }
    return AC_OK;
}
