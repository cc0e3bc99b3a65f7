// Counter-based random numbers: Philox-4x32-10 (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).  A stream is
// a 64-bit key; draws are indexed by a 32-bit block counter, 4 uniforms per
// block.  Streams never share state, so results do not depend on thread
// scheduling, and a (key, counter) pair can be stored with a particle.
#pragma once
#include <cstdint>

#include "omc_device.cuh"

namespace omc {

struct U4 {
    uint32_t x, y, z, w;
};

OMC_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

OMC_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = mulhi32(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = mulhi32(M1, c.z), lo1 = M1 * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// 64-bit finaliser (splitmix64) for deriving keys of new streams.
OMC_HD uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform in (0,1): double from 32 bits, float from 23 bits, both at bin
// midpoints so neither 0 nor 1 is ever returned.
OMC_HD double u01d(uint32_t x) { return ((double)x + 0.5) * 2.3283064365386963e-10; }
OMC_HD float u01f(uint32_t x) { return ((float)(x >> 9) + 0.5f) * 1.1920928955078125e-07f; }

// One block of a stream.  One out-of-line copy instead of one per draw
// site keeps the transport kernels small; its arguments and result travel
// by value, so the stream's state stays in registers (an out-of-line member
// function would take the state's address and keep it in local memory).
__host__ __device__ __noinline__ inline U4 philox_block(uint32_t ctr, uint32_t seedw, uint32_t k0, uint32_t k1) {
    return philox4x32_10(U4{ctr, seedw, 0x6f6d6321u, 0u}, k0, k1);
}

// A stream with a 4-number buffer.  `ctr` counts blocks consumed.
template <typename R>
struct Philox {
    uint32_t k0, k1, ctr, seedw;
    U4 buf;
    int pos;
    // Stream `key` positioned after `position` numbers were drawn from it:
    // a particle that stops mid-block resumes with the next number of that
    // block, so its stream does not depend on where events are cut.
    OMC_HD void init(uint64_t key, uint32_t seed_word, uint32_t position = 0) {
        k0 = (uint32_t)key;
        k1 = (uint32_t)(key >> 32);
        seedw = seed_word;
        ctr = position >> 2;
        pos = (int)(position & 3u);
        if (pos == 0) {
            pos = 4;
        } else {
            buf = philox4x32_10(U4{ctr, seedw, 0x6f6d6321u, 0u}, k0, k1);
            ctr++;
        }
    }
    // Numbers drawn so far (the argument init() resumes from).
    OMC_HD uint32_t position() const { return (ctr << 2) - 4u + (uint32_t)pos; }
    // The block generator runs once per four numbers.
    OMC_HD void refill() {
        buf = philox_block(ctr, seedw, k0, k1);
        ctr++;
        pos = 0;
    }
    OMC_HD uint32_t next32() {
        if (pos >= 4) refill();
        uint32_t v = pos == 0 ? buf.x : pos == 1 ? buf.y : pos == 2 ? buf.z : buf.w;
        pos++;
        return v;
    }
    OMC_HD R uni();
};
template <>
OMC_HD double Philox<double>::uni() { return u01d(next32()); }
template <>
OMC_HD float Philox<float>::uni() { return u01f(next32()); }

}  // namespace omc
