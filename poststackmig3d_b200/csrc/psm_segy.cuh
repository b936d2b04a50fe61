// SEG-Y trace decode and encode on the GPU (sm_100a).
//
// The reference decodes and encodes on the CPU, trace by trace: readTraceData
// (src/segy_utils.cpp:272-318) byte-swaps big-endian samples and converts IBM floats with
// ibmToIeee (:243-254); writeTrace (:598-648) writes a 240-byte header and the samples, IBM
// through ieeeToIbm (:257-270).  Here the file's trace records are uploaded as they are and
// one warp handles one record: coalesced 4-byte loads and stores along the samples, the byte
// swap by __byte_perm.
//
// The IBM conversions are exact integer arithmetic, so no float unit (and no flush-to-zero
// mode) touches the values:
//   * IBM -> IEEE: the value frac * 16^(exp-64) / 2^24 has at most 24 significant bits, so it
//     is exact in fp32 unless it falls below the normal range (rounded to nearest even, as the
//     reference's double -> float conversion rounds) or above it (infinity);
//   * IEEE -> IBM: the reference normalises |v| into [1/16, 1) by exact multiplications by 16
//     and truncates v * 2^24 to 24 bits.  With v = M 2^E (M the 24-bit significand) that is
//     X = floor(log2 v / 4) + 1 and F = trunc(M 2^(E + 24 - 4X)).  Zero encodes as 0, NaN as
//     0x40000000 and +-inf as sign | 0x7FFFFFFF: the reference never terminates on inf.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace psm {

constexpr int kSegyTraceHeader = 240;

__host__ __device__ inline int msb32(uint32_t x) {  // index of the highest set bit, x != 0
#ifdef __CUDA_ARCH__
    return 31 - __clz(x);
#else
    return 31 - __builtin_clz(x);
#endif
}

// IEEE single bits of the IBM single-precision word w.
__host__ __device__ inline uint32_t ibm_to_ieee_bits(uint32_t w) {
    const uint32_t sign = w & 0x80000000u;
    const uint32_t frac = w & 0x00FFFFFFu;
    if (frac == 0) return sign;  // +-0 (any exponent)
    const int expo = static_cast<int>((w >> 24) & 0x7F) - 64;
    const int msb = msb32(frac);
    const int E = msb + 4 * expo - 24;  // value in [2^E, 2^(E+1))
    if (E > 127) return sign | 0x7F800000u;
    if (E >= -126)
        return sign | (static_cast<uint32_t>(E + 127) << 23) |
               ((frac << (23 - msb)) & 0x007FFFFFu);
    // below the normal range: the value in units of 2^-149, rounded to nearest even
    const int s = 4 * expo + 125;
    if (s >= 0) return sign | (frac << s);
    const int k = -s;
    if (k >= 32) return sign;
    uint32_t m = frac >> k;
    const uint32_t rem = frac & ((1u << k) - 1u), half = 1u << (k - 1);
    if (rem > half || (rem == half && (m & 1u))) ++m;
    return sign | m;
}

// IBM single-precision word of the IEEE single with bits b (the reference's truncating
// normalisation).
__host__ __device__ inline uint32_t ieee_bits_to_ibm(uint32_t b) {
    if ((b & 0x7FFFFFFFu) == 0) return 0;  // +0 and -0
    const uint32_t sign = b & 0x80000000u;
    const uint32_t e = (b >> 23) & 0xFF, m = b & 0x007FFFFFu;
    if (e == 0xFF) return m ? 0x40000000u : (sign | 0x7FFFFFFFu);  // NaN, +-inf
    const uint32_t M = e ? (m | 0x00800000u) : m;
    const int E = e ? static_cast<int>(e) - 150 : -149;  // |v| = M 2^E
    const int b2 = msb32(M) + E;                           // floor(log2 |v|)
    const int X = (b2 >> 2) + 1;                           // floor(b2 / 4) + 1
    const int shift = E + 24 - 4 * X;
    const uint32_t F = shift >= 0 ? (M << shift) : (M >> -shift);
    return sign | (static_cast<uint32_t>(64 + X) << 24) | (F & 0x00FFFFFFu);
}

__device__ __forceinline__ uint32_t bswap32(uint32_t w) { return __byte_perm(w, 0, 0x0123); }

// Records [rec_bytes each: 240-byte header + n_t big-endian samples] -> cube rows of ns floats
// (row position[r], skipped when -1).  format 1: IBM, otherwise IEEE.
__global__ void segy_decode_kernel(const unsigned char* __restrict__ records, int64_t n_records,
                                   int rec_bytes, int n_t, int ns, int format,
                                   const int32_t* __restrict__ position,
                                   float* __restrict__ cube) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x >> 5) + (threadIdx.x >> 5);
         r < n_records; r += warps) {
        const int32_t pos = position[r];
        if (pos < 0) continue;
        const uint32_t* src =
            reinterpret_cast<const uint32_t*>(records + r * rec_bytes + kSegyTraceHeader);
        float* dst = cube + static_cast<int64_t>(pos) * ns;
        for (int t = lane; t < n_t; t += 32) {
            const uint32_t w = bswap32(__ldg(src + t));
            dst[t] = __uint_as_float(format == 1 ? ibm_to_ieee_bits(w) : w);
        }
    }
}

// Image rows [n_oi * n_ox][n_t] -> output records (240-byte header + n_t big-endian samples).
// Output trace r copies the header of input record source[r], or, when source[r] < 0, gets a
// zero header with INLINE_3D@188 = il_label[r / n_ox] and CROSSLINE_3D@192 =
// xl_label[r % n_ox] (src/segy_utils.cpp:605-620).
__global__ void segy_encode_kernel(const float* __restrict__ image, int64_t n_out, int n_ox,
                                   int n_t, int format, const int32_t* __restrict__ source,
                                   const unsigned char* __restrict__ in_records,
                                   int in_rec_bytes, const int32_t* __restrict__ il_label,
                                   const int32_t* __restrict__ xl_label,
                                   unsigned char* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int out_rec_bytes = kSegyTraceHeader + 4 * n_t;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x >> 5) + (threadIdx.x >> 5);
         r < n_out; r += warps) {
        uint32_t* dst = reinterpret_cast<uint32_t*>(out + r * out_rec_bytes);
        const int32_t src = source[r];
        for (int k = lane; k < kSegyTraceHeader / 4; k += 32) {
            uint32_t w = 0;
            if (src >= 0) {
                w = __ldg(reinterpret_cast<const uint32_t*>(
                              in_records + static_cast<int64_t>(src) * in_rec_bytes) +
                          k);
            } else if (k == 188 / 4) {
                w = bswap32(static_cast<uint32_t>(il_label[r / n_ox]));
            } else if (k == 192 / 4) {
                w = bswap32(static_cast<uint32_t>(xl_label[r % n_ox]));
            }
            dst[k] = w;
        }
        const float* row = image + r * n_t;
        for (int t = lane; t < n_t; t += 32) {
            const uint32_t b = __float_as_uint(__ldg(row + t));
            dst[kSegyTraceHeader / 4 + t] = bswap32(format == 1 ? ieee_bits_to_ibm(b) : b);
        }
    }
}

}  // namespace psm
