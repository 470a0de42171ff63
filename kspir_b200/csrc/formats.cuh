// Wire and file formats around the answer path: packing helpers, headers and
// checksums (the C-ABI entry points that use them are in kspir.cu).
//
// The reference keeps everything in std::vector<uint64_t> objects and has no
// serialization (RlweCiphertext lwe.h:48-110: a then b, N words each;
// AutoKeyBSGSRNS lwe.h:381-466, AutoKey lwe.h:175-234, RGSWCiphertext
// lwe.h:113-170).  These formats carry exactly those words, in the flattened
// orders of include/kspir_b200.h, packed to the bits their moduli need:
// words mod crtMod (< 2^56) as 7 little-endian bytes, words mod bsMod
// (< 2^24) as 3.  The database file keeps the datacrt words whole (8 bytes):
// its words need not be canonical.
//
// Every container starts with a fixed header and carries a 64-bit checksum of
// its payload: sum over 8-byte little-endian chunks c_i (the last zero-padded)
// of mix64(c_i ^ (i * 0x9E3779B97F4A7C15)) mod 2^64, with mix64 the
// splitmix64 finaliser -- order-dependent, and summable in parallel (the
// database file's checksum is computed on the device).
#pragma once

#include <cstdint>
#include <cstring>

#include "common.cuh"

namespace kspir {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

__host__ __device__ __forceinline__ uint64_t chunk_hash(uint64_t chunk, uint64_t i) {
    return mix64(chunk ^ (i * 0x9E3779B97F4A7C15ull));
}

inline uint64_t payload_checksum(const uint8_t* p, size_t bytes) {
    uint64_t h = 0;
    const size_t full = bytes / 8;
    for (size_t i = 0; i < full; i++) {
        uint64_t c;
        memcpy(&c, p + 8 * i, 8);
        h += chunk_hash(c, i);
    }
    if (bytes % 8) {
        uint64_t c = 0;
        memcpy(&c, p + 8 * full, bytes % 8);
        h += chunk_hash(c, full);
    }
    return h;
}

// checksum of n 64-bit words on the device: partial sums per thread, one
// 64-bit atomic add per warp (sums mod 2^64 commute)
__global__ void k_words_checksum(const uint64_t* __restrict__ w, size_t n, unsigned long long* out) {
    uint64_t h = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        h += chunk_hash(w[i], i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)h);
}

// n words, `width` bytes each (little-endian); words must be < 2^(8 width)
inline void pack_words(const uint64_t* w, size_t n, int width, uint8_t* out) {
    for (size_t i = 0; i < n; i++) {
        uint64_t v = w[i];
        for (int b = 0; b < width; b++) out[i * width + b] = (uint8_t)(v >> (8 * b));
    }
}

inline void unpack_words(const uint8_t* in, size_t n, int width, uint64_t* w) {
    for (size_t i = 0; i < n; i++) {
        uint64_t v = 0;
        for (int b = 0; b < width; b++) v |= (uint64_t)in[i * width + b] << (8 * b);
        w[i] = v;
    }
}

// ---------------------------------------------------------------------------
// headers

constexpr uint32_t kFormatVersion = 1;
constexpr int kWireHeader = 16;     // query / response: magic, version, kind, checksum
constexpr int kFileHeader = 64;     // key bundle / database file

struct FileHeader {                 // 64 bytes, little-endian
    char magic[8];
    uint32_t version, n, r, n1;
    uint64_t payload_bytes;
    uint64_t checksum;
    uint8_t reserved[24];
};
static_assert(sizeof(FileHeader) == kFileHeader, "file header layout");

struct WireHeader {                 // 16 bytes (N = 4096 is implied by the version)
    char magic[4];
    uint16_t version, kind;         // kind 1: query, 2: response
    uint64_t checksum;
};
static_assert(sizeof(WireHeader) == kWireHeader, "wire header layout");

constexpr char kKeyMagic[8] = {'K', 'S', 'P', 'I', 'R', 'K', 'E', 'Y'};
constexpr char kDbMagic[8] = {'K', 'S', 'P', 'I', 'R', 'D', 'B', '1'};
constexpr char kWireMagic[4] = {'K', 'S', 'P', 'W'};

inline int log2_ceil(int v) {
    int l = 0;
    while ((1 << l) < v) l++;
    return l;
}

// key-bundle payload: baby [N1/2][6][2][N] (rows 0-2 mod crtMod at 7 bytes,
// rows 3-5 mod bsMod at 3), then giant [N2-1][2][2][N], packing
// [log2 r][4][2][N] and rgsw [4][2][N], all mod crtMod at 7 bytes
inline size_t key_payload_bytes(int r, int N1) {
    const int N2 = kN / 2 / N1;
    const size_t baby = (size_t)(N1 / 2) * 2 * kN * (3 * 7 + 3 * 3);
    const size_t crt_words = ((size_t)(N2 - 1) * 2 * 2 + (size_t)log2_ceil(r) * 4 * 2 + 4 * 2) * kN;
    return baby + crt_words * 7;
}

constexpr size_t kQueryWireBytes = kWireHeader + (size_t)2 * kN * 7 + (size_t)2 * kN * 3;
constexpr size_t kResponseWireBytes = kWireHeader + (size_t)2 * kN * 7;

}  // namespace kspir
