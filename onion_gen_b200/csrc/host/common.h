// Small helpers shared by the engine's host code: error text, device
// buffers, conversions between the host field and the device limb layout.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../kernels.cuh"
#include "ed25519.h"

namespace og {

inline int fail(char* err, size_t errlen, int code, const char* fmt, ...) {
    if (err && errlen) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, errlen, fmt, ap);
        va_end(ap);
    }
    return code;
}

inline std::string cuda_text(cudaError_t e) {
    return std::string(cudaGetErrorName(e)) + ": " + cudaGetErrorString(e);
}

// A device allocation that frees itself.
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    cudaError_t alloc(size_t count) {
        reset();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// A pinned host allocation that frees itself.
template <typename T>
struct HostBuf {
    T* p = nullptr;
    size_t n = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { reset(); }
    cudaError_t alloc(size_t count) {
        reset();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMallocHost(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    void reset() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};

inline FeWords to_words(const F51& a) {
    uint8_t b[32];
    f_to_bytes(a, b);
    FeWords w;
    for (int k = 0; k < 8; k++)
        w.v[k] = (uint32_t)b[4 * k] | ((uint32_t)b[4 * k + 1] << 8) | ((uint32_t)b[4 * k + 2] << 16) |
                 ((uint32_t)b[4 * k + 3] << 24);
    return w;
}

// Writes a field element into the device's two-uint4 layout.
inline void put_fe(uint4* dst, size_t qstride, const F51& a) {
    FeWords w = to_words(a);
    dst[0] = make_uint4(w.v[0], w.v[1], w.v[2], w.v[3]);
    dst[qstride] = make_uint4(w.v[4], w.v[5], w.v[6], w.v[7]);
}

inline Pt point_from_bytes(const uint8_t in[128]) {
    return Pt{f_from_bytes(in), f_from_bytes(in + 32), f_from_bytes(in + 64), f_from_bytes(in + 96)};
}

inline void point_to_bytes(const Pt& p, uint8_t out[128]) {
    f_to_bytes(p.X, out);
    f_to_bytes(p.Y, out + 32);
    f_to_bytes(p.Z, out + 64);
    f_to_bytes(p.T, out + 96);
}

// Whether the four coordinates describe a point of the curve in extended
// coordinates: -X^2 + Y^2 = Z^2 + d T^2 and X Y = Z T.
inline bool point_valid(const Pt& p) {
    if (f_is_zero(p.Z)) return false;
    F51 lhs = f_sub(f_sq(p.Y), f_sq(p.X));
    F51 rhs = f_add(f_sq(p.Z), f_mul(curve_d(), f_sq(p.T)));
    return f_equal(lhs, rhs) && f_equal(f_mul(p.X, p.Y), f_mul(p.Z, p.T));
}

}  // namespace og
