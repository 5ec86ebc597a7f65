// Integer-multiply peak of the device, measured: the roofline denominator of
// the key search (which is bound by 32x32 -> 64 partial products on the
// integer multiply-add pipe, not by memory and not by tensor cores).
//
//  * imad: independent `mad.lo.u32` chains, eight per thread — the pipe's
//    issue rate in multiply-adds per second.
//  * fe_mul: independent GF(2^255-19) multiplications (field_asm.cuh), four
//    per thread — what one field multiplication really achieves, counted as
//    64 partial products each.
#include <cuda_runtime.h>

#include "../../include/onion_gen_b200.h"
#include "field.cuh"
#include "host/common.h"

namespace og {
namespace {

__global__ void __launch_bounds__(256) imad_kernel(uint32_t* sink, uint32_t iters, uint32_t salt) {
    uint32_t x[8];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = t * (k + 3) + salt;
    const uint32_t m = salt | 1u, c = salt ^ 0x9e3779b9u;
#pragma unroll 1
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int r = 0; r < 16; r++) {
#pragma unroll
            for (int k = 0; k < 8; k++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[k]) : "r"(m), "r"(c));
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s ^= x[k];
    if (s == 0x12345678u) sink[t] = s;
}

__global__ void __launch_bounds__(256) femul_kernel(uint32_t* sink, uint32_t iters, uint32_t salt) {
    fe a[4], b;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int k = 0; k < 8; k++) a[j].v[k] = t * (7 * j + k + 1) + salt;
#pragma unroll
    for (int k = 0; k < 8; k++) b.v[k] = salt * (k + 11) + 0x5bd1e995u;
#pragma unroll 1
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 4; j++) a[j] = fe_mulv(a[j], b);
    }
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int k = 0; k < 8; k++) s ^= a[j].v[k];
    if (s == 0x12345678u) sink[t] = s;
}

}  // namespace
}  // namespace og

using namespace og;

extern "C" int og_measure_int_peak(int ordinal, double* imad_per_s, double* mul_pp_per_s, char* err, size_t errlen) {
    cudaError_t e = cudaSetDevice(ordinal);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "%s", cuda_text(e).c_str());
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ordinal);
    const int block = 256, grid = sms * 8;
    DevBuf<uint32_t> sink;
    if ((e = sink.alloc((size_t)grid * block)) != cudaSuccess)
        return fail(err, errlen, OG_E_NOMEM, "%s", cuda_text(e).c_str());
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best_imad = 1e30f, best_mul = 1e30f;
    const uint32_t it_imad = 4096, it_mul = 512;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(a);
        imad_kernel<<<grid, block>>>(sink.p, it_imad, 0x1234567u + rep);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (rep && ms < best_imad) best_imad = ms;
        cudaEventRecord(a);
        femul_kernel<<<grid, block>>>(sink.p, it_mul, 0x7654321u + rep);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        if (rep && ms < best_mul) best_mul = ms;
    }
    e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return fail(err, errlen, OG_E_DEVICE, "%s", cuda_text(e).c_str());
    const double threads = (double)grid * block;
    if (imad_per_s) *imad_per_s = threads * it_imad * 16 * 8 / (best_imad * 1e-3);
    if (mul_pp_per_s) *mul_pp_per_s = threads * it_mul * 4 * 64 / (best_mul * 1e-3);
    return OG_OK;
}
