// probe.cu -- integer-ALU throughput probe (sm_100a): the denominator of the INT roofline.
//
// The SCA/SCABit update is bitwise work (LOP3 masks, funnel shifts, XORs); once temporal
// blocking takes HBM off the critical path, the bound is how many such operations the SMs
// retire per second.  This probe measures it on the GPU at hand: every thread runs eight
// interleaved dependency chains of one operation (a 3-input majority LOP3, or a 3-input add)
// that the assembler cannot fold, over a grid of 8 resident 256-thread CTAs per SM, timed
// with CUDA events.  No counterpart in the reference (a measurement helper).
#include <cuda_runtime.h>

#include <cstdint>

#include "kpzb.h"
#include "kpzb_api_internal.h"

namespace kpzb {

template <int OP>
__global__ void __launch_bounds__(256) alu_probe_kernel(uint32_t* out, int iters, uint32_t seed)
{
    uint32_t a[8];
    const uint32_t b = seed ^ (threadIdx.x * 0x9E3779B9u);
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = seed * (uint32_t)(j + 1) + threadIdx.x + blockIdx.x * 977u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (OP == 0)  // majority(a_j, a_{j+1}, b): one LOP3
                asm volatile("lop3.b32 %0, %0, %1, %2, 0xE8;" : "+r"(a[j]) : "r"(a[(j + 1) & 7]), "r"(b));
            else  // a_j + a_{j+1} + b: one IADD3
                asm volatile("add.u32 %0, %0, %1;\n\tadd.u32 %0, %0, %2;" : "+r"(a[j]) : "r"(a[(j + 1) & 7]), "r"(b));
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s ^= a[j];
    if (s == 0x2545F491u) out[blockIdx.x] = s;  // keeps the chains live; practically never taken
}

}  // namespace kpzb

using namespace kpzb;

extern "C" kpzb_status kpzb_probe_alu_peak(int device, double* lop3_per_s, double* iadd3_per_s)
{
    if (!lop3_per_s || !iadd3_per_s) return fail(KPZB_EINVAL, "null output pointer");
    cudaError_t e = cudaSuccess;
    if (device < 0 && (e = cudaGetDevice(&device)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    const int sms = sm_count_of(device);
    if (sms <= 0) return fail(KPZB_ECUDA, "cannot query the SM count");
    const int grid = sms * 8, block = 256, iters = 16384;
    uint32_t* out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(uint32_t) * grid)) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    cudaEvent_t ev[2];
    cudaEventCreate(&ev[0]);
    cudaEventCreate(&ev[1]);
    double rate[2] = {0.0, 0.0};
    for (int op = 0; op < 2 && e == cudaSuccess; ++op) {
        float best = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {  // first launch warms up; keep the fastest
            cudaEventRecord(ev[0]);
            if (op == 0)
                alu_probe_kernel<0><<<grid, block>>>(out, iters, 12345u + rep);
            else
                alu_probe_kernel<1><<<grid, block>>>(out, iters, 12345u + rep);
            cudaEventRecord(ev[1]);
            if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            if (rep > 0 && ms < best) best = ms;
        }
        const double ops = (double)grid * block * iters * 8.0;  // one LOP3 or one IADD3 per chain step
        rate[op] = ops / (best * 1e-3);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "alu_probe_kernel");
    *lop3_per_s = rate[0];
    *iadd3_per_s = rate[1];
    return KPZB_OK;
}
