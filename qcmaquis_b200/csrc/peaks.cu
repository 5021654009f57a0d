// FP64 throughput probes (the measured copy and bf16 peaks have no FP64 counterpart): a DMMA
// (mma.sync m8n8k4 .f64) loop and a DFMA loop,
// register-resident, one CTA per SM x occupancy.  Used as roofline denominators
// for the plain FP64 form.
#include <cuda_runtime.h>

#include "../../include/qcm_b200.h"
#include "capi_util.hpp"
#include "device.hpp"

namespace {

__global__ void k_dmma_loop(double* out, int iters) {
    double c[8][2];
    double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(c[i][0]), "+d"(c[i][1])
                         : "d"(a), "d"(b));
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
    if (s == 1234.5) out[0] = s;  // keep the loop alive
}

__global__ void k_dfma_loop(double* out, int iters) {
    double c[16];
    double a = 1.0 + 1e-9 * threadIdx.x, b = 0.999999;
#pragma unroll
    for (int i = 0; i < 16; ++i) c[i] = i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 16; ++i) c[i] = fma(c[i], b, a);
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) s += c[i];
    if (s == 1234.5) out[0] = s;
}

}  // namespace

extern "C" int qcm_probe_fp64_peaks(double* dmma_tflops, double* dfma_tflops) {
    QCM_TRY
    qcm::ensure_device();
    int dev = 0, sms = 0;
    QCM_CUDA(cudaGetDevice(&dev));
    QCM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    qcm::DBuf<double> out(1);
    cudaEvent_t e0, e1;
    QCM_CUDA(cudaEventCreate(&e0));
    QCM_CUDA(cudaEventCreate(&e1));
    const int blocks = sms * 4, threads = 256, iters = 4096;
    float ms = 0;
    for (int pass = 0; pass < 2; ++pass) {  // first pass warms up
        QCM_CUDA(cudaEventRecord(e0));
        k_dmma_loop<<<blocks, threads>>>(out.get(), iters);
        QCM_CUDA(cudaEventRecord(e1));
        QCM_CUDA(cudaEventSynchronize(e1));
        QCM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    }
    // per warp per mma: 8*8*4 FMA = 512 flops
    double warps = double(blocks) * threads / 32;
    *dmma_tflops = warps * iters * 8 * 512.0 / (ms * 1e-3) / 1e12;
    for (int pass = 0; pass < 2; ++pass) {
        QCM_CUDA(cudaEventRecord(e0));
        k_dfma_loop<<<blocks, threads>>>(out.get(), iters);
        QCM_CUDA(cudaEventRecord(e1));
        QCM_CUDA(cudaEventSynchronize(e1));
        QCM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    }
    *dfma_tflops = double(blocks) * threads * iters * 16 * 2.0 / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    QCM_CUDA(cudaGetLastError());
    return QCM_OK;
    QCM_CATCH
}
