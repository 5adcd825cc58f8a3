// eph_fields.cu - direct evaluation of an extended body's geopotential field on the device, with the same
// device functions the step kernel (gp_field_lanes, gp_field_columns) and the particle kernels (gp_field)
// use. It is what
// geopotential::sum (src/physics/geopotential.h:36) offers the reference's own known-answer test
// (src/tests/test_geopotential.cpp), so the device evaluation can be held to that test's bound.
#include <cuda_runtime.h>
#include <stdint.h>

#include "eph_models.cuh"
#include "../../include/eph_b200.h"

namespace eph {

// one point per thread (gp_field: the massless-particle kernels' evaluation)
__global__ void gp_field_kernel(const double *__restrict__ coef, int nz, int nt, double R, long long count,
                                const double *__restrict__ r, double *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const v3 a = gp_field(coef, nz, nt, R, mk(r[3 * i], r[3 * i + 1], r[3 * i + 2]));
    out[3 * i] = a.x;
    out[3 * i + 1] = a.y;
    out[3 * i + 2] = a.z;
}

// one point per group of 8 lanes (gp_field_lanes: the single-system step kernel's evaluation)
__global__ void gp_field_lanes_kernel(const double *__restrict__ coef, int nz, int nt, double R, long long count,
                                      const double *__restrict__ r, double *__restrict__ out) {
    __shared__ double X[kGpX];
    gp_expand(coef, nz, nt, X, threadIdx.x, blockDim.x);
    __syncthreads();
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 8;
    if (i >= count) return;   // uniform over the group
    const int lane = threadIdx.x & 31;
    const v3 a = gp_field_lanes<8>(X, GP_RCP, nz, nt, R, mk(r[3 * i], r[3 * i + 1], r[3 * i + 2]), lane & 7,
                                   0xffu << (lane & ~7));
    if ((lane & 7) == 0) {
        out[3 * i] = a.x;
        out[3 * i + 1] = a.y;
        out[3 * i + 2] = a.z;
    }
}

// one point per thread, as the step kernel's one-lane items (the column evaluation for models it covers,
// else gp_field_lanes on one lane)
__global__ void gp_field_item_kernel(const double *__restrict__ coef, int nz, int nt, double R, long long count,
                                     const double *__restrict__ r, double *__restrict__ out) {
    __shared__ double X[kGpX];
    gp_expand(coef, nz, nt, X, threadIdx.x, blockDim.x);
    __syncthreads();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const v3 p = mk(r[3 * i], r[3 * i + 1], r[3 * i + 2]);
    const v3 a = gp_fits_columns(nz, nt) ? gp_field_columns<kGpColK, kGpColM>(X, GP_RCP, R, p)
                                         : gp_field_lanes<1>(X, GP_RCP, nz, nt, R, p, 0, 1u << (threadIdx.x & 31));
    out[3 * i] = a.x;
    out[3 * i + 1] = a.y;
    out[3 * i + 2] = a.z;
}

}  // namespace eph

extern "C" int eph_geopotential_field(int device, const double *coef, int nz, int nt, double R, int lanes,
                                      int64_t count, const double *r, double *out) {
    if (!coef || !r || !out || count < 0 || nz < 0 || nz > EPH_GP_MAX_DEGREE || nt < 0 || nt > nz ||
        (lanes != 0 && lanes != 1 && lanes != 8))
        return EPH_ERR_ARG;
    if (count == 0) return EPH_OK;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return EPH_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return EPH_ERR_ARG;
    double *d_coef = nullptr, *d_r = nullptr, *d_out = nullptr;
    const size_t vb = (size_t)count * 3 * sizeof(double);
    cudaError_t e = cudaMalloc((void **)&d_coef, EPH_GP_TABLE_SIZE * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_r, vb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_out, vb);
    int rc = e == cudaSuccess ? EPH_OK : (e == cudaErrorMemoryAllocation ? EPH_ERR_OOM : EPH_ERR_CUDA);
    if (rc == EPH_OK) {
        if ((e = cudaMemcpy(d_coef, coef, EPH_GP_TABLE_SIZE * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(d_r, r, vb, cudaMemcpyHostToDevice)) != cudaSuccess) {
            rc = EPH_ERR_CUDA;
        }
    }
    if (rc == EPH_OK) {
        const int threads = 128;
        const long long blocks = (count * (lanes == 8 ? 8 : 1) + threads - 1) / threads;
        if (lanes == 1) eph::gp_field_kernel<<<(unsigned)blocks, threads>>>(d_coef, nz, nt, R, count, d_r, d_out);
        else if (lanes == 0) eph::gp_field_item_kernel<<<(unsigned)blocks, threads>>>(d_coef, nz, nt, R, count, d_r, d_out);
        else eph::gp_field_lanes_kernel<<<(unsigned)blocks, threads>>>(d_coef, nz, nt, R, count, d_r, d_out);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(out, d_out, vb, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = EPH_ERR_CUDA;
    }
    cudaFree(d_coef);
    cudaFree(d_r);
    cudaFree(d_out);
    cudaSetDevice(prev);
    return rc;
}

// ------------------------------------------------------------------ FP64 CUDA-core throughput probe
// The RK12 kernels run on the FP64 CUDA-core pipe (no tensor cores), whose peak a DGEMM does not show.
// Each thread runs 8 independent FMA chains (enough to cover the pipe's latency), every SM holds 1024
// threads, and the grid covers every SM several times over; the result is never stored unless a
// runtime-zero flag says so, which keeps the chains live without memory traffic.
namespace eph {
__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, double seed, int store, double *out) {
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = seed + q + threadIdx.x;
    const double m = 1.0 - 1e-16 * seed, c = 1e-300;
#pragma unroll 1
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int q = 0; q < 8; ++q) a[q] = fma(a[q], m, c);
        }
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += a[q];
    if (store) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace eph

extern "C" int eph_fp64_fma_rate(int device, double *tflops) {
    if (!tflops) return EPH_ERR_ARG;
    int prev = -1, sms = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return EPH_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return EPH_ERR_ARG;
    int rc = EPH_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = EPH_ERR_CUDA;
    } else {
        const int threads = 256, blocks = sms * 4 * 4, iters = 4096;
        float best = 0;
        for (int rep = 0; rep < 4 && rc == EPH_OK; ++rep) {   // the first launch warms the clocks up
            cudaEventRecord(e0);
            eph::fma_probe_kernel<<<blocks, threads>>>(iters, 1.0, 0, nullptr);
            cudaEventRecord(e1);
            float ms = 0;
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = EPH_ERR_CUDA;
            else if (rep > 0 && (best == 0 || ms < best)) best = ms;
        }
        if (rc == EPH_OK) *tflops = 2.0 * 16 * 8 * (double)iters * threads * blocks / (best * 1e-3) / 1e12;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaSetDevice(prev);
    return rc;
}
