// dnni_calibrate.cuh -- measured throughput of the operations that bound the
// hot path's kernels, for their op-count rooflines (dnni_measure_peaks):
//   integer multiply-adds    the distance evaluations of the nearest-site
//                            search (k_near_dense, k_near_far) are 32-bit
//                            integer arithmetic;
//   shared-memory atomics    the span window's marker adds (k_scatter_window);
//   L2 64-bit reductions     the window's flush and the direct span path.
// Each kernel runs on every SM with enough warps to saturate its unit, is
// timed with CUDA events after a warm-up launch, and is counted in the
// operations it issues.  Included by dnni_engine.cu.
#pragma once

namespace dnni {

constexpr int kCalThreads = 256;

// Eight independent multiply-add chains per thread.
__global__ void __launch_bounds__(kCalThreads) k_cal_imad(int iters, unsigned* out) {
    unsigned a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
             a7 = a0 + 7;
    const unsigned m = 0x9E3779B1u + blockIdx.x, c = 0x7F4A7C15u;
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
        a0 = a0 * m + c; a1 = a1 * m + c; a2 = a2 * m + c; a3 = a3 * m + c;
        a4 = a4 * m + c; a5 = a5 * m + c; a6 = a6 * m + c; a7 = a7 * m + c;
    }
    const unsigned r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x12345678u) out[blockIdx.x] = r;     // keeps the chains live
}

// Conflict-free 32-bit shared-memory atomic adds: each warp's lanes hit 32
// consecutive words.
__global__ void __launch_bounds__(kCalThreads) k_cal_smem_atomic(int iters, unsigned* out) {
    __shared__ unsigned s[4 * kCalThreads];
    for (int e = threadIdx.x; e < 4 * kCalThreads; e += kCalThreads) s[e] = 0;
    __syncthreads();
#pragma unroll 4
    for (int i = 0; i < iters; ++i) atomicAdd(&s[threadIdx.x + (i & 3) * kCalThreads], 1u);
    __syncthreads();
    if (threadIdx.x == 0 && s[0] == 0x12345678u) out[blockIdx.x] = s[0];
}

// Coalesced 64-bit global atomic adds over an L2-resident buffer (mask + 1
// words): each warp adds to 32 consecutive words per step.
__global__ void __launch_bounds__(kCalThreads) k_cal_red64(unsigned long long* buf, int iters, size_t mask) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll 4
    for (int i = 0; i < iters; ++i, w += stride) atomicAdd(&buf[w & mask], 1ull);
}

}  // namespace dnni

extern "C" dnni_status dnni_measure_peaks(int32_t device, dnni_peaks* out) {
    if (!out) return DNNI_E_INVAL;
    memset(out, 0, sizeof(*out));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return DNNI_E_INVAL;
    }
    DeviceGuard g(device);
    int sms = 0, clk_khz = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device);
    out->sm_count = sms;
    out->sm_clock_mhz = clk_khz / 1000.0;
    const size_t words = (size_t)1 << 22;               // 32 MB: resident in L2
    unsigned* sink = nullptr;
    unsigned long long* buf = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    dnni_status rs = DNNI_OK;
    if (cudaMalloc(&sink, sizeof(unsigned) * 4096) != cudaSuccess ||
        cudaMalloc(&buf, sizeof(unsigned long long) * words) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        rs = DNNI_E_NOMEM;
    }
    const int grid = sms * 8;                           // 2048 threads per SM
    auto timed = [&](auto launch, double ops) -> double {
        launch();                                       // warm-up
        cudaEventRecord(e0, st);
        launch();
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) return 0.0;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms > 0 ? ops / (ms * 1e-3) : 0.0;
    };
    if (!rs) {
        cudaMemsetAsync(buf, 0, sizeof(unsigned long long) * words, st);
        const int it_imad = 4096, it_atom = 4096, it_red = 256;
        const double thr = (double)grid * kCalThreads;
        out->int_ops_per_s = timed([&] { k_cal_imad<<<grid, kCalThreads, 0, st>>>(it_imad, sink); },
                                   thr * it_imad * 8.0);
        out->smem_atomics_per_s = timed([&] { k_cal_smem_atomic<<<grid, kCalThreads, 0, st>>>(it_atom, sink); },
                                        thr * it_atom);
        out->l2_red64_per_s = timed([&] { k_cal_red64<<<grid, kCalThreads, 0, st>>>(buf, it_red, words - 1); },
                                    thr * it_red);
        if (cudaGetLastError() != cudaSuccess) rs = DNNI_E_CUDA;
    }
    if (st) cudaStreamSynchronize(st);
    if (sink) cudaFree(sink);
    if (buf) cudaFree(buf);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    return rs;
}
