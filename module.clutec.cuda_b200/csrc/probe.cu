// probe.cu — issue-rate probe for the integer operations the matchers use.
//
// Each kernel runs 8 coupled dependency chains per thread of one operation
// kind, many warps per SM, for a fixed iteration count; the rate is
// operations / (SMs x elapsed seconds x SM clock). The chains are non-linear
// or coupled so the compiler cannot fold iterations. The SM clock is taken
// from clock64() against %globaltimer on one thread of the same launch.
#include "ct_internal.h"
#include "ct_device.cuh"

namespace ct {
namespace {

// One CTA waits on an mbarrier that nothing arrives at (no TMA is issued, no
// thread arrives), through the same bounded wait every TMA consumer uses, with
// `polls` as its limit. The wait gives up, and the kernel records CT_ETIMEOUT
// in the status word exactly as a kernel whose tile never arrived would, then
// returns normally: nothing is in flight, so the context stays usable.
__global__ void __launch_bounds__(32) wait_timeout_kernel(uint32_t polls, int32_t* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        dev::mbar_init(&bar, 1);
        dev::fence_barrier_init();
    }
    __syncwarp();
    const bool ok = dev::mbar_wait_bounded(&bar, 0, polls);
    if (!ok && threadIdx.x == 0) dev::report(status, CT_ETIMEOUT);
}

enum Op { kPopc = 0, kIadd3 = 1, kLop3 = 2, kVimnmx3 = 3, kImad = 4 };

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

template <int OP>
__global__ void __launch_bounds__(256) probe_kernel(uint32_t seed, int iters, uint32_t* sink,
                                                    unsigned long long* clk) {
    uint32_t a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = seed * (threadIdx.x + 1) + 0x9E3779B9u * (i + 1) + blockIdx.x;
    const long long c0 = clock64();
    const uint64_t g0 = gtimer();
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (OP == kPopc) a[i] = __popc(a[i]) + 0u;
                if (OP == kIadd3) a[i] = a[i] + a[(i + 1) & 7] + a[(i + 2) & 7];
                if (OP == kLop3) a[i] = a[i] ^ (a[(i + 1) & 7] & ~a[(i + 2) & 7]);
                if (OP == kVimnmx3) a[i] = __vimin3_u16x2(a[i], a[(i + 1) & 7] + 0u, a[(i + 2) & 7]);
                if (OP == kImad) a[i] = a[i] * a[(i + 1) & 7] + a[(i + 2) & 7];
            }
            if (OP == kPopc) {
#pragma unroll
                for (int i = 0; i < 8; ++i) a[i] = __popc(a[i] + seed);
            }
        }
    }
    const long long c1 = clock64();
    const uint64_t g1 = gtimer();
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) x ^= a[i];
    if (x == 0x12345678u) sink[blockIdx.x] = x;  // keeps the chains alive
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        clk[0] = (unsigned long long)(c1 - c0);
        clk[1] = (unsigned long long)(g1 - g0);
    }
}

// Operations of the probed kind per thread per loop iteration.
template <int OP>
constexpr int ops_per_iter() {
    return OP == kPopc ? 8 * 16 : 64;  // the popc kernel also does one popc per add
}

template <int OP>
int run_probe(int sms, double* rate, double* mhz) {
    uint32_t* sink = nullptr;
    unsigned long long* clk = nullptr;
    CT_CUDA_TRY(cudaMalloc(&sink, sizeof(uint32_t) * sms * 8));
    CT_CUDA_TRY(cudaMalloc(&clk, 2 * sizeof(unsigned long long)));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    probe_kernel<OP><<<blocks, threads>>>(1u, 64, sink, clk);  // warm-up
    cudaEventRecord(e0);
    probe_kernel<OP><<<blocks, threads>>>(1u, iters, sink, clk);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    unsigned long long c[2] = {0, 0};
    cudaMemcpy(c, clk, sizeof c, cudaMemcpyDeviceToHost);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    cudaFree(clk);
    if (err != cudaSuccess) return fail(CT_ECUDA, "probe kernel failed: %s", cudaGetErrorString(err));
    const double f_hz = c[1] ? double(c[0]) / (double(c[1]) * 1e-9) : 0.0;
    const double ops = double(blocks) * threads * iters * ops_per_iter<OP>();
    *rate = (f_hz > 0 && ms > 0) ? ops / (double(sms) * (ms * 1e-3) * f_hz) : 0.0;
    *mhz = f_hz * 1e-6;
    return CT_OK;
}

}  // namespace
}  // namespace ct

extern "C" int ct_probe_pipe_rates(int32_t device, ct_pipe_rates* out) {
    using namespace ct;
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output");
    if (int rc = use_device(device)) return rc;
    const int sms = sm_count(device);
    std::memset(out, 0, sizeof *out);
    out->sm_count = sms;
    double mhz = 0, m = 0;
    if (int rc = run_probe<kPopc>(sms, &out->popc_per_clk_sm, &mhz)) return rc;
    if (int rc = run_probe<kIadd3>(sms, &out->iadd3_per_clk_sm, &m)) return rc;
    if (int rc = run_probe<kLop3>(sms, &out->lop3_per_clk_sm, &m)) return rc;
    if (int rc = run_probe<kVimnmx3>(sms, &out->vimnmx_per_clk_sm, &m)) return rc;
    if (int rc = run_probe<kImad>(sms, &out->imad_per_clk_sm, &m)) return rc;
    out->sm_clock_mhz = mhz;
    return CT_OK;
}

extern "C" int ct_handle_test_wait_timeout(ct_handle* h, uint32_t poll_limit, ct_stream stream) {
    using namespace ct;
    clear_error();
    if (!h) return fail(CT_EINVAL, "null handle");
    if (!h->configured || !h->d_status) return fail(CT_ESTATE, "handle not configured");
    if (poll_limit < 1 || poll_limit > dev::kWaitLimit)
        return fail(CT_EINVAL, "poll_limit must be 1..%u", dev::kWaitLimit);
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    wait_timeout_kernel<<<1, 32, 0, s>>>(poll_limit, h->d_status);
    CT_LAUNCH_CHECK();
    h->last_stream = s;
    return CT_OK;
}
