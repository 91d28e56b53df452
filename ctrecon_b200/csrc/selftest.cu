// selftest.cu -- exercises the library's bounded device-side wait (tc_util.cuh: mbar_wait), the
// mechanism every pipelined kernel relies on to turn a stall into a reported error instead of
// a hung GPU. A single warp waits on an mbarrier that nothing ever arrives on: the wait must
// give up after its time limit, record its code in the context's device error word and return,
// and the host must report CTRECON_ERR_TIMEOUT. Nothing faults, traps or hangs.
#include "internal.h"
#include "tc_util.cuh"

namespace ctr {

namespace {

constexpr int kSelftestCode = 99;

__global__ void k_selftest_wait(int* err, int* result, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        tcu::mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // no thread arrives: phase 0 never completes
    const bool ok = tcu::mbar_wait(&bar, 0, err, kSelftestCode, limit_ns);
    if (threadIdx.x == 0) *result = ok ? 1 : 2;
}

}  // namespace

Status selftest_bounded_wait(ctrecon_ctx* ctx, cudaStream_t s, int limit_ms) {
    CTR_TRY(reset_device_flag(ctx, s));
    int* d = ctx->ws_flag.as<int>();  // [0] error word, [1] the kernel's verdict
    CTR_CUDA(cudaMemsetAsync(d + 1, 0, sizeof(int), s));
    k_selftest_wait<<<1, 32, 0, s>>>(d, d + 1, (unsigned long long)limit_ms * 1000000ull);
    CTR_CUDA(cudaGetLastError());
    CTR_CUDA(cudaStreamSynchronize(s));
    int h[2] = {0, 0};
    CTR_CUDA(cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost));
    if (h[1] != 2)
        return make_status(CTRECON_ERR_INTERNAL,
                           "bounded-wait self-test: the wait did not give up (verdict " +
                               std::to_string(h[1]) + ")");
    if (h[0] != kSelftestCode)
        return make_status(CTRECON_ERR_INTERNAL,
                           "bounded-wait self-test: error word " + std::to_string(h[0]));
    return make_status(CTRECON_ERR_TIMEOUT, "a device-side wait gave up (code " +
                                                std::to_string(h[0]) + ", self-test)");
}

}  // namespace ctr
