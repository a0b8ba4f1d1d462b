// selftest.cu -- a check of the device-side failure detection: a bounded
// wait that nothing can satisfy must give up after its limit, raise the
// error flag that the host reads, and return, leaving the context usable.
// The persistent solvers' grid barriers and TMA waits use the same pattern.
#include "device_common.cuh"

int dhara_internal_fail(int code, const char *msg);  // api.cu

namespace {

// One block waits at a counter barrier for a second arrival that never comes.
__global__ void k_wait_selftest(unsigned int *count, GridBarrier *gb, unsigned long long limit_ns) {
    counter_sync(count, 2u, gb, [] {}, limit_ns);
}

int st_fail(int code, const char *msg) { return dhara_internal_fail(code, msg); }

}  // namespace

extern "C" int dhara_selftest_bounded_wait(int device, double limit_ms, int *timed_out) {
    if (!timed_out || !(limit_ms > 0.0) || limit_ms > 10000.0)
        return st_fail(DHARA_ERR_INVALID, "dhara_selftest_bounded_wait: limit_ms must be in (0, 10000]");
    *timed_out = 0;
    if (cudaSetDevice(device) != cudaSuccess) return st_fail(DHARA_ERR_CUDA, "dhara_selftest_bounded_wait: no such device");
    struct Mem {
        unsigned int count;
        unsigned int pad;
        GridBarrier gb;
    } *m = nullptr;
    if (cudaMalloc((void **)&m, sizeof(Mem)) != cudaSuccess)
        return st_fail(DHARA_ERR_NOMEM, "dhara_selftest_bounded_wait: cudaMalloc failed");
    int rc = DHARA_OK;
    Mem host{};
    if (cudaMemset(m, 0, sizeof(Mem)) != cudaSuccess) rc = DHARA_ERR_CUDA;
    if (!rc) {
        k_wait_selftest<<<1, 32>>>(&m->count, &m->gb, (unsigned long long)(limit_ms * 1e6));
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = DHARA_ERR_CUDA;
    }
    if (!rc && cudaMemcpy(&host, m, sizeof(Mem), cudaMemcpyDeviceToHost) != cudaSuccess) rc = DHARA_ERR_CUDA;
    // the context must still work after the wait gave up
    if (!rc && (cudaMemset(m, 0, sizeof(Mem)) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess))
        rc = DHARA_ERR_CUDA;
    cudaFree(m);
    if (rc) return st_fail(rc, "dhara_selftest_bounded_wait: a CUDA call failed");
    *timed_out = host.gb.error != 0 && host.count == 1u;
    return DHARA_OK;
}
