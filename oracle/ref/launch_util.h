// launch_util.h -- device buffers for the launchers of the reference's own
// kernels (test infrastructure).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

struct RefBuf {
    void *p = nullptr;
    ~RefBuf() {
        if (p) cudaFree(p);
    }
};

// Device copy of count host values (zeros when h is NULL).
template <typename T>
static T *ref_up(RefBuf &b, const T *h, size_t count) {
    if (count == 0) count = 1;
    if (cudaMalloc(&b.p, count * sizeof(T)) != cudaSuccess) return nullptr;
    if (h)
        cudaMemcpy(b.p, h, count * sizeof(T), cudaMemcpyHostToDevice);
    else
        cudaMemset(b.p, 0, count * sizeof(T));
    return (T *)b.p;
}

template <typename T>
static void ref_down(T *h, const RefBuf &b, size_t count) {
    if (h) cudaMemcpy(h, b.p, count * sizeof(T), cudaMemcpyDeviceToHost);
}

// Copy back from a device pointer returned by ref_up (the safer form: the
// pointer names the buffer, so no index can pick the wrong one).
template <typename T>
static int ref_down_ptr(T *h, const T *d, size_t count) {
    if (!h) return 0;
    return cudaMemcpy(h, d, count * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 1;
}

// The reference's __constant__ physics (include/devconst.h), set from the
// runtime parameters in the reference's units (alpha in 1/cm).  Expanded in
// each launcher file because each reference .cu has its own copies.
#define REF_SET_CONSTANTS(p)                                                               \
    do {                                                                                   \
        double v_;                                                                         \
        cudaError_t e_;                                                                    \
        const double vals_[] = {(p)->dx,      (p)->dy,     (p)->dz,       (p)->dt,          \
                                (p)->sec_p_mm2dt_p_m, (p)->alpha / 100.0, (p)->porosity,   \
                                (p)->theta_s, (p)->theta_r, (p)->Ss,      (p)->n,           \
                                (p)->airdry,  (p)->psimin, (p)->am,       (p)->delta,       \
                                (p)->hmin,    (p)->hcri,   (p)->K0};                        \
        const void *syms_[] = {&dx,   &dy,      &dz,     &dt,    &sec_p_mm2dt_p_m, &alpha,   \
                               &poros, &theta_S, &theta_R, &Ss,  &n,   &air_dry, &psimin,  \
                               &am,   &delta,   &hmin,   &hcri,  &K0};                      \
        for (int q_ = 0; q_ < 18; ++q_) {                                                  \
            v_ = vals_[q_];                                                                \
            e_ = cudaMemcpyToSymbol(syms_[q_], &v_, sizeof(double));                       \
            if (e_ != cudaSuccess) return (int)e_;                                         \
        }                                                                                  \
    } while (0)
