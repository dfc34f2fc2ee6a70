// Host-side helpers shared by the translation units of libnkgpu.
#pragma once

#include <new>

#include "common.cuh"

namespace nkg {

// Makes `dev` current for the scope and restores the previous device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        NKG_CUDA(cudaGetDevice(&prev));
        if (prev != dev)
            NKG_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0)
            cudaSetDevice(prev);
    }
};

inline unsigned num_sms(int dev) {
    int v = 0;
    NKG_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    return static_cast<unsigned>(v);
}

template <typename T>
inline T read_scalar(const T *d, cudaStream_t s) {
    T h{};
    NKG_CUDA(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    return h;
}

// Run f, turning internal failures into an NKG_ERR_* code plus the
// thread-local message (the C-ABI convention).
template <typename F>
inline int guarded(F &&f) {
    try {
        f();
        return NKG_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return NKG_ERR_OOM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return NKG_ERR_CUDA;
    }
}

} // namespace nkg
