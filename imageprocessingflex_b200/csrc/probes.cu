// probes.cu -- run the kernels' scalar rules (border index, saturating store)
// on the device over caller-given values, so tests can check them one by one
// against ipf::borderIndex (core.hpp:187-214) and ipf::saturate_cast
// (core.hpp:69-103).
#include "../../include/ipfc.h"
#include "common.cuh"

namespace ipfc {
int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* fn);
}  // namespace ipfc

namespace {

__global__ void border_probe_kernel(const int* p, int* out, int n, int len, int border) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = ipfc::border_index(p[i], len, border);
}

template <typename T>
__global__ void saturate_probe_kernel(const float* v, T* out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = ipfc::sat_from_f<T>(v[i]);
}

}  // namespace

extern "C" {

int ipfc_probe_border_index(const int* p, int* out, int n, int len, int border, void* stream) {
    if (n < 0 || (n > 0 && (!p || !out))) return ipfc::set_error(IPFC_ERR_INVALID, "ipf: probe: invalid arguments");
    if (n == 0) return IPFC_OK;
    border_probe_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p, out, n, len, border);
    return ipfc::cuda_status(cudaGetLastError(), "probe");
}

int ipfc_probe_saturate(const float* v, void* out, int n, int to, void* stream) {
    if (n < 0 || (n > 0 && (!v || !out))) return ipfc::set_error(IPFC_ERR_INVALID, "ipf: probe: invalid arguments");
    if (n == 0) return IPFC_OK;
    const int g = (n + 255) / 256;
    cudaStream_t s = (cudaStream_t)stream;
    switch (to) {
        case IPFC_U8: saturate_probe_kernel<uint8_t><<<g, 256, 0, s>>>(v, (uint8_t*)out, n); break;
        case IPFC_U16: saturate_probe_kernel<uint16_t><<<g, 256, 0, s>>>(v, (uint16_t*)out, n); break;
        case IPFC_I16: saturate_probe_kernel<int16_t><<<g, 256, 0, s>>>(v, (int16_t*)out, n); break;
        case IPFC_F32: saturate_probe_kernel<float><<<g, 256, 0, s>>>(v, (float*)out, n); break;
        default: return ipfc::set_error(IPFC_ERR_UNSUPPORTED, "ipf: probe: unsupported type");
    }
    return ipfc::cuda_status(cudaGetLastError(), "probe");
}

}  // extern "C"
